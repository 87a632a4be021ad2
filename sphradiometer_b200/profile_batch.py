"""Run the batched cross-power integration on the c1 network for profiling.

``python -m sphradiometer_b200.profile_batch --segments 2048 --calls 5``
builds the 3-detector, 4096 Hz, l_max = 32 plan, uploads one seeded batch
and calls the batched integrator ``--calls`` times (after the split-K
choice), printing the mean device time per call; ``--graph N`` captures N
calls into a CUDA graph once and replays it ``--calls`` times.  Used to
drive ncu captures of one kernel on a bounded case.
"""
from __future__ import annotations

import argparse

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--segments", type=int, default=2048)
    ap.add_argument("--calls", type=int, default=5)
    ap.add_argument("--precision", default="bf16x3")
    ap.add_argument("--split", type=int, default=0)
    ap.add_argument("--autotune", action="store_true", help="use the autotuned split-K and pipeline variant")
    ap.add_argument("--ctas", type=int, default=0, help="pin the tcgen05 contraction's CTA count")
    ap.add_argument("--pipeline", type=int, default=-1, help="pin the tcgen05 pipeline variant (0, 1, 2)")
    ap.add_argument("--graph", type=int, default=0, help="capture this many calls into a CUDA graph and time --calls replays of it")
    args = ap.parse_args()
    import torch

    import sphradiometer_b200 as S
    from sphradiometer_b200 import workload as W

    n, dt, L = 4096, 1.0 / 4096, 32
    pos = W.random_positions(3, W.R_EARTH_S, W.rng_for(2))
    net = S.Network(pos, n, dt, l_max=L)
    bp = S.BatchPlan(net, args.precision)
    base = W.make_batch(pos, n, dt, min(args.segments, 512), seed=11)
    idx = np.arange(args.segments) % base["F"].shape[1]
    F = torch.from_numpy(np.ascontiguousarray(base["F"][:, idx, :])).cuda()
    g = torch.from_numpy(base["gmst"][idx].copy()).cuda()
    if args.autotune:
        bp.autotune(F)
    elif args.split:
        bp.set_split(args.segments, args.split)
    if args.ctas:
        bp.set_ctas(args.segments, args.ctas)
    if args.pipeline >= 0:
        bp.set_pipeline(args.segments, args.pipeline)
    out = bp.integrate(F, g)
    torch.cuda.synchronize()
    run = lambda: bp.integrate(F, g, out=out)  # noqa: E731
    per = 1
    if args.graph > 0:
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            for _ in range(args.graph):
                bp.integrate(F, g, out=out)
        run = graph.replay
        per = args.graph
        run()
        torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(args.calls):
        run()
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / (args.calls * per)
    print(f"segments {args.segments} split {bp.split(args.segments)} ctas {bp.ctas(args.segments) if args.precision.startswith('bf16') else '-'} "
          f"variant {bp.pipeline(args.segments)} "
          f"precision {args.precision}: {ms:.4f} ms/call, "
          f"{args.segments / ms * 1e3:.3e} maps/s, status {bp.status()}")


if __name__ == "__main__":
    main()
