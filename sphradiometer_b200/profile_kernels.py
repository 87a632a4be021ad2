"""Drive one family of kernels on a bounded case, for profiling.

``python -m sphradiometer_b200.profile_kernels <stage> [--n N] [--calls C] [--method M]``

stages:
  render    64 x 128 FP32 sky grids of N c1 skies (k_sht_F, k_sht_pix)
  peaks     the reference localisation of N c1 skies (k_sht_pix argmax,
            k_peak_refine)
  rotate    N series at l_max 48 rotated by their own Euler angles, FP32
            application (k_euler, k_rotate_fac)
  product   N / 2 pairwise products at l_max 48, FP32 (k_sht_F, k_sht_pix,
            k_sht_H, k_sht_A)
  mlp       forward and backward passes of the proposal network on a batch
            of N (k_gemm and its epilogues)
  uneven    the uneven batch of N segments (gathers, k_tc_contract,
            k_epilogue_f32, k_uneven_combine), default split
  uneven_tuned  the same after autotuning, every call inside the NVTX
            range "final" (capture with --nvtx --nvtx-include "final/")
  fseries   3 x N c1 time series (n = 4096) to whitened half spectra
            (k_rfft_whiten)
  nonpolar  N segments through projected (non-polar) c1 plans on the
            tensor cores (k_np_build_a, k_np_tc)
  td        the time-domain network correlator on the reference's
            validation setup (4 detectors, 512 Hz, N = 32438 samples; host
            series): k_td_samples, k_td_cross, k_td_node, k_td_power

Each stage builds its inputs, runs once untimed, then ``--calls`` times and
prints the mean device time per call (CUDA events).
"""
from __future__ import annotations

import argparse

import numpy as np


def c1_skies(S, W, n):
    import torch
    pos = W.random_positions(3, W.R_EARTH_S, W.rng_for(2))
    net = S.Network(pos, 4096, 1.0 / 4096, l_max=32)
    bp = S.BatchPlan(net, "bf16x3")
    b = W.make_batch_torch(pos, 4096, 1.0 / 4096, n, seed=5)
    sky = bp.integrate(b["F"])
    torch.cuda.synchronize()
    return sky, (net, bp)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("stage", choices=["render", "peaks", "rotate", "product", "mlp", "uneven", "uneven_tuned", "fseries", "nonpolar", "td"])
    ap.add_argument("--n", type=int, default=4096)
    ap.add_argument("--calls", type=int, default=3)
    ap.add_argument("--method", type=int, default=-1, help="peaks: refinement method (0 trust-region Newton, 1 BFGS2; default: the library's)")
    args = ap.parse_args()
    import torch

    import sphradiometer_b200 as S
    from sphradiometer_b200 import workload as W

    keep = []
    n = args.n
    if args.stage == "render":
        sky, keep = c1_skies(S, W, n)
        g = S.SkyGrid(32, 64, 128, kind="cell", fp32=True)
        out = torch.empty((n, 64, 128), dtype=torch.float32, device="cuda")
        run = lambda: g.render(sky, out=out)  # noqa: E731
    elif args.stage == "peaks":
        sky, keep = c1_skies(S, W, n)
        if args.method >= 0 and S.load().sphrad_sky_set_refinement(args.method):
            raise SystemExit(f"refinement method {args.method}: not accepted")
        run = lambda: S.sky_peaks(sky)  # noqa: E731
    elif args.stage in ("rotate", "product"):
        L = 48
        rng = np.random.default_rng(48)
        nq = (L + 1) ** 2
        ls = np.concatenate([np.arange(abs(m), L + 1) for m in list(range(0, L + 1)) + list(range(-L, 0))])
        x = (rng.normal(size=(n, nq)) + 1j * rng.normal(size=(n, nq))) / (ls + 1.0) / np.sqrt(2)
        xd = torch.from_numpy(x).cuda()
        if args.stage == "rotate":
            R = []
            for _ in range(n):
                a, g_ = rng.uniform(0, 2 * np.pi, 2)
                b = np.arccos(rng.uniform(-1, 1))
                ca, sa, cb, sb, cg, sg = np.cos(a), np.sin(a), np.cos(b), np.sin(b), np.cos(g_), np.sin(g_)
                Rz1 = np.array([[ca, -sa, 0], [sa, ca, 0], [0, 0, 1]])
                Ry = np.array([[cb, 0, sb], [0, 1, 0], [-sb, 0, cb]])
                Rz2 = np.array([[cg, -sg, 0], [sg, cg, 0], [0, 0, 1]])
                R.append((Rz1 @ Ry @ Rz2).ravel())
            Rd = torch.from_numpy(np.array(R)).cuda()
            out = torch.empty_like(xd)
            run = lambda: S.rotate_batch(xd, Rd, L, fp32=True, out=out)  # noqa: E731
        else:
            grid = S.ProductGrid(L, L, L, fp32=True)
            keep = [grid]
            a_, b_ = xd[0::2].contiguous(), xd[1::2].contiguous()
            run = lambda: grid.multiply(a_, b_)  # noqa: E731
    elif args.stage == "mlp":
        p = S.Proposal(max_batch=n, seed=1)
        keep = [p]
        rng = np.random.default_rng(1)
        X = rng.normal(size=(n, p.N_FEATURES)).astype(np.float32)
        T = rng.normal(size=(n, 3))
        T = (T / np.linalg.norm(T, axis=1, keepdims=True)).astype(np.float32)
        Xd, Td = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
        run = lambda: p.train_step(Xd, Td, 1e-4)  # noqa: E731
    elif args.stage == "nonpolar":
        import ctypes as C
        pos = W.random_positions(3, W.R_EARTH_S, W.rng_for(2))
        net = S.Network(pos, 4096, 1.0 / 4096, l_max=32)
        rng = np.random.default_rng(3)
        fp, fc = W.pattern_meshes(32, 3, rng)
        psd = np.ascontiguousarray(rng.uniform(0.5, 2.0, size=(4096, 3)))
        rows = (C.POINTER(C.c_double) * 4096)(*[np.ctypeslib.as_ctypes(psd[j]) for j in range(4096)])
        assert S.load().sphrad_network_plan_mult_by_projection(net.plan, 1.0, fp.ctypes.data, fc.ctypes.data, C.cast(rows, C.c_void_p)) == 0
        bp = S.BatchPlan(net, "bf16x3")
        F = torch.from_numpy(np.ascontiguousarray(rng.normal(size=(3, n, 4096)) + 1j * rng.normal(size=(3, n, 4096)))).cuda()
        g = torch.rand(n, dtype=torch.float64, device="cuda")
        out = torch.empty((n, 33 * 33), dtype=torch.complex128, device="cuda")
        keep = [net, bp, rows]
        run = lambda: bp.integrate(F, g, out=out)  # noqa: E731
    elif args.stage == "td":
        rng = np.random.Generator(np.random.Philox(11))
        pos = W.random_positions(4, W.R_EARTH_S, rng)
        net = S.TimeDomainNetwork(pos, 1.0 / 512)
        ts = rng.normal(size=(4, n))
        wins = [np.full(n - 2 * net.transient(k), 1.0 / (n - 2 * net.transient(k))) for k in range(net.n_baselines)]
        keep = [net]
        run = lambda: net.integrate(ts, wins)  # noqa: E731
    elif args.stage == "fseries":
        pos = W.random_positions(3, W.R_EARTH_S, W.rng_for(2))
        b = W.make_tseries_batch(pos, 4096, 1.0 / 4096, 256, seed=5)
        x = torch.from_numpy(np.ascontiguousarray(b["x"][:, np.arange(n) % 256, :])).cuda()
        fp = S.FseriesPlan(4096, b["psd"])
        keep = [fp]
        out = torch.empty((3, n, 2049), dtype=torch.complex128, device="cuda")
        run = lambda: fp.transform(x, out=out)  # noqa: E731
    else:
        pos = W.random_positions(4, W.R_EARTH_S, W.rng_for(9))
        batch = W.make_uneven_batch(pos, n, seed=11)
        plan = S.UnevenPlan(pos, 1.0 / 4096, batch["buckets"], 48)
        plan.set_segments(batch["bucket"], batch["mask"], batch["l_max"])
        keep = [plan, batch]
        out = torch.empty(plan.out_total, dtype=torch.complex128, device="cuda")
        if args.stage == "uneven_tuned":
            plan.autotune(batch["spectra"], out)
        plan.use_graph(False)

        def run():
            if args.stage == "uneven_tuned":
                torch.cuda.nvtx.range_push("final")
            plan.integrate(batch["spectra"], out=out)
            if args.stage == "uneven_tuned":
                torch.cuda.nvtx.range_pop()
    run()
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    for _ in range(args.calls):
        run()
    b.record(st)
    torch.cuda.synchronize()
    print(f"{args.stage}: n {n}, {a.elapsed_time(b) / args.calls:.4f} ms per call")
    del keep


if __name__ == "__main__":
    main()
