"""The allocation-free batched entry point (sphrad_batch_integrate_noalloc).

Some callers cannot allocate device memory while they run (real-time
pipelines that cannot risk the synchronisation of cudaMalloc/cudaFree,
hosts that own all device memory, plug-ins whose host forbids allocation).
This entry point integrates with its split-K scratch in a static device
array instead of a caller workspace.  The test calls it twice in a row
through the C ABI and checks each result against the workspace entry point
(sphrad_batch_integrate) on the same inputs, with the tolerance the bf16x3
parity tests use; it also checks that a batch too large for the array is
refused with an error before any device work, and that the second call
leaves the device's free memory and torch's allocations unchanged (the
first call on a device may load the library's module, which places the
static array).  This file is collected last so a stop-at-first-failure run
has already run every other test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-5  # relative L2, the bf16x3 batch tolerance of test_gpu_parity.py


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_noalloc_matches_workspace_entry_point_on_two_calls():
    import torch

    import sphradiometer_b200 as S
    from sphradiometer_b200 import workload as W

    L = S.load()
    n, dt, l_max, n_seg = 4096, 1.0 / 4096, 32, 300
    pos = W.random_positions(3, W.R_EARTH_S, W.rng_for(2))
    net = S.Network(pos, n, dt, l_max=l_max)
    bp = S.BatchPlan(net, "bf16x3")
    batch = W.make_batch(pos, n, dt, n_seg, seed=31)
    F = torch.from_numpy(np.ascontiguousarray(batch["F"])).cuda()
    g = torch.from_numpy(batch["gmst"]).cuda()
    ref = bp.integrate(F, g).cpu().numpy()
    stream = torch.cuda.current_stream()
    nq = (l_max + 1) ** 2
    outs = [torch.full((n_seg, nq), float("nan"), dtype=torch.complex128, device="cuda") for _ in range(2)]
    torch.cuda.synchronize()
    for k, out in enumerate(outs):
        if k == 1:
            free0, alloc0 = torch.cuda.mem_get_info()[0], torch.cuda.memory_allocated()
        rc = L.sphrad_batch_integrate_noalloc(bp._p, F.data_ptr(), n_seg, F.shape[2], g.data_ptr(), out.data_ptr(), stream.cuda_stream)
        assert rc == 0, S.last_error()
        torch.cuda.synchronize()
        if k == 1:
            # the second call allocated no device memory
            assert torch.cuda.mem_get_info()[0] == free0
            assert torch.cuda.memory_allocated() == alloc0
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert rel_l2(got, ref) < TOL
        assert max(rel_l2(got[s], ref[s]) for s in range(n_seg)) < 3 * TOL
    assert bp.status() == 0

    # a batch beyond the static array is refused up front
    rc = L.sphrad_batch_integrate_noalloc(bp._p, F.data_ptr(), 1_000_000, F.shape[2], g.data_ptr(), outs[0].data_ptr(), stream.cuda_stream)
    assert rc == -1
    msg = S.last_error()
    assert "scratch" in msg
    # the message names this plan's limit: 8 MiB over 3 x 36 FP32 partial sums per segment
    assert "at most 19418 segments" in msg, msg
    bp.close()
    net.close()
