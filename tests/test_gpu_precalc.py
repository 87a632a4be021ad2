"""Plans cached with the precalc writer and read back (the reference's
raw-binary cache, src/lib/inspiral_sky_map.c:1113-1811) integrate to the
same skies as the plans they came from, through the drop-in integrator and
the batched one (bit-identical tables: FP64 skies equal to 1e-15)."""
import ctypes as C

import numpy as np
import pytest

from sphradiometer_b200 import workload as W

pytestmark = pytest.mark.gpu


def test_cached_plans_integrate_like_the_originals(tmp_path):
    import torch
    import sphradiometer_b200 as S
    from sphradiometer_b200 import _abi as A
    L = S.load()
    pos = W.random_positions(3, W.R_EARTH_S, W.rng_for(2))
    n, dt, lm = 1024, 1.0 / 1024, 16
    net = S.Network(pos, n, dt, l_max=lm)
    root = str(tmp_path / "precalc").encode()
    assert L.make_precalc_directories(root, 3) == 0
    assert L.write_precalc_correlator_network_plan_fd(net.plan, net.plan, root) == 0
    nb = L.read_precalc_correlator_network_baselines(net._inst, root)
    assert nb
    P, N = A.correlator_network_plan_fd(), A.correlator_network_plan_fd()
    assert L.read_precalc_correlator_network_plan_fd(C.byref(P), C.byref(N), nb, n, root) == 0
    for k in range(3):
        assert np.array_equal(S.array_to_numpy(P.plans[k].contents.delay_product), net.delay_table(k))
        assert np.array_equal(S.rotation_plan_flat(P.plans[k].contents.rotation_plan), net.rotation_flat(k))
    b = W.make_batch(pos, n, dt, 4, seed=3)
    for s in range(4):
        F = W.full_from_half(b["F"][:, s, :], n)
        ref = net.integrate(F)
        Fc = [np.ascontiguousarray(f) for f in F]
        ptrs = (C.c_void_p * 3)(*[f.ctypes.data for f in Fc])
        sky = L.sh_series_new_zero(lm, 0)
        assert L.correlator_network_integrate_power_fd(sky, ptrs, C.byref(P))
        got = S.series_to_numpy(sky)
        L.sh_series_free(sky)
        assert np.max(np.abs(got - ref)) <= 1e-15 * np.max(np.abs(ref))
    # the batched integrator takes the cached plan as well
    bp = L.sphrad_batch_plan_new(C.byref(P), 0)
    assert bp
    bref = S.BatchPlan(net, "fp64")
    Fd = torch.from_numpy(np.ascontiguousarray(b["F"])).cuda()
    ws = torch.zeros(max(L.sphrad_batch_workspace_size(bp, 4), 16), dtype=torch.uint8, device="cuda")
    out = torch.empty((4, (lm + 1) ** 2), dtype=torch.complex128, device="cuda")
    assert L.sphrad_batch_integrate(bp, Fd.data_ptr(), 4, Fd.shape[2], None, out.data_ptr(), ws.data_ptr(), ws.numel(), None) == 0
    torch.cuda.synchronize()
    ref = bref.integrate(Fd).cpu().numpy()
    assert np.max(np.abs(out.cpu().numpy() - ref)) <= 1e-15 * np.max(np.abs(ref))
    L.sphrad_batch_plan_free(bp)
    bref.close()
    for k in range(3):
        L.correlator_plan_fd_free(P.plans[k])
        L.correlator_plan_fd_free(N.plans[k])
    L.correlator_network_baselines_free(nb)
    net.close()
