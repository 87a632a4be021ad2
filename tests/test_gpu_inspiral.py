"""Sky maps of the inspiral path (generate_alm_sky / generate_alm_skys,
src/lib/inspiral_sky_map.c:869-1101) and the complex-series transform they
start from (correlator_ctseries_to_fseries, src/lib/correlator.c:235-244),
through the C ABI, against the oracle: its DFT, its rotations, and the
projected kernels that the projection tests check against the oracle.

Tolerances: FP64 1e-12 of the largest value; the batched FP32 and bf16x3
integrations 1e-5 (relative L2 per sky), as in the projection tests."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from sphradiometer_b200 import workload as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [8, 16, 64, 512, 4096, 8192])
def test_complex_transform_matches_oracle_dft(n):
    import torch
    import sphradiometer_b200 as S
    rng = np.random.default_rng(n)
    rows = 5
    z = rng.normal(size=(rows, n)) + 1j * rng.normal(size=(rows, n))
    fp = S.FseriesPlan(n)
    got = fp.transform_complex(torch.from_numpy(z).cuda()).cpu().numpy()
    ref = np.array([O.dft(z[r], -1) for r in range(rows)]) if n <= 512 else np.fft.fft(z, axis=1)
    assert np.max(np.abs(got - ref)) <= 1e-13 * np.max(np.abs(ref))
    assert np.max(np.abs(fp.transform_complex_host(z[2]) - ref[2])) <= 1e-13 * np.max(np.abs(ref[2]))
    fp.close()


def test_complex_transform_limits():
    """Complex transforms take n <= 8192 (one CTA per series); above that
    the call fails and says so."""
    import sphradiometer_b200 as S
    fp = S.FseriesPlan(16384)
    with pytest.raises(S.SphradError, match="8192"):
        fp.transform_complex_host(np.zeros(16384, complex))
    fp.close()


def _projected_network(pos, n, dt, L, beta, fp, fc, psd):
    import sphradiometer_b200 as S
    net = S.Network(pos, n, dt, l_max=L)
    rows = (C.POINTER(C.c_double) * n)(*[np.ctypeslib.as_ctypes(psd[j]) for j in range(n)])
    assert S.load().sphrad_network_plan_mult_by_projection(net.plan, beta, fp.ctypes.data, fc.ctypes.data, C.cast(rows, C.c_void_p)) == 0, S.last_error()
    return net


def _oracle_sky(net, F, n, L, gmst, logprior):
    """generate_alm_sky on oracle pieces: each baseline's (F_j conj F_i) D / n
    rotated with the oracle's plan, the network mean, x 2 x 4 B, + prior,
    rotate_z."""
    B = net.n_baselines
    sky = np.zeros((L + 1) ** 2, complex)
    k = 0
    for i in range(1, 3):
        for j in range(i):
            bl = net.baseline(k)
            Pk = (F[j] * np.conj(F[i])) @ net.delay_table(k) / n
            sky += O.rotate(Pk, L, False, O.rotation_plan(L, O.rot_matrix(bl.theta, bl.phi))) / B
            k += 1
    return O.rotate_z(8.0 * B * sky + logprior, L, False, gmst)


def test_generate_alm_skys_match_oracle_and_batch():
    import torch
    import sphradiometer_b200 as S
    rng = np.random.default_rng(21)
    pos = W.random_positions(3, 0.02, W.rng_for(8))
    n, dt, L = 64, 1.0 / 256, 5
    nt = 2 * (L + 1)
    x, _ = O.gl_nodes(nt)
    th = np.arccos(x)[:, None]
    ph = 2 * np.pi * np.arange(nt)[None, :] / nt
    c = rng.uniform(0, 2 * np.pi, 3)
    fp = np.ascontiguousarray(np.stack([0.5 * (1 + np.cos(th) ** 2) * np.cos(2 * ph + c[k]) + 0.1 * k for k in range(3)]))
    fc = np.ascontiguousarray(np.stack([np.cos(th) * np.sin(2 * ph + c[k]) for k in range(3)]))
    psd = rng.uniform(0.5, 2.0, size=(n, 3))
    net_p = _projected_network(pos, n, dt, L, 0.8, fp, fc, psd)
    net_n = _projected_network(pos, n, dt, L, -0.8, fp, fc, psd)
    logprior = (rng.normal(size=(L + 1) ** 2) + 1j * rng.normal(size=(L + 1) ** 2)) * 0.1
    n_ev = 37
    z = rng.normal(size=(3, n_ev, n)) + 1j * rng.normal(size=(3, n_ev, n))
    gm = rng.uniform(0, 2 * np.pi, n_ev)
    # the drop-in entry point, event by event, against the oracle
    host_p, host_n = [], []
    for e in (0, 5, 36):
        sp, sn = S.generate_alm_skys(net_p, net_n, z[:, e, :], gm[e], logprior)
        F = np.stack([O.dft(z[k, e], -1) for k in range(3)])
        rp = _oracle_sky(net_p, F, n, L, gm[e], logprior)
        rn = _oracle_sky(net_n, F, n, L, gm[e], logprior)
        assert np.max(np.abs(sp - rp)) <= 1e-12 * np.max(np.abs(rp))
        assert np.max(np.abs(sn - rn)) <= 1e-12 * np.max(np.abs(rn))
        assert np.max(np.abs(sp - sn)) > 1e-6 * np.max(np.abs(sp))  # the two signs differ
    refs_p, refs_n = [], []
    for e in range(n_ev):
        F = np.stack([O.dft(z[k, e], -1) for k in range(3)])
        refs_p.append(_oracle_sky(net_p, F, n, L, gm[e], logprior))
        refs_n.append(_oracle_sky(net_n, F, n, L, gm[e], logprior))
    refs_p, refs_n = np.array(refs_p), np.array(refs_n)
    # the batched entry point, all events at once
    fplan = S.FseriesPlan(n)
    zt = torch.from_numpy(np.ascontiguousarray(z)).cuda()
    gt = torch.from_numpy(gm).cuda()
    pt = torch.from_numpy(logprior).cuda()
    for prec, tol in (("fp64", 1e-12), ("fp32", 1e-5), ("bf16x3", 1e-5)):
        bp, bn = S.BatchPlan(net_p, prec), S.BatchPlan(net_n, prec)
        gp, gn = S.batch_generate_alm_skys(bp, bn, fplan, zt, gt, pt)
        gp, gn = gp.cpu().numpy(), gn.cpu().numpy()
        for got, ref in ((gp, refs_p), (gn, refs_n)):
            worst = max(np.linalg.norm(got[e] - ref[e]) / np.linalg.norm(ref[e]) for e in range(n_ev))
            assert worst < tol, (prec, worst)
        assert bp.status() == 0 and bn.status() == 0
        bp.close()
        bn.close()
    fplan.close()
    net_p.close()
    net_n.close()
