"""GPU parity of the projection operator of the inspiral path
(correlator_network_plan_mult_by_projection, src/lib/inspiral_sky_map.c:
423-549) against a numpy restatement on the oracle's transforms, rotations
and products, and of the resulting non-polar plans in the drop-in
integrator.

Tolerances: FP64 throughout, 1e-12 of the largest coefficient (the
transforms, rotations and products are each pinned at that level in the
other tests)."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from sphradiometer_b200 import workload as W

pytestmark = pytest.mark.gpu


def patterns(L, n_det, rng):
    """Smooth stand-ins for F+ and Fx of each detector on the reference
    mesh of L (rows acos of the decreasing GL nodes, columns 2 pi j / np)."""
    nt = 2 * (L + 1)
    x, _ = O.gl_nodes(nt)
    th = np.arccos(x)[:, None]
    ph = 2 * np.pi * np.arange(nt)[None, :] / nt
    c = rng.uniform(0, 2 * np.pi, n_det)
    fp = np.stack([0.5 * (1 + np.cos(th) ** 2) * np.cos(2 * ph + c[k]) + 0.1 * k for k in range(n_det)])
    fc = np.stack([np.cos(th) * np.sin(2 * ph + c[k]) for k in range(n_det)])
    return np.ascontiguousarray(fp), np.ascontiguousarray(fc)


def test_projection_plan_and_integration_match_numpy():
    import sphradiometer_b200 as S
    L_ = S.load()
    rng = np.random.default_rng(12)
    pos = W.random_positions(3, 0.02, W.rng_for(7))
    n, dt, L = 64, 1.0 / 256, 5
    net = S.Network(pos, n, dt, l_max=L)
    assert all(net.baseline_l_max(k) == L for k in range(3))
    D0 = [net.delay_table(k).copy() for k in range(3)]
    fp, fc = patterns(L, 3, rng)
    psd = rng.uniform(0.5, 2.0, size=(n, 3))
    rows = (C.POINTER(C.c_double) * n)(*[np.ctypeslib.as_ctypes(psd[j]) for j in range(n)])
    beta = 0.7
    assert L_.sphrad_network_plan_mult_by_projection(net.plan, beta, fp.ctypes.data, fc.ctypes.data, C.cast(rows, C.c_void_p)) == 0, S.last_error()

    pairs = [(1, 0), (2, 0), (2, 1)]
    for k, (a, b) in enumerate(pairs):
        bl = net.baseline(k)
        assert (bl.index_a, bl.index_b) == (a, b)
        got = net.delay_table(k)
        assert got.shape == (n, (L + 1) ** 2)
        # the inverse rotation: the transpose of the (flat, row-major) matrix
        Rinv = np.asarray(O.rot_matrix(bl.theta, bl.phi)).reshape(3, 3).T.ravel()
        Rot_inv = O.rotation_plan(L, Rinv)
        ref = np.empty_like(got)
        for j in range(n):
            u = (fp + 1j * beta * fc) / psd[j][:, None, None]
            norm = np.sum((fp / psd[j][:, None, None]) ** 2 + beta ** 2 * (fc / psd[j][:, None, None]) ** 2, axis=0)
            P = u[a] * np.conj(u[b]) / norm
            proj = O.rotate(O.from_mesh(P, L, False), L, False, Rot_inv)
            ref[j] = O.product_microcode(D0[k][j], L, True, proj, L, False, L, False)
        assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref)), (k, np.max(np.abs(got - ref)))
        pw = net.plan_fd(k).contents.power_1d.contents
        assert pw.polar == 0 and pw.l_max == L
        assert np.max(np.abs(net.rotation_flat(k) - O.rotation_plan(L, O.rot_matrix(bl.theta, bl.phi)))) < 1e-12

    # the drop-in integrator on the projected (non-polar) plans
    F = rng.normal(size=(3, n)) + 1j * rng.normal(size=(3, n))
    sky = net.integrate(F)
    ref = np.zeros((L + 1) ** 2, complex)
    for k, (i, j) in enumerate(pairs):
        bl = net.baseline(k)
        Pk = (F[j] * np.conj(F[i])) @ net.delay_table(k) / n
        ref += O.rotate(Pk, L, False, O.rotation_plan(L, O.rot_matrix(bl.theta, bl.phi))) / 3
    assert np.max(np.abs(sky - ref)) <= 1e-12 * np.max(np.abs(ref))

    # the batched integrator on the projected plans: full (non-Hermitian)
    # spectra of many segments, GMST phases, FP64 and FP32
    import torch
    Sg = 70
    Fb = rng.normal(size=(3, Sg, n)) + 1j * rng.normal(size=(3, Sg, n))
    gm = rng.uniform(0, 2 * np.pi, Sg)
    refs = np.array([O.rotate_z(net.integrate(Fb[:, s, :]), L, False, gm[s]) for s in range(Sg)])
    for prec, tol in (("fp64", 1e-12), ("fp32", 1e-5), ("bf16x3", 1e-5)):
        bp = S.BatchPlan(net, prec)
        assert bp.l_max == L and bp.bins == n
        got = bp.integrate(torch.from_numpy(np.ascontiguousarray(Fb)).cuda(), torch.from_numpy(gm).cuda()).cpu().numpy()
        err = np.linalg.norm(got - refs) / np.linalg.norm(refs)
        worst = max(np.linalg.norm(got[s] - refs[s]) / np.linalg.norm(refs[s]) for s in range(Sg))
        assert err < tol and worst < 3 * tol, (prec, err, worst)
        assert bp.status() == 0
        bp.close()
    with pytest.raises(S.SphradError):
        S.BatchPlan(net, "bf16x6")
    net.close()


def test_projection_refuses_mixed_plans():
    import sphradiometer_b200 as S
    L_ = S.load()
    pos = W.random_positions(3, 0.02, W.rng_for(7))
    net = S.Network(pos, 64, 1.0 / 256, l_max=5)
    fp = np.ones((3, 12, 12))
    psd = np.ones((64, 3))
    rows = (C.POINTER(C.c_double) * 64)(*[np.ctypeslib.as_ctypes(psd[j]) for j in range(64)])
    assert L_.sphrad_network_plan_mult_by_projection(net.plan, 1.0, fp.ctypes.data, fp.ctypes.data, C.cast(rows, C.c_void_p)) == 0
    # a second projection needs polar kernels: refused
    assert L_.sphrad_network_plan_mult_by_projection(net.plan, 1.0, fp.ctypes.data, fp.ctypes.data, C.cast(rows, C.c_void_p)) < 0
    net.close()


def test_nonpolar_tensor_core_path_across_tiles():
    """The bf16x3 path of projected plans over several 128-segment tiles,
    two 256-column tiles and 24 K stages, against the FP64 batched path
    (itself checked against the drop-in integrator above)."""
    import torch
    import sphradiometer_b200 as S
    L_ = S.load()
    rng = np.random.default_rng(21)
    pos = W.random_positions(3, 0.02, W.rng_for(7))
    n, dt, L = 256, 1.0 / 512, 12
    net = S.Network(pos, n, dt, l_max=L)
    assert all(net.baseline_l_max(k) == L for k in range(3))
    fp, fc = W.pattern_meshes(L, 3, rng)
    psd = rng.uniform(0.5, 2.0, size=(n, 3))
    rows = (C.POINTER(C.c_double) * n)(*[np.ctypeslib.as_ctypes(psd[j]) for j in range(n)])
    assert L_.sphrad_network_plan_mult_by_projection(net.plan, 0.4, fp.ctypes.data, fc.ctypes.data, C.cast(rows, C.c_void_p)) == 0
    Sg = 300
    Fb = torch.from_numpy(np.ascontiguousarray(rng.normal(size=(3, Sg, n)) + 1j * rng.normal(size=(3, Sg, n)))).cuda()
    gm = torch.from_numpy(rng.uniform(0, 2 * np.pi, Sg)).cuda()
    ref = S.BatchPlan(net, "fp64")
    r = ref.integrate(Fb, gm).cpu().numpy()
    bp = S.BatchPlan(net, "bf16x3")
    got = bp.integrate(Fb, gm).cpu().numpy()
    again = bp.integrate(Fb, gm).cpu().numpy()
    err = np.linalg.norm(got - r) / np.linalg.norm(r)
    worst = max(np.linalg.norm(got[s] - r[s]) / np.linalg.norm(r[s]) for s in range(Sg))
    assert err < 1e-5 and worst < 3e-5, (err, worst)
    assert np.array_equal(got, again)  # no atomics: every call is bit-identical
    assert bp.status() == 0
    bp.close()
    ref.close()
    net.close()
