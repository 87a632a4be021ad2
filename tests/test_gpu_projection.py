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


class LALDetector(C.Structure):
    # the leading members of LAL's LALDetector (vertex in metres, response tensor)
    _fields_ = [("location", C.c_double * 3), ("response", (C.c_float * 3) * 3)]


def lal_like_detector(theta, phi, azimuth):
    """A detector on the Earth's surface at co-latitude theta, longitude
    phi: perpendicular arms along azimuth and azimuth + 90 deg in the local
    horizontal plane, response tensor (x x^T - y y^T) / 2."""
    R = 6.371e6
    r = np.array([np.sin(theta) * np.cos(phi), np.sin(theta) * np.sin(phi), np.cos(theta)])
    e_t = np.array([np.cos(theta) * np.cos(phi), np.cos(theta) * np.sin(phi), -np.sin(theta)])
    e_p = np.array([-np.sin(phi), np.cos(phi), 0.0])
    x = np.cos(azimuth) * e_t + np.sin(azimuth) * e_p
    y = -np.sin(azimuth) * e_t + np.cos(azimuth) * e_p
    d = LALDetector()
    for i in range(3):
        d.location[i] = R * r[i]
    D = 0.5 * (np.outer(x, x) - np.outer(y, y))
    for i in range(3):
        for j in range(3):
            d.response[i][j] = float(D[i, j])
    return d


def am_response(D, ra, dec, psi, gmst):
    """The published detector response (Anderson et al. 2001, PRD 63 042003,
    app. B), in numpy."""
    h = gmst - ra
    X = np.array([-np.cos(psi) * np.sin(h) - np.sin(psi) * np.cos(h) * np.sin(dec),
                  -np.cos(psi) * np.cos(h) + np.sin(psi) * np.sin(h) * np.sin(dec), np.sin(psi) * np.cos(dec)])
    Y = np.array([np.sin(psi) * np.sin(h) - np.cos(psi) * np.cos(h) * np.sin(dec),
                  np.sin(psi) * np.cos(h) + np.cos(psi) * np.sin(h) * np.sin(dec), np.cos(psi) * np.cos(dec)])
    return X @ D @ X - Y @ D @ Y, X @ D @ Y + Y @ D @ X


def test_reference_named_projection_uses_detector_responses():
    """correlator_network_plan_mult_by_projection (inspiral_sky_map.c:423-549)
    with instruments made by instrument_new_from_LALDetector equals the
    mesh-taking variant fed the same antenna patterns computed in numpy from
    the response tensors at the reference's call (:357: phi as right
    ascension, pi/2 - theta as declination, gmst 0)."""
    import sphradiometer_b200 as S
    L_ = S.load()
    dets = [lal_like_detector(0.9, 0.3, 0.2), lal_like_detector(1.4, 2.1, 1.1), lal_like_detector(2.0, -1.2, 2.5)]
    n, dt, L, beta, psi = 256, 1.0 / 2048, 6, 0.6, 0.35
    rng = np.random.default_rng(5)
    psd = rng.uniform(0.5, 2.0, size=(n, 3))
    rows = (C.POINTER(C.c_double) * n)(*[np.ctypeslib.as_ctypes(psd[j]) for j in range(n)])

    def network():
        arr = L_.instrument_array_new(0)
        for d in dets:
            assert L_.instrument_array_append(arr, L_.instrument_new_from_LALDetector(C.byref(d)))
        bl = L_.correlator_network_baselines_new(arr)
        plan = L_.correlator_network_plan_fd_new_l(bl, n, dt, L)
        assert plan, S.last_error()
        return arr, bl, plan

    a_arr, a_bl, a_plan = network()
    assert L_.correlator_network_plan_mult_by_projection(a_plan, beta, psi, C.cast(rows, C.c_void_p)) == 0, S.last_error()
    # the same patterns from numpy
    nt = 2 * (L + 1)
    x, _ = O.gl_nodes(nt)
    fp = np.zeros((3, nt, nt))
    fc = np.zeros((3, nt, nt))
    for k, d in enumerate(dets):
        D = np.array([[d.response[i][j] for j in range(3)] for i in range(3)], dtype=np.float64)
        for i in range(nt):
            for j in range(nt):
                fp[k, i, j], fc[k, i, j] = am_response(D, 2 * np.pi * j / nt, np.pi / 2 - np.arccos(x[i]), psi, 0.0)
    b_arr, b_bl, b_plan = network()
    assert L_.sphrad_network_plan_mult_by_projection(b_plan, beta, np.ascontiguousarray(fp).ctypes.data, np.ascontiguousarray(fc).ctypes.data,
                                                     C.cast(rows, C.c_void_p)) == 0, S.last_error()
    for k in range(3):
        da = S.array_to_numpy(a_plan.contents.plans[k].contents.delay_product)
        db = S.array_to_numpy(b_plan.contents.plans[k].contents.delay_product)
        assert np.max(np.abs(da - db)) <= 1e-12 * np.max(np.abs(db)), k
    for plan, bl, arr in ((a_plan, a_bl, a_arr), (b_plan, b_bl, b_arr)):
        L_.correlator_network_plan_fd_free(plan)
        L_.correlator_network_baselines_free(bl)
        L_.instrument_array_free(arr)
