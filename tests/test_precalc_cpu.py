"""The precalculated-plan cache in the reference's raw-binary format
(src/lib/inspiral_sky_map.c:1113-1811), read and written on the host.

The tree below is built byte by byte here, field by field in the order the
reference's reader takes them (fread of int index_a, int index_b, double
theta, double phi per baseline, :1130-1133; double delta_t, int transient
per plan, :1246-1247; unsigned l_max then the (2l+1)^2 complex matrices of
l = 1 .. l_max, :1203-1219; unsigned l_max, int polar, int n, int stride and
the n * stride coefficients of each delay table, :1277-1283), so the test
pins the format, not just a round trip of this library's own writer.
"""
import ctypes as C
import os
import struct

import numpy as np
import pytest


@pytest.fixture(scope="module")
def L():
    from sphradiometer_b200 import _abi
    return _abi.load()


def instruments(L, pos):
    arr = L.instrument_array_new(0)
    for p in pos:
        L.instrument_array_append(arr, L.instrument_new(float(p[0]), float(p[1]), float(p[2]), None))
    return arr


def write_tree(root, baselines, plans, tlen):
    """baselines: [(a, b, theta, phi)]; plans: [(delta_t, transient, rot, Dp, Dn, l_max, polar)]"""
    net = os.path.join(root, "correlator_network_plan_fd")
    os.makedirs(os.path.join(net, "correlator_network_baselines", "baselines"))
    with open(os.path.join(net, "correlator_network_baselines", "n_baselines.dat"), "wb") as f:
        f.write(struct.pack("=i", len(baselines)))
    for i, (a, b, th, ph) in enumerate(baselines):
        d = os.path.join(net, "correlator_network_baselines", "baselines", str(i))
        os.makedirs(d)
        with open(os.path.join(d, "correlator_baseline.dat"), "wb") as f:
            f.write(struct.pack("=iidd", a, b, th, ph))
    for i, (dt, tr, rot, Dp, Dn, lm, polar) in enumerate(plans):
        d = os.path.join(net, "correlator_plan_fd", str(i))
        for sub in ("rotation_plan", "delay_product_p", "delay_product_n"):
            os.makedirs(os.path.join(d, sub))
        with open(os.path.join(d, "correlator_plan_fd.dat"), "wb") as f:
            f.write(struct.pack("=di", dt, tr))
        with open(os.path.join(d, "rotation_plan", "l_max.dat"), "wb") as f:
            f.write(struct.pack("=I", len(rot)))
        with open(os.path.join(d, "rotation_plan", "D.dat"), "wb") as f:
            for M in rot:
                f.write(np.ascontiguousarray(M, np.complex128).tobytes())
        for sub, D in (("delay_product_p", Dp), ("delay_product_n", Dn)):
            with open(os.path.join(d, sub, "sh_series_array.dat"), "wb") as f:
                f.write(struct.pack("=Iiii", lm, polar, D.shape[0], D.shape[1]))
                f.write(np.ascontiguousarray(D, np.complex128).tobytes())
    with open(os.path.join(root, "time_series_length.dat"), "wb") as f:
        f.write(struct.pack("=I", tlen))


def carray(ptr, n):
    return np.ctypeslib.as_array((C.c_double * (2 * n)).from_address(ptr)).view(np.complex128).copy()


def test_reads_the_reference_layout_and_writes_it_back(L, tmp_path):
    from sphradiometer_b200 import _abi as A
    rng = np.random.default_rng(4)
    pos = rng.normal(size=(3, 3)) * 0.01
    inst = instruments(L, pos)
    nb_ref = L.correlator_network_baselines_new(inst).contents
    baselines, plans = [], []
    n, lm, tlen = 16, 3, 16
    for i in range(nb_ref.n_baselines):
        b = nb_ref.baselines[i].contents
        baselines.append((b.index_a, b.index_b, b.theta, b.phi))
        rot = [rng.normal(size=(2 * l + 1, 2 * l + 1)) + 1j * rng.normal(size=(2 * l + 1, 2 * l + 1)) for l in range(1, lm + 1)]
        polar = i % 2
        stride = lm + 1 if polar else (lm + 1) ** 2
        Dp = rng.normal(size=(n, stride)) + 1j * rng.normal(size=(n, stride))
        Dn = rng.normal(size=(n, stride)) + 1j * rng.normal(size=(n, stride))
        plans.append((1.0 / 2048 * (i + 1), 7 + i, rot, Dp, Dn, lm, polar))
    root = str(tmp_path / "pre")
    write_tree(root, baselines, plans, tlen)

    length = C.c_uint(0)
    assert L.read_precalc_time_series_length(C.byref(length), root.encode()) == 0 and length.value == tlen
    nb = L.read_precalc_correlator_network_baselines(inst, root.encode())
    assert nb, _abi_err()
    P, N = A.correlator_network_plan_fd(), A.correlator_network_plan_fd()
    assert L.read_precalc_correlator_network_plan_fd(C.byref(P), C.byref(N), nb, tlen, root.encode()) == 0, _abi_err()
    for i, (dt, tr, rot, Dp, Dn, lm_, polar) in enumerate(plans):
        for plan, D in ((P.plans[i].contents, Dp), (N.plans[i].contents, Dn)):
            assert plan.delta_t == dt and plan.transient == tr
            a = plan.delay_product.contents
            assert (a.l_max, a.polar, a.n, a.stride) == (lm_, polar, n, D.shape[1])
            assert np.array_equal(carray(a.coeff, n * a.stride).reshape(n, -1), D)
            assert plan.power_1d.contents.l_max == lm_ and plan.power_1d.contents.polar == polar
            rp = plan.rotation_plan
            assert rp.contents.l_max == lm_
            for l in range(1, lm_ + 1):
                for m in range(-l, l + 1):
                    for mp in (-l, 0, l):
                        z = L.sh_series_rotation_plan_wigner_D(rp, l, m, mp)
                        ref = rot[l - 1].ravel()[(2 * l + 1) * (mp + l) + (m + l)]
                        assert complex(z.re, z.im) == ref
        b = nb.contents.baselines[i].contents
        assert (b.index_a, b.index_b, b.theta, b.phi) == baselines[i]

    # written back in the same format: every file byte-identical, plus d.dat
    out = str(tmp_path / "out")
    assert L.make_precalc_directories(out.encode(), 3) == 0
    assert L.make_precalc_directories(out.encode(), 3) < 0  # the tree must be new
    assert L.write_precalc_correlator_network_plan_fd(C.byref(P), C.byref(N), out.encode()) == 0, _abi_err()
    assert L.write_precalc_time_series_length(tlen, out.encode()) == 0
    for dirpath, _, files in os.walk(root):
        for fn in files:
            rel = os.path.relpath(os.path.join(dirpath, fn), root)
            with open(os.path.join(root, rel), "rb") as f1, open(os.path.join(out, rel), "rb") as f2:
                assert f1.read() == f2.read(), rel
    for i in range(len(baselines)):
        b = nb.contents.baselines[i].contents
        d = np.fromfile(os.path.join(out, "correlator_network_plan_fd", "correlator_network_baselines", "baselines", str(i), "d.dat"))
        assert np.array_equal(d, pos[b.index_a] - pos[b.index_b]) or np.allclose(d, pos[b.index_a] - pos[b.index_b], rtol=0, atol=1e-18)


def test_rejects_a_cache_of_other_instruments(L, tmp_path):
    rng = np.random.default_rng(5)
    pos = rng.normal(size=(2, 3)) * 0.01
    inst = instruments(L, pos)
    nb_ref = L.correlator_network_baselines_new(inst).contents.baselines[0].contents
    root = str(tmp_path / "pre")
    write_tree(root, [(nb_ref.index_a, nb_ref.index_b, nb_ref.theta + 1e-3, nb_ref.phi)],
               [(1.0 / 1024, 3, [np.eye(3, dtype=complex)], np.zeros((4, 2), complex), np.zeros((4, 2), complex), 1, 1)], 4)
    assert not L.read_precalc_correlator_network_baselines(inst, root.encode())
    # a truncated delay table is refused
    good = str(tmp_path / "good")
    write_tree(good, [(nb_ref.index_a, nb_ref.index_b, nb_ref.theta, nb_ref.phi)],
               [(1.0 / 1024, 3, [np.eye(3, dtype=complex)], np.zeros((4, 2), complex), np.zeros((4, 2), complex), 1, 1)], 4)
    f = os.path.join(good, "correlator_network_plan_fd", "correlator_plan_fd", "0", "delay_product_n", "sh_series_array.dat")
    with open(f, "r+b") as fh:
        fh.truncate(os.path.getsize(f) - 16)
    from sphradiometer_b200 import _abi as A
    nb = L.read_precalc_correlator_network_baselines(inst, good.encode())
    assert nb
    P, N = A.correlator_network_plan_fd(), A.correlator_network_plan_fd()
    assert L.read_precalc_correlator_network_plan_fd(C.byref(P), C.byref(N), nb, 4, good.encode()) < 0


def _abi_err():
    from sphradiometer_b200 import _abi as A
    return A.last_error() if hasattr(A, "last_error") else ""
