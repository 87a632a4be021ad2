"""Time-domain correlator (correlator.c:325-418, 648-673, 820-858,
967-984) and the delay projection matrices (projection.c:99-131) through
the C ABI, against the oracle's restatement of the reference's per-sample
loop (sample dot products, Gaunt-microcode products, windowed sum,
rotation).  The library contracts the windowed sum of outer products
instead of multiplying per sample, so agreement is to FP64 rounding: the
bar is 1e-10 of the largest coefficient."""
import numpy as np
import pytest

from oracle import oracle as O
from sphradiometer_b200 import workload as W

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _rel(got, ref):
    return np.max(np.abs(got - ref)) / np.max(np.abs(ref))


@pytest.mark.parametrize("r", [0.004, -0.004, 0.0113])
def test_polar_projection_matrix_matches_oracle_taps(r):
    import sphradiometer_b200 as S
    dt = 1.0 / 1024
    n_el = O.projection_n_elements(abs(r), dt)
    a_l = O.projection_l_max(abs(r), dt)
    got = S.projection_matrix_delay([0.0, 0.0, r], n_el, a_l, dt)
    ref = O.projection_taps(r, dt)
    assert got.shape == ref.shape
    assert _rel(got, ref) < 1e-12


def test_off_axis_projection_matrix_matches_mesh_analysis():
    """An off-axis phase centre gives full series: each tap's sinc sampled
    on the reference mesh of l_max and analysed (sh_series_from_realfunc)."""
    import sphradiometer_b200 as S
    dt, L = 1.0 / 1024, 9
    r = np.array([0.0021, -0.0013, 0.0017])
    n_el = 9
    got = S.projection_matrix_delay(r, n_el, L, dt)
    nt = 2 * (L + 1)
    x, _ = O.gl_nodes(nt)
    th = np.arccos(x)[:, None]
    ph = (2 * np.pi * np.arange(nt) / nt)[None, :]
    rs = r[0] * np.sin(th) * np.cos(ph) + r[1] * np.sin(th) * np.sin(ph) + r[2] * np.cos(th)
    ref = []
    for t in range(n_el):
        k = t - (n_el - 1) // 2
        ref.append(O.from_mesh(np.sinc(-k - rs / dt).astype(np.complex128), L, False))
    ref = np.array(ref)
    assert got.shape == ref.shape
    assert _rel(got, ref) < 1e-12
    # a phase centre on the axis through the same route equals the polar taps
    pol = S.projection_matrix_delay([0.0, 0.0, 0.003], n_el, L, dt)
    ref_p = []
    rs = 0.003 * np.cos(th) + 0 * ph
    for t in range(n_el):
        k = t - (n_el - 1) // 2
        full = O.from_mesh(np.sinc(-k - rs / dt).astype(np.complex128), L, False)
        ref_p.append(O.assign(full, L, False, L, True))
    assert _rel(pol, np.array(ref_p)) < 1e-12


def _plan_matches_oracle(net, k, dt):
    b = net.baseline(k)
    d = np.array([b.d.contents.data[i] for i in range(3)])
    dl = float(np.linalg.norm(d))
    pa, pb = net.projections(k)
    assert _rel(pa, O.projection_taps(dl / 2, dt)) < 1e-12
    assert _rel(pb, O.projection_taps(-dl / 2, dt)) < 1e-12
    assert net.transient(k) == (O.projection_n_elements(dl / 2, dt) - 1) // 2
    assert net.power_l_max(k) == O.td_power_l_max(dl, dt)
    return dl, b.theta, b.phi


def test_baseline_integrator_matches_oracle():
    import sphradiometer_b200 as S
    dt = 1.0 / 512
    pos = W.random_positions(2, W.R_EARTH_S, W.rng_for(31))
    net = S.TimeDomainNetwork(pos, dt)
    dl, th, ph = _plan_matches_oracle(net, 0, dt)
    pl = net.power_l_max(0)
    rng = np.random.Generator(np.random.Philox(5))
    n = 2 * net.transient(0) + 333
    ts = rng.normal(size=(2, n))
    win = rng.uniform(0.5, 1.5, n - 2 * net.transient(0))
    got = net.integrate_baseline(0, ts[1], ts[0], win)
    ref = O.baseline_integrate_power_td(ts[1], ts[0], win, dl, dt, pl, O.rotation_plan(pl, O.rot_matrix(th, ph)))
    assert _rel(got, ref) < TOL
    # power_1d keeps the unrotated sum, as in the reference
    p1 = S.series_to_numpy(net.plan_td(0).contents.power_1d)
    ref1 = O.baseline_integrate_power_td(ts[1], ts[0], win, dl, dt, pl, O.rotation_plan(pl, O.rot_matrix(0.0, 0.0)))
    assert _rel(p1, O.assign(ref1, pl, False, pl, True)) < TOL
    net.close()


def test_network_integrator_matches_oracle():
    """3 detectors, Tukey windows, the sky at the network's l_max and two
    degrees above it; each plan's power_1d keeps its unrotated sum."""
    import sphradiometer_b200 as S
    dt = 1.0 / 512
    pos = W.random_positions(3, W.R_EARTH_S, W.rng_for(32))
    net = S.TimeDomainNetwork(pos, dt)
    rng = np.random.Generator(np.random.Philox(6))
    n = 2 * max(net.transient(k) for k in range(3)) + 257
    ts = rng.normal(size=(3, n))
    wins, ref, p1 = [], np.zeros(O.length(net.l_max, False), np.complex128), []
    k = 0
    for i in range(1, 3):
        for j in range(i):
            dl, th, ph = _plan_matches_oracle(net, k, dt)
            m = n - 2 * net.transient(k)
            w = np.ones(m)
            w[:40] = 0.5 * (1 - np.cos(np.pi * np.arange(40) / 40))
            w[m - 40:] = w[:40][::-1]
            w /= m
            wins.append(w)
            pl = net.power_l_max(k)
            p = O.baseline_integrate_power_td(ts[i], ts[j], w, dl, dt, pl, O.rotation_plan(pl, O.rot_matrix(th, ph)))
            ref += O.assign(p, pl, False, net.l_max, False) / 3
            u = O.baseline_integrate_power_td(ts[i], ts[j], w, dl, dt, pl, O.rotation_plan(pl, O.rot_matrix(0.0, 0.0)))
            p1.append(O.assign(u, pl, False, pl, True))
            k += 1
    got = net.integrate(ts, wins)
    assert _rel(got, ref) < TOL
    for k in range(3):
        assert _rel(S.series_to_numpy(net.plan_td(k).contents.power_1d), p1[k]) < TOL
    big = net.integrate(ts, wins, sky_l_max=net.l_max + 2)
    assert _rel(big, O.assign(ref, net.l_max, False, net.l_max + 2, False)) < TOL
    net.close()


def test_edge_lengths():
    """n = 2 transient integrates nothing (a zero sky); n below it is an
    error (correlator.c:651-653)."""
    import sphradiometer_b200 as S
    dt = 1.0 / 256
    pos = W.random_positions(2, W.R_EARTH_S, W.rng_for(33))
    net = S.TimeDomainNetwork(pos, dt)
    tr = net.transient(0)
    ts = np.ones((2, 2 * tr))
    got = net.integrate_baseline(0, ts[1], ts[0], np.zeros(1))
    assert not np.any(got)
    with pytest.raises(S.SphradError):
        net.integrate_baseline(0, ts[1][:-1], ts[0][:-1], np.zeros(1))
    net.close()


def test_complex_taps_follow_the_reference_loop():
    """A caller may write complex coefficients into proj_a / proj_b; the
    integrator then forms complex samples and products (the path that real
    taps skip), checked against a numpy restatement of the reference's loop
    (sh_series_array_dot per sample, Gaunt-microcode products, windowed
    sum, rotation)."""
    import ctypes as C
    import sphradiometer_b200 as S
    dt = 1.0 / 512
    pos = W.random_positions(2, W.R_EARTH_S, W.rng_for(34))
    net = S.TimeDomainNetwork(pos, dt)
    p = net.plan_td(0).contents
    rng = np.random.Generator(np.random.Philox(9))
    views = []
    for arr in (p.proj_a.contents, p.proj_b.contents):
        buf = (C.c_double * (2 * arr.n * arr.stride)).from_address(arr.coeff)
        v = np.frombuffer(buf, dtype=np.complex128).reshape(arr.n, arr.stride)
        v += 0.05j * rng.normal(size=v.shape) * np.abs(v).max()
        views.append(v.copy())
    ta, tb = views
    La, Lb = ta.shape[1] - 1, tb.shape[1] - 1
    pl, tr = net.power_l_max(0), net.transient(0)
    n = 2 * tr + 97
    ts = rng.normal(size=(2, n))
    win = rng.uniform(0.5, 1.5, n - 2 * tr)
    got = net.integrate_baseline(0, ts[1], ts[0], win)
    plan = O.product_plan(pl, True, La, True, Lb, True)
    p1 = np.zeros(pl + 1, np.complex128)
    for t in range(n - 2 * tr):
        sa = ta.T @ ts[1][t:t + ta.shape[0]]
        sb = tb.T @ ts[0][t:t + tb.shape[0]]
        p1 += win[t] * O.product_microcode(sa, La, True, sb, Lb, True, pl, True, plan)
    b = net.baseline(0)
    ref = O.rotate(p1, pl, True, O.rotation_plan(pl, O.rot_matrix(b.theta, b.phi)))
    assert np.max(np.abs(p1.imag)) > 1e-3 * np.max(np.abs(p1))  # the taps' imaginary parts matter
    assert _rel(got, ref) < TOL
    net.close()
