"""The CPU oracle pinned against the reference's own known-answer tests.

Each test restates one of the reference's assert-based validation
programs with a fixed seed (the reference seeds from the clock):

* Y_lm / Legendre values        -- test/sh_series_validate.c:220-296
* mesh round trip               -- test/sh_series_validate.c:518-538
* D diagonal for z rotations    -- test/rotation_validate.c:328-353
* D real for y rotations        -- test/rotation_validate.c:360-384
* rotated impulse               -- test/rotation_validate.c:396-437, 494-498
* product vs pointwise product  -- test/product_validate.c:46-126
* FD correlator vs the analytic
  band-limited noise solution   -- test/correlator_validate.c:78-114, 222-376
"""
import numpy as np
import pytest
import scipy.special as sp

from oracle import oracle as O
from sphradiometer_b200 import workload as W


def test_wigner_3j_against_exact_values():
    from sympy.physics.wigner import wigner_3j
    rng = np.random.default_rng(11)
    worst = 0.0
    for _ in range(300):
        j2, j3 = rng.integers(0, 13, 2)
        j1 = int(rng.integers(abs(j2 - j3), j2 + j3 + 1))
        m2 = int(rng.integers(-j2, j2 + 1))
        m3 = int(rng.integers(-j3, j3 + 1))
        m1 = -m2 - m3
        if abs(m1) > j1:
            continue
        ref = float(wigner_3j(j1, int(j2), int(j3), m1, m2, m3))
        worst = max(worst, abs(O.wigner_3j(j1, int(j2), int(j3), m1, m2, m3) - ref))
    assert worst < 1e-14
    for args in [(48, 48, 48, 5, -3, -2), (96, 48, 48, 0, 12, -12), (30, 40, 70, -20, 20, 0)]:
        ref = float(wigner_3j(*args).evalf(30))
        assert abs(O.wigner_3j(*args) - ref) <= 1e-13 * abs(ref)


def test_legendre_and_Y_against_scipy():
    for x in (-0.97, -0.3, 0.0, 0.41, 0.999):
        th = np.arccos(x)
        for m in (0, 1, 4, 9):
            P = O.sphPlm_array(30, m, x)
            ref = [np.real(sp.sph_harm_y(l, m, th, 0.0)) for l in range(m, 31)]
            assert np.max(np.abs(P - ref)) < 1e-13
    for l, m in [(3, -2), (5, 5), (7, -7), (10, 0), (12, -3)]:
        th, ph = 1.1, 2.3
        assert abs(O.Y(l, m, th, ph) - sp.sph_harm_y(l, m, th, ph)) < 1e-13


def test_gauss_legendre_nodes():
    for n in (2, 7, 66, 550):
        x, w = O.gl_nodes(n)
        xr, wr = np.polynomial.legendre.leggauss(n)
        assert np.all(np.diff(x) < 0)
        assert np.max(np.abs(x[::-1] - xr)) < 1e-14
        assert np.max(np.abs(w[::-1] - wr)) < 1e-13


def _random_series(rng, l_max, polar):
    n = O.length(l_max, polar)
    s = 1.0 / (l_max + 1)
    return rng.uniform(-s, s, n) + 1j * rng.uniform(-s, s, n)


def test_mesh_round_trip():
    rng = np.random.default_rng(5)
    for l in (1, 7, 20, 49):
        a = _random_series(rng, l, False)
        b = O.from_mesh(O.to_mesh(a, l, False), l, False)
        assert np.max(np.abs(a - b)) <= 1e-12 * l * l


def test_z_rotation_is_diagonal_and_y_rotation_real():
    for omega in np.arange(0.125, 7.0, 0.5):
        Dz = O.rotation_plan(10, O.euler_rotation_matrix(omega, 0.0, 0.0))
        Dy = O.rotation_plan(10, O.euler_rotation_matrix(0.0, omega, 0.0))
        for l in range(1, 11):
            for m in range(-l, l + 1):
                for mp in range(-l, l + 1):
                    if m != mp:
                        assert O.wigner_D(Dz, l, m, mp) == 0
                    assert np.imag(O.wigner_D(Dy, l, m, mp)) == 0


@pytest.mark.parametrize("l_max,delta_l", [(1, 0), (13, 0), (13, -5)])
def test_rotated_impulse(l_max, delta_l):
    rng = np.random.default_rng(100 + l_max)
    L = l_max + delta_l
    for _ in range(200):
        th, ph = rng.uniform(0, np.pi), rng.uniform(0, 2 * np.pi)
        dth, dph = rng.uniform(0, np.pi) - th, rng.uniform(0, 2 * np.pi) - ph
        s = O.assign(O.impulse(l_max, th, ph), l_max, False, L, False)
        c = O.assign(O.impulse(l_max, th + dth, ph + dph), l_max, False, L, False)
        D = O.rotation_plan(l_max, O.euler_rotation_matrix(-ph, dth, ph + dph))
        r = O.rotate(s, L, False, D)
        assert O.rms_error(r, c, L) < 1e-10


@pytest.mark.parametrize("l1,p1,l2,p2", [(5, 0, 10, 0), (5, 0, 10, 1), (5, 1, 10, 0), (5, 1, 10, 1),
                                         (40, 0, 70, 0), (40, 0, 70, 1), (40, 1, 70, 0), (40, 1, 70, 1)])
def test_product_pointwise(l1, p1, l2, p2):
    rng = np.random.default_rng(l1 * 100 + l2 + 10 * p1 + p2)
    a, b = _random_series(rng, l1, p1), _random_series(rng, l2, p2)
    dl, dp = l1 + l2, bool(p1 and p2)
    # dest < 60 runs the Gaunt microcode, larger ones the pixel product,
    # as sh_series_product_plan_new() chooses (sh_series_product.c:199)
    if dl < 60:
        prod = O.product_microcode(a, l1, p1, b, l2, p2, dl, dp)
    else:
        prod = O.product_pixel(a, l1, p1, b, l2, p2, dl, dp)
    worst = 0.0
    for _ in range(300):
        th, ph = rng.uniform(0, np.pi), rng.uniform(0, 2 * np.pi)
        v = O.eval_at(a, l1, p1, th, ph) * O.eval_at(b, l2, p2, th, ph)
        worst = max(worst, abs(v - O.eval_at(prod, dl, dp, th, ph)) / (l1 * l1 + l2 * l2))
    assert worst <= 1e-13


def test_product_microcode_matches_pixel_domain():
    rng = np.random.default_rng(9)
    for (l1, p1, l2, p2, dl, dp) in [(8, 0, 9, 0, 12, 0), (6, 1, 11, 0, 17, 0), (10, 1, 10, 1, 20, 1)]:
        a, b = _random_series(rng, l1, p1), _random_series(rng, l2, p2)
        m = O.product_microcode(a, l1, p1, b, l2, p2, dl, dp)
        p = O.product_pixel(a, l1, p1, b, l2, p2, dl, dp)
        assert np.max(np.abs(m - p)) < 1e-14


def _noise_solution(b, l, var, dt, ra, dec, gmst):
    """correlator_validate.c:78-114, projected with the oracle's from_mesh."""
    f0, df = 0.25 / dt, 0.5 / dt
    th_b, ph_b = b["theta"], b["phi"] + gmst
    it, ip = np.pi / 2 - dec, ra
    cgs = np.cos(it) * np.cos(th_b) + np.sin(it) * np.sin(th_b) * np.cos(ip - ph_b)
    nt = 2 * (l + 1)
    x, _ = O.gl_nodes(nt)
    theta = np.arccos(x)[:, None]
    phi = (2 * np.pi / nt * np.arange(nt))[None, :]
    cg = np.cos(theta) * np.cos(th_b) + np.sin(theta) * np.sin(th_b) * np.cos(phi - ph_b)
    zeta = b["d_len"] * (cg - cgs)
    val = var * np.sinc(zeta * df) * np.cos(2 * np.pi * zeta * f0)
    return O.from_mesh(val.astype(np.complex128), l, False)


def test_fd_correlator_against_analytic_noise_solution():
    """4 detectors (seeded positions on the Earth sphere instead of LAL's
    H1/L1/V1/K1), 512 Hz, a white-noise source at RA = Dec = 0, three GMSTs;
    RMS(FD - order-reduced exact) must be <= -21 dB of the variance."""
    rng = np.random.Generator(np.random.Philox(7))
    pos = W.random_positions(4, W.R_EARTH_S, rng)
    dt = 1.0 / 512
    pairs = [(i, j) for i in range(1, 4) for j in range(i)]
    sky_l = max(O.power_l_max_naive(float(np.linalg.norm(pos[i] - pos[j])), dt) for i, j in pairs)
    n = int((86164.0 / sky_l / 20) / dt)  # correlator_dump_interval(sky_l, 20)
    bls = []
    for i, j in pairs:
        d = pos[i] - pos[j]
        dl = float(np.linalg.norm(d))
        th, ph = O.vector_direction(d)
        pl = O.native_power_l_max(dl, dt)
        bls.append(dict(i=i, j=j, d_len=dl, theta=th, phi=ph, pl=pl,
                        D=O.delay_product(dl, dt, n, pl), Rot=O.rotation_plan(pl, O.rot_matrix(th, ph))))
    for gi in range(3):
        gmst = gi * np.pi / 4
        ts = np.zeros((4, n))
        inj = W.gaussian_white_noise(n, 1.0, rng)
        for k in range(4):
            W.inject_into(pos[k], ts[k], inj, dt, 0.0, 0.0, gmst)
        F = np.stack([W.tseries_to_fseries(ts[k]) for k in range(4)])
        sky = np.zeros(O.length(sky_l, False), np.complex128)
        for b in bls:
            p = O.baseline_integrate_power_fd(F[b["i"]], F[b["j"]], b["D"], b["pl"], b["Rot"])
            sky += O.assign(p, b["pl"], False, sky_l, False) / len(bls)
        sky = O.rotate_z(sky, sky_l, False, gmst)
        sol = sum(_noise_solution(b, 2 * sky_l, 1.0, dt, 0.0, 0.0, gmst) for b in bls) / len(bls)
        sol_lo = O.assign(sol, 2 * sky_l, False, sky_l, False)
        assert 10 * np.log10(O.rms_error(sky, sol_lo, sky_l)) <= -21.0


def test_td_correlator_against_analytic_noise_solution():
    """The time-domain leg of the same validation (correlator_validate.c:
    238, 265-268, 308, 374): square windows of n - 2 transient samples with
    amplitude 1 / (n - 2 transient); RMS(TD - order-reduced exact) must be
    <= -21 dB of the variance.  One GMST: the oracle runs the reference's
    per-sample loop."""
    rng = np.random.Generator(np.random.Philox(11))
    pos = W.random_positions(4, W.R_EARTH_S, rng)
    dt = 1.0 / 512
    pairs = [(i, j) for i in range(1, 4) for j in range(i)]
    sky_l = max(O.power_l_max_naive(float(np.linalg.norm(pos[i] - pos[j])), dt) for i, j in pairs)
    n = int((86164.0 / sky_l / 20) / dt)
    gmst = np.pi / 3
    ts = np.zeros((4, n))
    inj = W.gaussian_white_noise(n, 1.0, rng)
    for k in range(4):
        W.inject_into(pos[k], ts[k], inj, dt, 0.0, 0.0, gmst)
    sky = np.zeros(O.length(sky_l, False), np.complex128)
    bls = []
    for i, j in pairs:
        d = pos[i] - pos[j]
        dl = float(np.linalg.norm(d))
        th, ph = O.vector_direction(d)
        pl = O.td_power_l_max(dl, dt)
        tr = (O.projection_n_elements(dl / 2, dt) - 1) // 2
        win = np.full(n - 2 * tr, 1.0 / (n - 2 * tr))
        p = O.baseline_integrate_power_td(ts[i], ts[j], win, dl, dt, pl, O.rotation_plan(pl, O.rot_matrix(th, ph)))
        sky += O.assign(p, pl, False, sky_l, False) / len(pairs)
        bls.append(dict(d_len=dl, theta=th, phi=ph))
    sky = O.rotate_z(sky, sky_l, False, gmst)
    sol = sum(_noise_solution(b, 2 * sky_l, 1.0, dt, 0.0, 0.0, gmst) for b in bls) / len(bls)
    sol_lo = O.assign(sol, 2 * sky_l, False, sky_l, False)
    assert 10 * np.log10(O.rms_error(sky, sol_lo, sky_l)) <= -21.0


def test_delay_table_is_hermitian_along_bins():
    """Real taps give D[n-k] = conj(D[k]) (correlator.c:482-489)."""
    D = O.delay_product(0.0101, 1.0 / 1024, 256, 12)
    k = np.arange(1, 256)
    assert np.max(np.abs(D[256 - k] - np.conj(D[k]))) < 1e-13 * np.max(np.abs(D))
