"""GPU parity of the mesh transforms, products, extremizer, array Fourier
transforms and batched sky grids / peak localisation against the oracle.

Tolerances (all through the C ABI):
* FP64 meshes, products and array transforms: max |error| <= 1e-12 of the
  largest value (the reference's own product test asks 1e-13 pointwise of
  unit-sized values, test/product_validate.c:84; its mesh round trip asks
  1e-12 l^2, test/sh_series_validate.c:532);
* sky grids (float32 pixels): max |error| <= 2e-6 of the largest |value|
  for FP32 transforms, 1.2e-7 (the pixels' own rounding) for FP64 ones;
* extremizer: the same local maximum as the oracle's, direction within
  1e-7 rad and value within 1e-10 relative.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def random_series(rng, l_max, polar):
    """a_lm ~ CN(0, 1/(l+1)^2) (the reference's random_sh_series
    distribution, diagnostics.c:53-64)."""
    n = O.length(l_max, polar)
    ls, _ = O.lm_index_arrays(l_max, polar)
    sig = 1.0 / (ls + 1.0)
    return (rng.normal(size=n) + 1j * rng.normal(size=n)) * sig / np.sqrt(2)


@pytest.fixture(scope="module")
def S():
    import torch
    assert torch.cuda.is_available()
    import sphradiometer_b200 as S
    S.load()
    return S


def maxrel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("l_max,polar", [(0, False), (1, True), (7, False), (25, False), (25, True), (48, False)])
def test_to_mesh_matches_oracle(S, l_max, polar):
    rng = np.random.default_rng(100 + l_max)
    a = random_series(rng, l_max, polar)
    mesh, cx = S.to_mesh(a, l_max, polar)
    ref = O.to_mesh(a, l_max, polar)
    assert mesh.shape == ref.shape == (2 * (l_max + 1), 2 * (l_max + 1))
    assert maxrel(mesh, ref) < 1e-12
    x, _ = O.gl_nodes(2 * (l_max + 1))
    assert np.max(np.abs(cx - x)) < 1e-14


@pytest.mark.parametrize("l_max,polar", [(0, False), (3, True), (12, False), (33, False)])
def test_from_mesh_matches_oracle_and_round_trips(S, l_max, polar):
    rng = np.random.default_rng(200 + l_max)
    nt = 2 * (l_max + 1)
    mesh = rng.normal(size=(nt, nt)) + 1j * rng.normal(size=(nt, nt))
    got = S.from_mesh(mesh, l_max, polar)
    ref = O.from_mesh(mesh, l_max, polar)
    assert maxrel(got, ref) < 1e-12
    a = random_series(rng, l_max, polar)
    back = S.from_mesh(S.to_mesh(a, l_max, polar)[0], l_max, polar)
    assert maxrel(back, a) < 1e-12


PRODUCT_CASES = [
    # (a_l, a_polar, b_l, b_polar, dest_l, dest_polar)
    (0, False, 0, False, 0, False),
    (3, True, 4, True, 7, True),
    (5, False, 3, True, 6, False),
    (6, True, 6, True, 12, False),
    (10, False, 8, False, 18, False),
    (12, False, 12, False, 9, False),
    (20, False, 20, False, 20, True),
    (32, False, 32, False, 64, False),
]


@pytest.mark.parametrize("la,pa,lb,pb,ld,pd", PRODUCT_CASES)
def test_product_matches_oracle(S, la, pa, lb, pb, ld, pd):
    rng = np.random.default_rng(300 + la + lb + ld)
    a = random_series(rng, la, pa)
    b = random_series(rng, lb, pb)
    got = S.product(a, la, pa, b, lb, pb, ld, pd)
    dl = min(ld, la + lb)
    if dl < 60 and la + lb < 40:
        ref = O.product_microcode(a, la, pa, b, lb, pb, ld, pd)
    else:
        ref = O.product_pixel(a, la, pa, b, lb, pb, ld, pd)
    assert got.shape == ref.shape
    assert maxrel(got, ref) < 1e-12


def test_product_pointwise(S):
    """test/product_validate.c:70-85: (a b)(theta, phi) = a(theta, phi) b(theta, phi)
    when the destination holds the full product bandwidth."""
    rng = np.random.default_rng(7)
    la, lb = 9, 14
    a, b = random_series(rng, la, False), random_series(rng, lb, False)
    p = S.product(a, la, False, b, lb, False, la + lb, False)
    for _ in range(20):
        th, ph = np.arccos(rng.uniform(-1, 1)), rng.uniform(0, 2 * np.pi)
        lhs = O.eval_at(p, la + lb, False, th, ph)
        rhs = O.eval_at(a, la, False, th, ph) * O.eval_at(b, lb, False, th, ph)
        assert abs(lhs - rhs) < 1e-12 * max(1.0, abs(rhs))


def test_product_plan_checks(S):
    """sh_series_product refuses a plan built for other series
    (sh_series_product.c:343-344)."""
    L = S.load()
    a = L.sh_series_new_zero(4, 0)
    b = L.sh_series_new_zero(4, 0)
    d = L.sh_series_new_zero(8, 0)
    d2 = L.sh_series_new_zero(8, 1)
    plan = L.sh_series_product_plan_new(d, a, b)
    assert plan
    pl = plan
    assert not L.sh_series_product(d2, a, b, pl)
    assert L.sh_series_product(d, a, b, pl)
    L.sh_series_product_plan_free(pl)
    for s in (a, b, d, d2):
        L.sh_series_free(s)


@pytest.mark.parametrize("l_max,seed", [(6, 1), (12, 2), (25, 3), (32, 4), (32, 5)])
def test_real_minimum_matches_oracle(S, l_max, seed):
    """sh_series_real_minimum runs the reference's method (l <= 6 mesh
    start, BFGS2 with its unit-vector gradient components, co-ordinates
    returned as the minimiser leaves them): the oracle's restatement of it
    lands on the same point."""
    rng = np.random.default_rng(400 + seed)
    # a sky with one clear peak on noise, as the correlator produces
    th0, ph0 = np.arccos(rng.uniform(-0.9, 0.9)), rng.uniform(0, 2 * np.pi)
    a = 0.05 * O.impulse(l_max, th0, ph0) / np.sqrt(l_max + 1) + random_series(rng, l_max, False)
    v, t, p = S.real_minimum(-a, l_max)  # minimum of -Re f = maximum of Re f
    ref_v, ref_t, ref_p = O.real_minimum_ref(-a, l_max, False)
    assert abs(t - ref_t) < 1e-8 and abs(p - ref_p) < 1e-8, (t, p, ref_t, ref_p)
    assert abs(v - ref_v) <= 1e-10 * abs(ref_v)


def _ang(t1, p1, t2, p2):
    u = np.array([np.sin(t1) * np.cos(p1), np.sin(t1) * np.sin(p1), np.cos(t1)])
    w = np.array([np.sin(t2) * np.cos(p2), np.sin(t2) * np.sin(p2), np.cos(t2)])
    return float(np.arctan2(np.linalg.norm(np.cross(u, w)), np.dot(u, w)))


@pytest.mark.parametrize("n,l_max,polar", [(1, 3, False), (16, 4, True), (30, 5, False), (128, 2, False)])
def test_array_fft_matches_numpy(S, n, l_max, polar):
    import ctypes as C
    L = S.load()
    rng = np.random.default_rng(n)
    arr = L.sh_series_array_new(n, l_max, int(polar))
    stride = arr.contents.stride
    x = rng.normal(size=(n, stride)) + 1j * rng.normal(size=(n, stride))
    C.memmove(arr.contents.coeff, x.ctypes.data, x.nbytes)
    assert L.sh_series_array_forward_fft(arr)
    got = S.array_to_numpy(arr)
    assert maxrel(got, np.fft.fft(x, axis=0)) < 1e-12
    assert L.sh_series_array_reverse_fft(arr)
    back = S.array_to_numpy(arr)
    assert maxrel(back, n * x) < 1e-12
    L.sh_series_array_free(arr)


# ------------------------------------------------------------ batched skies --

def sky_batch(rng, n, l_max):
    skies, truth = [], []
    for _ in range(n):
        th0, ph0 = np.arccos(rng.uniform(-0.95, 0.95)), rng.uniform(0, 2 * np.pi)
        a = 0.08 * O.impulse(l_max, th0, ph0) + random_series(rng, l_max, False) / (l_max + 1)
        skies.append(a)
        truth.append((th0, ph0))
    return np.array(skies), truth


@pytest.mark.parametrize("fp32,kind", [(True, "cell"), (False, "cell"), (True, "gl"), (False, "gl")])
def test_sky_render_matches_oracle(S, fp32, kind):
    import torch
    rng = np.random.default_rng(11)
    L, nt, nph = 25, 64, 128
    skies, _ = sky_batch(rng, 3, L)
    g = S.SkyGrid(L, nt, nph, kind=kind, fp32=fp32)
    got = g.render(torch.from_numpy(skies).cuda()).cpu().numpy()
    th = g.rows()
    if kind == "cell":
        assert np.allclose(th, np.pi * (np.arange(nt) + 0.5) / nt, rtol=0, atol=1e-15)
    for s in range(len(skies)):
        ref = np.array([[O.eval_at(skies[s], L, False, t, 2 * np.pi * j / nph).real for j in range(nph)] for t in th]) if kind == "gl" \
            else O.render_grid(skies[s], L, False, nt, nph)
        # FP64 transforms still write float32 pixels: 6e-8 rounding
        tol = 2e-6 if fp32 else 1.2e-7
        assert maxrel(got[s], ref) < tol
    g.close()


def test_sky_render_folds_orders_above_nyquist(S):
    """A grid with fewer columns than 2 l_max + 1 samples e^{i m phi_j}
    exactly (orders fold), like direct evaluation."""
    import torch
    rng = np.random.default_rng(12)
    L, nt, nph = 20, 9, 16
    skies, _ = sky_batch(rng, 2, L)
    g = S.SkyGrid(L, nt, nph, kind="cell", fp32=False)
    got = g.render(torch.from_numpy(skies).cuda()).cpu().numpy()
    for s in range(2):
        assert maxrel(got[s], O.render_grid(skies[s], L, False, nt, nph)) < 1.2e-7


@pytest.mark.parametrize("l_max", [16, 32])
def test_sky_peaks_match_oracle(S, l_max):
    import torch
    rng = np.random.default_rng(20 + l_max)
    skies, truth = sky_batch(rng, 12, l_max)
    out, st = S.sky_peaks(torch.from_numpy(skies).cuda())
    out, st = out.cpu().numpy(), st.cpu().numpy()
    for s in range(len(skies)):
        rv, rt, rp = O.real_maximum(skies[s], l_max, False)
        assert st[s] & 1, "refinement did not converge"
        assert _ang(out[s, 0], out[s, 1], rt, rp) < 1e-7
        assert abs(out[s, 2] - rv) <= 1e-10 * abs(rv)


def test_grid_argmax_then_refine(S):
    """Full-grid search + refinement reaches the injected peak's maximum,
    and agrees with the reference localisation when both start in its
    basin."""
    import torch
    rng = np.random.default_rng(31)
    L = 32
    skies, truth = sky_batch(rng, 16, L)
    d = torch.from_numpy(skies).cuda()
    g = S.SkyGrid(L, 64, 128, kind="cell", fp32=True)
    th, ph = g.argmax(d)
    out, st = S.refine_peaks(d, th, ph)
    ref, _ = S.sky_peaks(d)
    out, ref = out.cpu().numpy(), ref.cpu().numpy()
    th, ph = th.cpu().numpy(), ph.cpu().numpy()
    # the coarse pixel is the grid's best pixel
    grid = g.render(d).cpu().numpy()
    rows = g.rows()
    for s in range(len(skies)):
        i, j = np.unravel_index(np.argmax(grid[s]), grid[s].shape)
        assert abs(th[s] - rows[i]) < 1e-12 and abs(ph[s] - 2 * np.pi * j / 128) < 1e-12
        # the same peak (BFGS2 stops at |gradient| < 1e-3, so two starts end
        # a few micro-radians apart), or a higher one
        assert _ang(out[s, 0], out[s, 1], ref[s, 0], ref[s, 1]) < 1e-5 or out[s, 2] >= ref[s, 2] - 1e-9 * abs(ref[s, 2])


def healpix_ring_angles(nside):
    """(theta, phi) of every pixel of a HEALPix map in RING order, from the
    published pixel-to-angle relations of the RING scheme (Gorski et al.
    2005, ApJ 622, 759, sec. 4)."""
    N = nside
    npix, ncap = 12 * N * N, 2 * N * (N - 1)
    th, ph = np.empty(npix), np.empty(npix)
    for p in range(npix):
        if p < ncap:
            hip = (p + 1) / 2.0
            i = int(np.sqrt(hip - np.sqrt(np.floor(hip)))) + 1
            j = p + 1 - 2 * i * (i - 1)
            z, phi = 1 - i * i / (3.0 * N * N), (j - 0.5) * np.pi / (2 * i)
        elif p < npix - ncap:
            q = p - ncap
            i, j = q // (4 * N) + N, q % (4 * N) + 1
            fodd = 0.5 * (1 + (i + N) % 2)
            z, phi = (2 * N - i) * 2.0 / (3 * N), (j - fodd) * np.pi / (2 * N)
        else:
            q = npix - p
            hip = q / 2.0
            i = int(np.sqrt(hip - np.sqrt(np.floor(hip)))) + 1
            j = 4 * i + 1 - (q - 2 * i * (i - 1))
            z, phi = -1 + i * i / (3.0 * N * N), (j - 0.5) * np.pi / (2 * i)
        th[p], ph[p] = np.arccos(z), phi
    return th, ph


@pytest.mark.parametrize("fp32,nside,L", [(False, 8, 12), (True, 8, 12), (False, 16, 32), (True, 16, 32)])
def test_healpix_ring_render_matches_oracle(S, fp32, nside, L):
    """Rendering onto a HEALPix-like ring grid (the map of the reference's
    sh_series_write_healpix_map, sh_series_healpix.cc:245-286) agrees with
    direct evaluation at every pixel: FP32 transforms 2e-6 of the largest
    value; FP64 transforms (which still write float32 pixels) to the
    rounding of each pixel to float32, 2^-24 of its value, plus 1e-12 of the
    largest."""
    import torch
    rng = np.random.default_rng(70 + nside)
    skies, _ = sky_batch(rng, 2, L)
    g = S.SkyGrid(L, nside, kind="healpix", fp32=fp32)
    assert g.n_pixels == 12 * nside * nside and g.n_rows == 4 * nside - 1
    got = g.render(torch.from_numpy(skies).cuda()).cpu().numpy()
    th, ph = healpix_ring_angles(nside)
    rows = g.rows()
    assert np.max(np.abs(np.unique(np.round(th, 12)) - np.round(rows, 12))) < 1e-12
    for s in range(2):
        ref = np.array([O.eval_at(skies[s], L, False, th[p], ph[p]).real for p in range(len(th))])
        big = np.max(np.abs(ref))
        if fp32:
            err = np.max(np.abs(got[s] - ref)) / big
            assert err < 2e-6, err
        else:
            excess = np.abs(got[s] - ref) - (2.0 ** -24 * np.abs(ref) + 1e-12 * big)
            assert np.max(excess) <= 0, np.max(excess)
