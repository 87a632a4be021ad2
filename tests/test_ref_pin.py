"""The oracle pinned to the reference itself.

The reference's own C code for this path (src/lib/correlator.c,
projection.c, sh_series*.c, instrument.c), compiled unmodified against the
project's FFTW/GSL/LAL stand-ins (oracle/Makefile "ref" target,
oracle/ref_shims), produced the fixtures in tests/golden (script:
tests/golden/make_ref_golden.py).  These tests hold the oracle
(oracle/sphrad_oracle.c) to those outputs at FP64 rounding:

* c0 (2 detectors 3000 km apart, 2048 Hz, l_max 25) and c1 (3 detectors on
  the Earth sphere, 4096 Hz, l_max 32, native plan l_max ~547): each
  baseline's geometry and l_max, delay table (every 64th bin row and two
  seeded projections over all bins), rotation plan (every 31st element),
  and the network skies of 4 seeded segments before and after the GMST
  rotation.  Bound: relative L2 <= 1e-12 (measured ~1e-14).

Where oracle/_ref is built (machines with the reference checkout), the
remaining tests compare the oracle with the live reference on small cases:
rotation plans, products (Gaunt microcode and pixel domain), meshes, the
drop-in network integration at native and reduced l_max, and the
extremizer sh_series_real_minimum.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from oracle import ref as R
from sphradiometer_b200 import workload as W

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def golden(name):
    return np.load(os.path.join(GOLDEN, f"ref_{name}.npz"))


def projection_vectors(seed: int, n: int):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(2, n)) + 1j * rng.normal(size=(2, n))


@pytest.mark.parametrize("name", ["c0", "c1"])
def test_oracle_plans_match_reference_fixture(name):
    g = golden(name)
    n, dt, L = int(g["n"]), float(g["dt"]), int(g["l_max"])
    op = O.NetworkPlan(g["positions"], n, dt, L)
    rvec = projection_vectors(int(g["rvec_seed"]), n)
    assert len(op.baselines) == len(g["baselines"])
    for k, b in enumerate(op.baselines):
        ia, ib, th, ph, lb = g["baselines"][k]
        assert (b["i"], b["j"], b["l"]) == (int(ia), int(ib), int(lb))
        assert abs(b["theta"] - th) < 1e-15 and abs(b["phi"] - ph) < 1e-15
        assert rel(b["D"][::int(g["row_step"])], g[f"D_rows_{k}"]) < 1e-12, k
        assert rel(rvec @ b["D"], g[f"D_proj_{k}"]) < 1e-12, k
        assert rel(b["Rot"][::int(g["rot_step"])], g[f"rot_{k}"]) < 1e-13, k


@pytest.mark.parametrize("name", ["c0", "c1"])
def test_oracle_skies_match_reference_fixture(name):
    g = golden(name)
    n, dt, L = int(g["n"]), float(g["dt"]), int(g["l_max"])
    op = O.NetworkPlan(g["positions"], n, dt, L)
    nsk = len(g["skies"])
    batch = W.make_batch(g["positions"], n, dt, nsk, seed=int(g["batch_seed"]))
    for s in range(nsk):
        F = W.full_from_half(batch["F"][:, s, :], n)
        # the regenerated inputs are the ones the fixture was made from
        assert rel([F.sum(), (np.abs(F) ** 2).sum()], g["spectra_checksums"][s]) < 1e-13
        sky = op.integrate(F)
        assert rel(sky, g["skies"][s]) < 1e-12, s
        assert rel(O.rotate_z(sky, L, False, float(g["gmst"][s])), g["skies_gmst"][s]) < 1e-12, s


# ------------------------------------------------------------ live reference --

needs_ref = pytest.mark.skipif(not R.available(), reason="oracle/_ref not built (needs the reference checkout)")


@needs_ref
def test_rotation_plans_match_live_reference():
    rng = np.random.default_rng(5)
    for l_max in (1, 6, 25, 48):
        g, b, a = rng.uniform(0, 2 * np.pi), np.arccos(rng.uniform(-1, 1)), rng.uniform(0, 2 * np.pi)
        got = O.rotation_plan(l_max, O.euler_rotation_matrix(g, b, a))
        assert rel(got, R.rotation_plan(l_max, g, b, a)) < 1e-13, l_max


@needs_ref
@pytest.mark.parametrize("a_l,a_p,b_l,b_p,d_l,d_p", [(5, 0, 10, 0, 15, 0), (5, 1, 10, 0, 15, 0), (6, 1, 9, 1, 15, 1), (30, 0, 35, 1, 65, 0), (40, 1, 30, 1, 70, 1)])
def test_products_match_live_reference(a_l, a_p, b_l, b_p, d_l, d_p):
    """Microcode below dest l_max 60, pixel domain above
    (sh_series_product.c:199)."""
    rng = np.random.default_rng(a_l * 100 + b_l)
    a = rng.normal(size=O.length(a_l, a_p)) + 1j * rng.normal(size=O.length(a_l, a_p))
    b = rng.normal(size=O.length(b_l, b_p)) + 1j * rng.normal(size=O.length(b_l, b_p))
    ref = R.product(a, a_l, a_p, b, b_l, b_p, d_l, d_p)
    if d_l < 60:
        got = O.product_microcode(a, a_l, a_p, b, b_l, b_p, d_l, d_p)
    else:
        got = O.product_pixel(a, a_l, a_p, b, b_l, b_p, d_l, d_p)
    assert rel(got, ref) < 1e-12


@needs_ref
@pytest.mark.parametrize("l_max,polar", [(7, False), (20, True), (33, False)])
def test_meshes_match_live_reference(l_max, polar):
    rng = np.random.default_rng(l_max)
    a = rng.normal(size=O.length(l_max, polar)) + 1j * rng.normal(size=O.length(l_max, polar))
    assert rel(O.to_mesh(a, l_max, polar), R.to_mesh(a, l_max, polar)) < 1e-13


@needs_ref
@pytest.mark.parametrize("l_max", [None, 5])
def test_network_integration_matches_live_reference(l_max):
    """3 detectors, n = 256 at 256 Hz: native l_max (no set_l) and reduced."""
    pos = W.random_positions(3, 0.02, W.rng_for(4))
    n, dt = 256, 1.0 / 256
    rn = R.Network(pos, n, dt, l_max)
    L = max(rn.baseline_l_max(k) for k in range(rn.n_baselines))
    op = O.NetworkPlan(pos, n, dt, 10 ** 6 if l_max is None else l_max)
    assert op.l_max == L
    for k, b in enumerate(op.baselines):
        assert rel(b["D"], rn.delay_table(k)) < 1e-12
        assert rel(b["Rot"], rn.rotation_flat(k)) < 1e-13
    rng = np.random.default_rng(9)
    F = rng.normal(size=(3, n)) + 1j * rng.normal(size=(3, n))
    assert rel(op.integrate(F), rn.integrate(F, L)) < 1e-12


@needs_ref
def test_extremizer_matches_live_reference():
    """sh_series_real_minimum: the oracle's restatement (l <= 6 start, the
    BFGS2 restatement with the reference's gradient convention) lands where
    the reference does, compiled against the same GSL stand-in."""
    rng = np.random.default_rng(17)
    for trial in range(12):
        L = (6, 12, 25)[trial % 3]
        a = rng.normal(size=O.length(L, False)) + 1j * rng.normal(size=O.length(L, False))
        v0, t0, p0 = R.real_minimum(a, L, False)
        v1, t1, p1 = O.real_minimum_ref(a, L, False)
        assert abs(v0 - v1) <= 1e-12 * max(1.0, abs(v0)), trial
        assert abs(t0 - t1) < 1e-9 and abs(p0 - p1) < 1e-9, trial
