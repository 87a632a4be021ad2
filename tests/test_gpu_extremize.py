"""GPU extremizer against the oracle on c1 skies.

The reference's sh_series_real_minimum (sh_series_extremize.c:273-360)
takes the best pixel of the l <= 6 low-passed series on its 14 x 14 mesh
and refines it with GSL's vector_bfgs2 (first step pi/24, line tolerance
0.001, <= 100 iterations, stop at |gradient| < 1e-3).  GSL is not in this
image: the oracle (oracle/ref_shims/bfgs2.h) and the library
(csrc/sht.cu) restate the published algorithm (Fletcher's line search,
memoryless BFGS directions).

* sh_series_real_minimum on the GPU runs that method exactly as the
  reference does -- gradient components along the unit vectors, which are
  not the derivatives in (theta, phi), and co-ordinates returned as the
  minimiser leaves them: it must land on the oracle's restatement's point
  (and on the reference's own, compiled against the stand-ins, where
  oracle/_ref is built).
* The batched localiser (sphrad_sky_peaks) runs the same method with the
  gradient in the co-ordinates: on 32 c1 skies it must reach the oracle's
  maximum (same point to 1e-6 rad, same value to 1e-9) on at least 31.

Skies: 32 c1 segments (3 detectors on the Earth sphere, 4096 Hz, l_max
32), integrated by the oracle on its own plan, GMST applied.
"""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import ref as R
from sphradiometer_b200 import workload as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def S():
    import torch
    assert torch.cuda.is_available()
    import sphradiometer_b200 as S
    S.load()
    return S


@pytest.fixture(scope="module")
def skies():
    pos = W.random_positions(3, W.R_EARTH_S, W.rng_for(2))
    n, dt, L = 4096, 1.0 / 4096, 32
    op = O.NetworkPlan(pos, n, dt, L)
    batch = W.make_batch(pos, n, dt, 32, seed=1234)
    out = []
    for s in range(32):
        F = W.full_from_half(batch["F"][:, s, :], n)
        out.append(O.rotate_z(op.integrate(F), L, False, batch["gmst"][s]))
    return np.array(out), L


def ang(t1, p1, t2, p2):
    u = np.array([np.sin(t1) * np.cos(p1), np.sin(t1) * np.sin(p1), np.cos(t1)])
    w = np.array([np.sin(t2) * np.cos(p2), np.sin(t2) * np.sin(p2), np.cos(t2)])
    return float(np.arctan2(np.linalg.norm(np.cross(u, w)), u @ w))


def test_drop_in_real_minimum_runs_the_reference_method(S, skies):
    a, L = skies
    same = 0
    for s in range(len(a)):
        v, t, p = S.real_minimum(-a[s], L)
        rv, rt, rp = O.real_minimum_ref(-a[s], L, False)
        if abs(t - rt) < 1e-8 and abs(p - rp) < 1e-8 and abs(v - rv) <= 1e-9 * abs(rv):
            same += 1
        if R.available():
            ev, et, ep = R.real_minimum(-a[s], L, False)
            assert abs(rt - et) < 1e-9 and abs(rp - ep) < 1e-9
    assert same >= len(a) - 1, same


def test_localiser_reaches_the_oracle_maximum_on_c1_skies(S, skies):
    import torch
    a, L = skies
    assert S.load().sphrad_sky_refinement() == 1  # BFGS2 by default
    out, st = S.sky_peaks(torch.from_numpy(a).cuda())
    out, st = out.cpu().numpy(), st.cpu().numpy()
    same = 0
    for s in range(len(a)):
        rv, rt, rp = O.real_maximum(a[s], L, False)
        assert st[s] & 1
        if ang(out[s, 0], out[s, 1], rt, rp) < 1e-6 and abs(out[s, 2] - rv) <= 1e-9 * abs(rv):
            same += 1
    assert same >= len(a) - 1, same


def test_newton_refinement_still_selectable(S, skies):
    """The trust-region Newton refinement reaches a local maximum at least
    as high as its start from the same pixels."""
    import torch
    a, L = skies
    lib = S.load()
    assert lib.sphrad_sky_set_refinement(0) == 0
    try:
        out, st = S.sky_peaks(torch.from_numpy(a[:8]).cuda())
    finally:
        assert lib.sphrad_sky_set_refinement(1) == 0
    out, st = out.cpu().numpy(), st.cpu().numpy()
    for s in range(8):
        assert st[s] & 1
        _, t0, p0 = O.find_near_minimum(-a[s], L, False)
        assert out[s, 2] >= O.eval_at(a[s], L, False, t0, p0).real - 1e-9
    assert lib.sphrad_sky_set_refinement(7) == -1
