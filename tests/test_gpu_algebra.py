"""GPU parity of the batched spherical-harmonic algebra (the SH algebra
batch: many series rotated by their own rotations, and pairwise products)
against the FP64 oracle.

Tolerances: FP64 application / transforms, relative L2 per series
<= 1e-12; FP32 application / transforms, <= 2e-6 (single-precision
rounding of O(100)-term sums of unit-sized products).
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def random_series(rng, l_max, polar):
    n = O.length(l_max, polar)
    ls, _ = O.lm_index_arrays(l_max, polar)
    return (rng.normal(size=n) + 1j * rng.normal(size=n)) / (ls + 1.0) / np.sqrt(2)


def random_rotations(rng, n):
    """Euler angles alpha, gamma ~ U[0, 2 pi), cos beta ~ U[-1, 1] and the
    matrices euler_rotation_matrix(gamma, beta, alpha) returns."""
    out = []
    for _ in range(n):
        a, g = rng.uniform(0, 2 * np.pi, 2)
        b = np.arccos(rng.uniform(-1, 1))
        out.append(((g, b, a), O.euler_rotation_matrix(g, b, a)))
    return out


@pytest.fixture(scope="module")
def S():
    import torch
    assert torch.cuda.is_available()
    import sphradiometer_b200 as S
    S.load()
    return S


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("l_max,polar", [(0, False), (1, False), (2, True), (7, False), (32, False), (48, False), (48, True)])
@pytest.mark.parametrize("fp32", [False, True])
def test_rotate_batch_matches_oracle(S, l_max, polar, fp32):
    import torch
    rng = np.random.default_rng(1000 + l_max)
    n = 37
    series = np.array([random_series(rng, l_max, polar) for _ in range(n)])
    rots = random_rotations(rng, n)
    R = np.array([r for _, r in rots])
    got = S.rotate_batch(torch.from_numpy(series).cuda(), torch.from_numpy(R).cuda(), l_max, polar=polar, fp32=fp32).cpu().numpy()
    tol = 2e-6 if fp32 else 1e-12
    for s in range(n):
        ref = O.rotate(series[s], l_max, polar, O.rotation_plan(l_max, R[s]))
        assert rel(got[s], ref) < tol, (s, rel(got[s], ref))


@pytest.mark.parametrize("fp32", [False, True])
def test_rotate_batch_large_lmax(S, fp32):
    """l_max 80: in FP64 a degree's Delta block and the block's series no
    longer fit shared memory together, so the products read Delta from the
    (L2-resident) table in its padded layout; in FP32 the shared-memory
    tile is about 150 KB.  Bound: the FP32 application's 2e-6, and in FP64
    the accuracy of the reference recursion's Delta at this degree (its
    orthogonality error grows from 5e-13 at l = 48 to 1e-11 at 64)."""
    import torch
    l_max, n = 80, 5
    rng = np.random.default_rng(80)
    series = np.array([random_series(rng, l_max, False) for _ in range(n)])
    R = np.array([r for _, r in random_rotations(rng, n)])
    got = S.rotate_batch(torch.from_numpy(series).cuda(), torch.from_numpy(R).cuda(), l_max, polar=False, fp32=fp32).cpu().numpy()
    tol = 2e-6 if fp32 else 1e-9
    for s in range(n):
        ref = O.rotate(series[s], l_max, False, O.rotation_plan(l_max, R[s]))
        assert rel(got[s], ref) < tol, (s, rel(got[s], ref))


@pytest.mark.parametrize("la,lb,ld", [(0, 0, 0), (3, 5, 8), (12, 12, 12), (20, 16, 40), (48, 48, 48), (10, 6, 30)])
@pytest.mark.parametrize("fp32", [False, True])
def test_product_batch_matches_oracle(S, la, lb, ld, fp32):
    import torch
    rng = np.random.default_rng(2000 + la + lb + ld)
    n = 9
    a = np.array([random_series(rng, la, False) for _ in range(n)])
    b = np.array([random_series(rng, lb, False) for _ in range(n)])
    g = S.ProductGrid(la, lb, ld, fp32=fp32)
    got = g.multiply(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()).cpu().numpy()
    g.close()
    tol = 2e-6 if fp32 else 1e-12
    for s in range(n):
        ref = O.product_pixel(a[s], la, False, b[s], lb, False, ld, False)
        assert rel(got[s], ref) < tol, (s, rel(got[s], ref))


def test_rotate_then_multiply_sh_algebra_batch(S):
    """The SH algebra batch at l_max 48 on a sample: rotate every series by
    its own Euler angles (FP64 recursion, FP32 apply), multiply consecutive
    pairs, truncate to 48; both stages against the oracle."""
    import torch
    rng = np.random.default_rng(48)
    L, n = 48, 16
    series = np.array([random_series(rng, L, False) for _ in range(n)])
    R = np.array([r for _, r in random_rotations(rng, n)])
    rot = S.rotate_batch(torch.from_numpy(series).cuda(), torch.from_numpy(R).cuda(), L, fp32=True)
    g = S.ProductGrid(L, L, L, fp32=True)
    prod = g.multiply(rot[0::2].contiguous(), rot[1::2].contiguous()).cpu().numpy()
    rot = rot.cpu().numpy()
    for s in range(0, n, 2):
        r0 = O.rotate(series[s], L, False, O.rotation_plan(L, R[s]))
        r1 = O.rotate(series[s + 1], L, False, O.rotation_plan(L, R[s + 1]))
        assert rel(rot[s], r0) < 2e-6
        ref = O.product_pixel(r0, L, False, r1, L, False, L, False)
        assert rel(prod[s // 2], ref) < 4e-6
