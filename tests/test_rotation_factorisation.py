"""The identity the batched rotation kernel (k_rotate_fac) is built on,
checked on the CPU against the oracle's restatement of the reference's
Wigner-D recursion (sh_series_rotation.c:287-422) and rotation
(sh_series_rotation.c:546-589):

    rotate(c, plan of R) = Z(-alpha) P* Delta E(beta) Delta^T P Z(-gamma) c

per degree, with R = euler_rotation_matrix(gamma, beta, alpha),
Z(x) = diag(e^{i m x}), P = diag(i^m), E(b) = diag(e^{i k b}) and
Delta = D(R_y(pi/2)) (the recursion's own matrix for euler_rotation_matrix
(0, pi/2, 0)); the Euler angles are recovered from R as the kernel does
(atan2 of R's entries, gamma = 0 where sin beta = 0)."""
import numpy as np
import pytest

from oracle import oracle as O

L = 10


def _block(D, l):
    w = 2 * l + 1
    off = O.rot_offset(l)
    return D[off:off + w * w].reshape(w, w).T  # [m][m'] = element (m, m')


def _lmo(L, l, m):
    LL = L + 1
    x = m * (m - 1)
    mo = LL * m - x // 2 if m >= 0 else LL * (LL + m) + x // 2
    return mo + l - abs(m)


def _euler(R):
    R = np.asarray(R).reshape(9)
    sb = np.hypot(R[2], R[5])
    b = np.arctan2(sb, R[8])
    if sb > 1e-14:
        return np.arctan2(R[5], R[2]), b, np.arctan2(R[7], -R[6])
    s = 1.0 if R[8] >= 0 else -1.0
    return np.arctan2(R[3] * s, R[0] * s), b, 0.0


def _rotate_factorised(c, polar, R, Delta):
    a, b, g = _euler(R)
    out = np.zeros((L + 1) ** 2, complex)
    out[_lmo(L, 0, 0)] = c[0]
    for l in range(1, L + 1):
        ms = np.arange(-l, l + 1)
        if polar:
            f = np.zeros(2 * l + 1, complex)
            f[l] = c[l]
        else:
            f = np.array([c[_lmo(L, l, m)] for m in ms])
        D = _block(Delta, l).real
        t = (1j) ** ms * np.exp(-1j * ms * g) * f
        t = np.exp(1j * ms * b) * (D.T @ t)
        t = (-1j) ** ms * np.exp(-1j * ms * a) * (D @ t)
        for i, m in enumerate(ms):
            out[_lmo(L, l, m)] = t[i]
    return out


@pytest.mark.parametrize("case", range(8))
def test_factorised_rotation_equals_the_plan(case):
    rng = np.random.default_rng(700 + case)
    Delta = O.rotation_plan(L, O.euler_rotation_matrix(0.0, np.pi / 2, 0.0))
    assert np.max(np.abs(Delta.imag)) < 1e-14
    if case == 6:
        R = O.euler_rotation_matrix(0.4, 0.0, 1.3)       # beta = 0
    elif case == 7:
        R = O.euler_rotation_matrix(0.4, np.pi, 1.3)     # beta = pi
    else:
        R = O.euler_rotation_matrix(rng.uniform(0, 2 * np.pi), np.arccos(rng.uniform(-1, 1)), rng.uniform(0, 2 * np.pi))
    for polar in (False, True):
        n = O.length(L, polar)
        c = rng.normal(size=n) + 1j * rng.normal(size=n)
        ref = O.rotate(c, L, polar, O.rotation_plan(L, R))
        got = _rotate_factorised(c, polar, R, Delta)
        assert np.max(np.abs(got - ref)) < 1e-13 * np.max(np.abs(ref))
