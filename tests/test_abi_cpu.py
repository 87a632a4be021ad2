"""CPU-side checks of libsphradiometer_b200 (no GPU needed).

* the library loads and exports every function that include/*.h declares;
* host bookkeeping functions (assign, resize, add, conj, real/imag,
  rotate_z, eval, impulse, Y) agree with the oracle;
* GPU-backed entry points fail loudly (NULL plus an error message) when no
  CUDA device is present, rather than falling back to host code.
"""
import ctypes as C
import os
import re

import numpy as np
import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def S():
    import sphradiometer_b200 as S
    from sphradiometer_b200 import build
    build.build()
    S.load()
    return S


def declared_functions():
    names = set()
    for dp, _, fs in os.walk(os.path.join(ROOT, "include")):
        for f in fs:
            if not f.endswith(".h"):
                continue
            src = open(os.path.join(dp, f)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            src = re.sub(r"static inline[^{]*\{.*?\n\}", "", src, flags=re.S)
            for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b([a-z_][a-z0-9_]*)\s*\([^;{]*\)\s*;", src, flags=re.M):
                names.add(m.group(1))
    return names


def test_library_exports_every_declared_function(S):
    lib = S.load()
    names = declared_functions()
    assert len(names) > 80
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def _rand(rng, l_max, polar):
    n = O.length(l_max, polar)
    return rng.normal(size=n) + 1j * rng.normal(size=n)


def test_host_bookkeeping_matches_oracle(S):
    L = S.load()
    rng = np.random.default_rng(1)
    for polar in (0, 1):
        a = _rand(rng, 9, polar)
        s = S.numpy_to_series(a, 9, polar)
        # resize up and down (sh_series.c:200-233)
        L.sh_series_resize(s, 13)
        assert np.allclose(S.series_to_numpy(s), O.assign(a, 9, polar, 13, polar), atol=0, rtol=0)
        L.sh_series_resize(s, 5)
        assert np.array_equal(S.series_to_numpy(s), O.assign(a, 9, polar, 5, polar))
        L.sh_series_free(s)
    a = _rand(rng, 11, 0)
    for fn, ref in (("sh_series_conj", lambda x: O.conj(x, 11, False)),):
        s = S.numpy_to_series(a, 11, 0)
        getattr(L, fn)(s)
        assert np.allclose(S.series_to_numpy(s), ref(a), rtol=0, atol=1e-15)
        L.sh_series_free(s)
    # real + i imag reproduces the function (sh_series.c:487-600)
    s1, s2 = S.numpy_to_series(a, 11, 0), S.numpy_to_series(a, 11, 0)
    L.sh_series_real(s1)
    L.sh_series_imag(s2)
    r, i = S.series_to_numpy(s1), S.series_to_numpy(s2)
    assert np.allclose(r + 1j * i, a, atol=1e-14)
    for t, p in ((0.3, 1.2), (2.9, 5.0)):
        assert abs(np.imag(O.eval_at(r, 11, False, t, p))) < 1e-12
    L.sh_series_free(s1)
    L.sh_series_free(s2)
    # rotate_z, eval, impulse, Y
    s = S.numpy_to_series(a, 11, 0)
    L.sh_series_rotate_z(s, s, 0.7)
    assert np.allclose(S.series_to_numpy(s), O.rotate_z(a, 11, False, 0.7), atol=1e-14)
    v = L.sh_series_eval(s, 1.0, 2.0)
    ref = O.eval_at(O.rotate_z(a, 11, False, 0.7), 11, False, 1.0, 2.0)
    assert abs(complex(v.re, v.im) - ref) < 1e-12
    L.sh_series_free(s)
    imp = L.sh_series_impulse(10, 0.4, 1.9)
    assert np.allclose(S.series_to_numpy(imp), O.impulse(10, 0.4, 1.9), atol=1e-14)
    L.sh_series_free(imp)
    y = L.sh_series_Y(7, -3, 0.8, 0.2)
    assert abs(complex(y.re, y.im) - O.Y(7, -3, 0.8, 0.2)) < 1e-14


def test_add_checks_shapes(S):
    L = S.load()
    a = L.sh_series_new_zero(4, 1)
    b = L.sh_series_new_zero(6, 0)
    assert not L.sh_series_add(a, S._abi.cplx(1.0), b)  # lossy: refused
    assert L.sh_series_add(b, S._abi.cplx(1.0), a)
    L.sh_series_free(a)
    L.sh_series_free(b)


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="checks the no-GPU behaviour")
def test_gpu_entry_points_fail_loudly_without_a_device(S):
    L = S.load()
    s = L.sh_series_new_zero(4, 0)
    R = L.euler_rotation_matrix(0.1, 0.2, 0.3)
    assert not L.sh_series_rotation_plan_new(s, R)
    assert "CUDA" in S.last_error() or "device" in S.last_error()
    L.sh_series_free(s)
    with pytest.raises(S.SphradError):
        S.Network(np.array([[0, 0, 0.001], [0.001, 0, 0]]), 64, 1.0 / 256, l_max=2)


def test_library_wigner_3j_against_exact_values(S):
    """sh_series_wigner_3j (host recursion in the library) against sympy's
    exact 3-j symbols and the oracle, including the j1min = 0 and
    single-term cases and large j."""
    from sympy.physics.wigner import wigner_3j as exact
    from oracle import oracle as O
    L = S.load()
    rng = np.random.default_rng(5)
    cases = [(0, 0, 0, 0, 0, 0), (1, 1, 0, 0, 0, 0), (2, 1, 1, 0, 0, 0), (3, 2, 1, 1, -1, 0), (4, 2, 2, 0, 1, -1), (7, 3, 4, -2, 1, 1),
             (10, 10, 0, 3, -3, 0), (5, 5, 10, 5, 5, -10), (2, 3, 4, 1, 1, -2), (3, 3, 3, 0, 0, 0), (1, 2, 5, 0, 0, 0)]
    for _ in range(60):
        j2, j3 = int(rng.integers(0, 25)), int(rng.integers(0, 25))
        j1 = int(rng.integers(abs(j2 - j3), j2 + j3 + 1))
        m2, m3 = int(rng.integers(-j2, j2 + 1)), int(rng.integers(-j3, j3 + 1))
        cases.append((j1, j2, j3, -m2 - m3, m2, m3))
    for args in cases:
        ref = float(exact(*args).evalf(30))
        got = L.sh_series_wigner_3j(*args)
        assert abs(got - ref) <= 1e-13 * max(abs(ref), 1e-3), (args, got, ref)
        assert abs(got - O.wigner_3j(*args)) <= 1e-13 * max(abs(ref), 1e-3)
    for args in [(80, 60, 50, 3, -7, 4), (96, 48, 48, 0, 12, -12), (59, 59, 30, 20, -25, 5)]:
        assert abs(L.sh_series_wigner_3j(*args) - O.wigner_3j(*args)) <= 1e-12 * max(abs(O.wigner_3j(*args)), 1e-6)


def test_healpix_nside_follows_the_reference_rule():
    """sphrad_healpix_nside: lmax2nside of sh_series_healpix.cc:220-238, the
    smallest power of two not below ceil(l_max / 2 + 0.75)."""
    import math
    import sphradiometer_b200 as S
    lib = S.load()
    for L in range(0, 300):
        want = 1
        while want < math.ceil(L / 2.0 + 0.75):
            want *= 2
        assert lib.sphrad_healpix_nside(L) == want, L
    assert lib.sphrad_healpix_nside(32) == 32 and lib.sphrad_healpix_nside(25) == 16


def test_antenna_response_known_answers():
    """sphrad_antenna_response (LAL's XLALComputeDetAMResponse, Anderson et
    al. 2001 app. B): an L-shaped detector with arms along x and y sees a
    wave from overhead (declination 90 deg) with F+ = -cos 2a, Fx = sin 2a,
    a = psi + gmst - ra; any wave has F+^2 + Fx^2 independent of psi."""
    import ctypes as C
    import math
    import sphradiometer_b200 as S
    lib = S.load()
    D = ((C.c_float * 3) * 3)()
    D[0][0], D[1][1] = 0.5, -0.5
    fp, fc = C.c_double(), C.c_double()
    for psi, gmst, ra in ((0.0, 0.0, 0.0), (0.3, 1.0, 0.4), (1.2, -0.7, 2.2)):
        lib.sphrad_antenna_response(C.byref(fp), C.byref(fc), D, ra, math.pi / 2, psi, gmst)
        a = psi + gmst - ra
        assert abs(fp.value + math.cos(2 * a)) < 1e-7 and abs(fc.value - math.sin(2 * a)) < 1e-7
    norms = []
    for psi in (0.0, 0.5, 1.3):
        lib.sphrad_antenna_response(C.byref(fp), C.byref(fc), D, 0.7, 0.4, psi, 0.2)
        norms.append(fp.value ** 2 + fc.value ** 2)
    assert max(norms) - min(norms) < 1e-7


def c_caller(out_path):
    """Compile tests/c/fd_caller.c (a C program of the reference's kind)
    against include/sphradiometer and link it with the library."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lib_dir = os.path.join(ROOT, "sphradiometer_b200")
    cmd = [cc, "-O2", "-Wall", "-Wextra", "-Werror", "-std=c11", "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "c", "fd_caller.c"),
           "-L", lib_dir, "-lsphradiometer_b200", "-Wl,-rpath," + lib_dir, "-lm", "-o", str(out_path)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return str(out_path)


def test_c_caller_compiles_against_headers_and_links(tmp_path):
    """The headers compile as C (no warnings) and every function the
    drop-in FD path needs resolves in the library at link time."""
    exe = c_caller(tmp_path / "fd_caller")
    assert os.path.exists(exe)
