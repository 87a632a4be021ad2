"""ctypes view of oracle/_ref/libsphrad_ref.so -- TEST INFRASTRUCTURE ONLY.

The library is the reference's own hot-path C code (cannon-zz/sphradiometer
src/lib: correlator.c, projection.c, sh_series*.c, instrument.c,
diagnostics.c), compiled unmodified by ``make -C oracle ref`` against the
project-written FFTW/GSL/LAL stand-ins in oracle/ref_shims, plus the flat
entry points of oracle/ref_driver.c.  It needs the reference checkout to
build; where it has not been built, ``available()`` is False and callers
skip.  Used by the tests and by tests/golden/make_ref_golden.py to pin the
oracle to the reference itself; the product never loads it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libsphrad_ref.so")
REF_SRC = os.environ.get("SPHRAD_REFERENCE", "/root/reference")

_lib = None


def build(quiet: bool = True) -> bool:
    """Builds oracle/_ref when the reference checkout is present; returns
    whether the library exists afterwards."""
    if os.path.isdir(os.path.join(REF_SRC, "src", "lib")):
        r = subprocess.run(["make", "-C", HERE, "ref", f"REF={REF_SRC}"], capture_output=True, text=True)
        if r.returncode != 0 and not quiet:
            raise RuntimeError(r.stdout + r.stderr)
    return os.path.exists(LIB)


def available() -> bool:
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB)
        vp, i, d, u = C.c_void_p, C.c_int, C.c_double, C.c_uint
        cp = np.ctypeslib.ndpointer(np.complex128, flags="C_CONTIGUOUS")
        dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
        L.ref_network_new.restype = vp
        L.ref_network_new.argtypes = [i, dp, i, d, i]
        L.ref_network_free.argtypes = [vp]
        L.ref_network_n_baselines.argtypes = [vp]
        L.ref_network_baseline.argtypes = [vp, i, C.POINTER(i), C.POINTER(i), C.POINTER(d), C.POINTER(d)]
        L.ref_network_baseline_l_max.argtypes = [vp, i]
        L.ref_network_delay_table.argtypes = [vp, i, cp]
        L.ref_network_rotation.argtypes = [vp, i, cp]
        L.ref_network_integrate.argtypes = [vp, cp, u, cp]
        L.ref_rotate_z.argtypes = [cp, u, i, d, cp]
        L.ref_rotation_plan.argtypes = [u, d, d, d, cp]
        L.ref_real_minimum.restype = d
        L.ref_real_minimum.argtypes = [cp, u, i, C.POINTER(d), C.POINTER(d)]
        L.ref_product.argtypes = [cp, u, i, cp, u, i, u, i, cp]
        L.ref_to_mesh.argtypes = [cp, u, i, cp]
        L.ref_network_set_delay_table.argtypes = [vp, i, i, cp]
        L.ref_network_copy.restype = vp
        L.ref_network_copy.argtypes = [vp]
        L.ref_network_copy_free.argtypes = [vp]
        L.ref_network_integrate_rotz.argtypes = [vp, cp, d, vp, vp]
        L.ref_series_new.restype = vp
        L.ref_series_new.argtypes = [u, i]
        L.ref_series_free.argtypes = [vp]
        _lib = L
    return _lib


def _c(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


def length(l_max: int, polar: bool) -> int:
    return l_max + 1 if polar else (l_max + 1) ** 2


def rot_len(l_max: int) -> int:
    return sum((2 * l + 1) ** 2 for l in range(1, l_max + 1))


class Network:
    """correlator_network_plan_fd of the reference for detectors at
    ``positions`` (light-seconds), DFT length n, sample interval dt, then
    correlator_network_plan_fd_set_l(l_max) unless l_max is None."""

    def __init__(self, positions, n: int, dt: float, l_max=None):
        self._p = None
        pos = np.ascontiguousarray(np.asarray(positions, np.float64).ravel())
        self.n_det = len(pos) // 3
        self.n = n
        self._p = lib().ref_network_new(self.n_det, pos, n, dt, -1 if l_max is None else int(l_max))
        if not self._p:
            raise RuntimeError("correlator_network_plan_fd_new failed")
        self.n_baselines = lib().ref_network_n_baselines(self._p)

    def close(self):
        if self._p:
            lib().ref_network_free(self._p)
            self._p = None

    def __del__(self):
        self.close()

    def baseline(self, k: int):
        ia, ib, th, ph = C.c_int(), C.c_int(), C.c_double(), C.c_double()
        lib().ref_network_baseline(self._p, k, C.byref(ia), C.byref(ib), C.byref(th), C.byref(ph))
        return ia.value, ib.value, th.value, ph.value

    def baseline_l_max(self, k: int) -> int:
        return lib().ref_network_baseline_l_max(self._p, k)

    def delay_table(self, k: int) -> np.ndarray:
        L = self.baseline_l_max(k)
        out = np.zeros(self.n * (L + 1), np.complex128)
        lib().ref_network_delay_table(self._p, k, out)
        return out.reshape(self.n, L + 1)

    def rotation_flat(self, k: int) -> np.ndarray:
        out = np.zeros(rot_len(self.baseline_l_max(k)), np.complex128)
        lib().ref_network_rotation(self._p, k, out)
        return out

    def set_delay_tables(self, tables):
        """Give every baseline the n x (l_max+1) delay table tables[k] (the
        plan's own l_max), through the reference's own allocators; the
        network then integrates spectra of that length."""
        for k, D in enumerate(tables):
            D = _c(D)
            if lib().ref_network_set_delay_table(self._p, k, D.shape[0], D):
                raise RuntimeError("delay table replacement failed")
        self.n = tables[0].shape[0]

    def integrate(self, fseries, sky_l_max: int) -> np.ndarray:
        """correlator_network_integrate_power_fd; fseries is n_det x n."""
        F = _c(fseries)
        assert F.shape == (self.n_det, self.n)
        out = np.zeros((sky_l_max + 1) ** 2, np.complex128)
        if lib().ref_network_integrate(self._p, F, sky_l_max, out):
            raise RuntimeError("correlator_network_integrate_power_fd failed")
        return out


def rotate_z(a, l_max: int, polar: bool, phi: float) -> np.ndarray:
    out = np.zeros(length(l_max, polar), np.complex128)
    assert lib().ref_rotate_z(_c(a), l_max, int(polar), phi, out) == 0
    return out


def rotation_plan(l_max: int, gamma: float, beta: float, alpha: float) -> np.ndarray:
    out = np.zeros(rot_len(l_max), np.complex128)
    assert lib().ref_rotation_plan(l_max, gamma, beta, alpha, out) == 0
    return out


def real_minimum(a, l_max: int, polar: bool):
    """sh_series_real_minimum: (value, theta, phi) as the reference returns
    them (co-ordinates not conditioned)."""
    t, p = C.c_double(), C.c_double()
    v = lib().ref_real_minimum(_c(a), l_max, int(polar), C.byref(t), C.byref(p))
    return v, t.value, p.value


def product(a, a_l, a_polar, b, b_l, b_polar, d_l, d_polar) -> np.ndarray:
    out = np.zeros(length(d_l, d_polar), np.complex128)
    assert lib().ref_product(_c(a), a_l, int(a_polar), _c(b), b_l, int(b_polar), d_l, int(d_polar), out) == 0
    return out


def to_mesh(a, l_max: int, polar: bool) -> np.ndarray:
    n = 2 * (l_max + 1)
    out = np.zeros(n * n, np.complex128)
    assert lib().ref_to_mesh(_c(a), l_max, int(polar), out) == 0
    return out.reshape(n, n)
