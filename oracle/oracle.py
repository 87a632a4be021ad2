"""ctypes bindings of the CPU oracle (oracle/sphrad_oracle.c).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, by ``__graft_entry__.smoke``
and by ``bench.py``'s CPU-baseline leg as the checker; the product package
never imports it.  Every function is a thin numpy wrapper of the C
restatement of the reference's FP64 algorithms.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libsphrad_oracle.so")
_lib = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_cp = np.ctypeslib.ndpointer(dtype=np.complex128, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


class _Cplx(C.Structure):
    """C99 double complex as returned by value (two doubles in registers)."""
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


def build() -> str:
    """Compile the oracle with its Makefile if the .so is missing or stale."""
    src = os.path.join(_HERE, "sphrad_oracle.c")
    if (not os.path.exists(_LIB_PATH)) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB_PATH)
        u, i, d = C.c_uint, C.c_int, C.c_double
        L.orc_moffset.restype = C.c_size_t
        L.orc_moffset.argtypes = [u, i]
        L.orc_lmoffset.restype = C.c_size_t
        L.orc_lmoffset.argtypes = [u, u, i]
        L.orc_length.restype = C.c_size_t
        L.orc_length.argtypes = [u, i]
        L.orc_sphPlm_array.argtypes = [i, i, d, _dp]
        L.orc_Y.restype = _Cplx
        L.orc_Y.argtypes = [u, i, d, d]
        L.orc_gl_nodes.argtypes = [i, _dp, _dp]
        L.orc_dft.argtypes = [_cp, i, i]
        L.orc_assign.argtypes = [_cp, u, i, _cp, u, i]
        L.orc_conj.argtypes = [_cp, u, i]
        L.orc_rotate_z.argtypes = [_cp, u, i, d]
        L.orc_eval.restype = _Cplx
        L.orc_eval.argtypes = [_cp, u, i, d, d]
        L.orc_to_mesh.argtypes = [_cp, u, i, _cp]
        L.orc_from_mesh.argtypes = [_cp, u, i, _cp]
        L.orc_impulse.argtypes = [_cp, u, d, d]
        L.orc_euler_rotation_matrix.argtypes = [d, d, d, _dp]
        L.orc_rot_offset.restype = C.c_size_t
        L.orc_rot_offset.argtypes = [u]
        L.orc_rot_plan_len.restype = C.c_size_t
        L.orc_rot_plan_len.argtypes = [u]
        L.orc_rotation_plan.argtypes = [u, _dp, _cp]
        L.orc_rotate.restype = i
        L.orc_rotate.argtypes = [_cp, _cp, u, i, _cp]
        L.orc_wigner_3j.restype = d
        L.orc_wigner_3j.argtypes = [i, i, i, i, i, i]
        L.orc_product_plan_length.restype = C.c_long
        L.orc_product_plan_length.argtypes = [u, i, u, i, u, i]
        L.orc_product_plan.restype = C.c_long
        L.orc_product_plan.argtypes = [u, i, u, i, u, i, _dp, _ip, _ip, _ip]
        L.orc_product_microcode.argtypes = [_cp, u, i, _cp, _cp, C.c_long, _dp, _ip, _ip, _ip]
        L.orc_product_pixel.argtypes = [_cp, u, i, _cp, u, i, _cp, u, i]
        L.orc_projection_n_elements.restype = i
        L.orc_projection_n_elements.argtypes = [d, d]
        L.orc_projection_l_max.restype = u
        L.orc_projection_l_max.argtypes = [d, d]
        L.orc_power_l_max_naive.restype = u
        L.orc_power_l_max_naive.argtypes = [d, d]
        L.orc_projection_taps.argtypes = [d, d, i, u, _dp]
        L.orc_delay_product.restype = i
        L.orc_delay_product.argtypes = [d, d, i, u, _cp]
        L.orc_baseline_integrate_power_td.restype = i
        L.orc_baseline_integrate_power_td.argtypes = [_dp, _dp, _dp, i, d, d, u, _cp, _cp]
        L.orc_baseline_integrate_power_fd.restype = i
        L.orc_baseline_integrate_power_fd.argtypes = [_cp, _cp, i, _cp, u, _cp, _cp]
        L.orc_vector_direction.argtypes = [_dp, C.POINTER(d), C.POINTER(d)]
        L.orc_render_grid.argtypes = [_cp, u, i, i, i, _dp]
        L.orc_find_near_minimum.restype = d
        L.orc_find_near_minimum.argtypes = [_cp, u, i, u, C.POINTER(d), C.POINTER(d)]
        L.orc_real_maximum.restype = d
        L.orc_real_maximum.argtypes = [_cp, u, i, C.POINTER(d), C.POINTER(d)]
        L.orc_real_minimum_ref.restype = d
        L.orc_real_minimum_ref.argtypes = [_cp, u, i, C.POINTER(d), C.POINTER(d)]
        _lib = L
    return _lib


def _c(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


def length(l_max: int, polar: bool) -> int:
    return (l_max + 1) if polar else (l_max + 1) ** 2


def lmoffset(l_max: int, l: int, m: int) -> int:
    return int(lib().orc_lmoffset(l_max, l, m))


def lm_index_arrays(l_max: int, polar: bool = False):
    """(l, m) of every position of a series in the reference's order."""
    n = length(l_max, polar)
    ls = np.zeros(n, np.int64)
    ms = np.zeros(n, np.int64)
    mm = 0 if polar else l_max
    for m in range(-mm, mm + 1):
        for l in range(abs(m), l_max + 1):
            k = lmoffset(l_max, l, m)
            ls[k] = l
            ms[k] = m
    return ls, ms


def sphPlm_array(l_max: int, m: int, x: float) -> np.ndarray:
    out = np.zeros(l_max - m + 1)
    lib().orc_sphPlm_array(l_max, m, x, out)
    return out


def Y(l: int, m: int, theta: float, phi: float) -> complex:
    r = lib().orc_Y(l, m, theta, phi)
    return complex(r.re, r.im)


def gl_nodes(n: int):
    x = np.zeros(n)
    w = np.zeros(n)
    lib().orc_gl_nodes(n, x, w)
    return x, w


def dft(a, sign: int) -> np.ndarray:
    a = _c(a).copy()
    lib().orc_dft(a, len(a), sign)
    return a


def assign(src, src_l: int, src_polar: bool, dst_l: int, dst_polar: bool) -> np.ndarray:
    out = np.zeros(length(dst_l, dst_polar), np.complex128)
    lib().orc_assign(out, dst_l, int(dst_polar), _c(src), src_l, int(src_polar))
    return out


def conj(a, l_max: int, polar: bool) -> np.ndarray:
    a = _c(a).copy()
    lib().orc_conj(a, l_max, int(polar))
    return a


def rotate_z(a, l_max: int, polar: bool, phi: float) -> np.ndarray:
    a = _c(a).copy()
    lib().orc_rotate_z(a, l_max, int(polar), phi)
    return a


def eval_at(a, l_max: int, polar: bool, theta: float, phi: float) -> complex:
    r = lib().orc_eval(_c(a), l_max, int(polar), theta, phi)
    return complex(r.re, r.im)


def to_mesh(a, l_max: int, polar: bool) -> np.ndarray:
    n = 2 * (l_max + 1)
    out = np.zeros(n * n, np.complex128)
    lib().orc_to_mesh(_c(a), l_max, int(polar), out)
    return out.reshape(n, n)


def from_mesh(mesh, l_max: int, polar: bool) -> np.ndarray:
    out = np.zeros(length(l_max, polar), np.complex128)
    lib().orc_from_mesh(out, l_max, int(polar), _c(mesh).ravel())
    return out


def impulse(l_max: int, theta: float, phi: float) -> np.ndarray:
    out = np.zeros(length(l_max, False), np.complex128)
    lib().orc_impulse(out, l_max, theta, phi)
    return out


def euler_rotation_matrix(gamma: float, beta: float, alpha: float) -> np.ndarray:
    R = np.zeros(9)
    lib().orc_euler_rotation_matrix(gamma, beta, alpha, R)
    return R


def rot_offset(l: int) -> int:
    return int(lib().orc_rot_offset(l))


def rotation_plan(l_max: int, R) -> np.ndarray:
    D = np.zeros(int(lib().orc_rot_plan_len(l_max)), np.complex128)
    lib().orc_rotation_plan(l_max, np.ascontiguousarray(R, np.float64), D)
    return D


def wigner_D(D, l: int, m: int, mp: int) -> complex:
    if l == 0:
        return 1.0
    return D[rot_offset(l) + (2 * l + 1) * (mp + l) + (m + l)]


def rotate(series, l_max: int, polar: bool, D) -> np.ndarray:
    out = np.zeros(length(l_max, False), np.complex128)
    rc = lib().orc_rotate(out, _c(series), l_max, int(polar), _c(D))
    assert rc == 0
    return out


def wigner_3j(j1, j2, j3, m1, m2, m3) -> float:
    return lib().orc_wigner_3j(j1, j2, j3, m1, m2, m3)


def product_plan(d_l, d_polar, a_l, a_polar, b_l, b_polar):
    n = lib().orc_product_plan_length(d_l, int(d_polar), a_l, int(a_polar), b_l, int(b_polar))
    f = np.zeros(n)
    do, ao, bo = (np.zeros(n, np.int32) for _ in range(3))
    lib().orc_product_plan(d_l, int(d_polar), a_l, int(a_polar), b_l, int(b_polar), f, do, ao, bo)
    return f, do, ao, bo


def product_microcode(a, a_l, a_polar, b, b_l, b_polar, d_l, d_polar, plan=None):
    """Product via the Gaunt microcode; dest l_max is min(d_l, a_l + b_l)."""
    dl = min(d_l, a_l + b_l)
    if plan is None:
        plan = product_plan(d_l, d_polar, a_l, a_polar, b_l, b_polar)
    f, do, ao, bo = plan
    out = np.zeros(length(dl, d_polar), np.complex128)
    lib().orc_product_microcode(out, dl, int(d_polar), _c(a), _c(b), len(f), f, do, ao, bo)
    return assign(out, dl, d_polar, d_l, d_polar)


def product_pixel(a, a_l, a_polar, b, b_l, b_polar, d_l, d_polar):
    out = np.zeros(length(d_l, d_polar), np.complex128)
    lib().orc_product_pixel(out, d_l, int(d_polar), _c(a), a_l, int(a_polar), _c(b), b_l, int(b_polar))
    return out


def projection_n_elements(r, dt):
    return lib().orc_projection_n_elements(r, dt)


def projection_l_max(r, dt):
    return lib().orc_projection_l_max(r, dt)


def power_l_max_naive(d, dt):
    return lib().orc_power_l_max_naive(d, dt)


def native_power_l_max(d_len: float, dt: float) -> int:
    """correlator.c:337-339: min(naive estimate, a_l_max + b_l_max)."""
    a = projection_l_max(d_len / 2, dt)
    return min(power_l_max_naive(d_len, dt), 2 * a)


def projection_taps(r, dt):
    a_l = projection_l_max(abs(r), dt)
    n_el = projection_n_elements(abs(r), dt)
    out = np.zeros(n_el * (a_l + 1))
    lib().orc_projection_taps(r, dt, n_el, a_l, out)
    return out.reshape(n_el, a_l + 1)


def delay_product(d_len: float, dt: float, n: int, l_max: int) -> np.ndarray:
    """n x (l_max+1) polar delay table of one baseline (1/n applied)."""
    D = np.zeros(n * (l_max + 1), np.complex128)
    rc = lib().orc_delay_product(d_len, dt, n, l_max, D)
    if rc:
        raise ValueError("bad delay-product arguments")
    return D.reshape(n, l_max + 1)


def vector_direction(v):
    t, p = C.c_double(), C.c_double()
    lib().orc_vector_direction(np.ascontiguousarray(v, np.float64), C.byref(t), C.byref(p))
    return t.value, p.value


def rot_matrix(theta: float, phi: float) -> np.ndarray:
    """sh_series_rotation.c:162-173: z-hat to (theta, phi)."""
    return euler_rotation_matrix(0.0, theta, phi)


def baseline_integrate_power_fd(a, b, D, l_max, Rot) -> np.ndarray:
    out = np.zeros(length(l_max, False), np.complex128)
    n = len(a)
    rc = lib().orc_baseline_integrate_power_fd(_c(a), _c(b), n, _c(D).ravel(), l_max, _c(Rot), out)
    assert rc == 0
    return out


def td_power_l_max(d_len: float, dt: float) -> int:
    """correlator.c:336-339: the time-domain plan's power l_max."""
    return min(power_l_max_naive(d_len, dt), 2 * projection_l_max(d_len / 2, dt))


def baseline_integrate_power_td(a, b, window, d_len: float, dt: float, l_max: int, Rot) -> np.ndarray:
    """Time-domain cross power of one baseline (correlator.c:648-673),
    rotated with the flat rotation plan Rot of degree l_max."""
    out = np.zeros(length(l_max, False), np.complex128)
    a = np.ascontiguousarray(a, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    w = np.ascontiguousarray(window, np.float64)
    rc = lib().orc_baseline_integrate_power_td(a, b, w, len(a), d_len, dt, l_max, _c(Rot), out)
    if rc:
        raise ValueError("time series shorter than twice the transient")
    return out


class NetworkPlan:
    """Oracle-side equivalent of a correlator_network_plan_fd at l_max."""

    def __init__(self, positions, n: int, dt: float, l_max: int):
        """Each baseline's power l_max is min(l_max, its native value), as
        correlator_network_plan_fd_set_l leaves it (correlator.c:949-959);
        skies come out at the largest of them."""
        self.positions = np.asarray(positions, np.float64)
        self.n = n
        self.dt = dt
        self.baselines = []
        nd = len(self.positions)
        for i in range(1, nd):
            for j in range(i):
                d = self.positions[i] - self.positions[j]
                th, ph = vector_direction(d)
                d_len = float(np.sqrt(d @ d))
                lb = min(l_max, native_power_l_max(d_len, dt))
                D = delay_product(d_len, dt, n, lb)
                Rot = rotation_plan(lb, rot_matrix(th, ph))
                self.baselines.append(dict(i=i, j=j, d=d, d_len=d_len, theta=th, phi=ph, l=lb, D=D, Rot=Rot))
        self.l_max = max(b["l"] for b in self.baselines)

    def integrate(self, fseries) -> np.ndarray:
        """correlator.c:993-1010 for one segment; fseries is n_det x n."""
        sky = np.zeros(length(self.l_max, False), np.complex128)
        nb = len(self.baselines)
        for b in self.baselines:
            p = baseline_integrate_power_fd(fseries[b["i"]], fseries[b["j"]], b["D"], b["l"], b["Rot"])
            sky += (1.0 / nb) * assign(p, b["l"], False, self.l_max, False)
        return sky


def render_grid(a, l_max, polar, ntheta=64, nphi=128) -> np.ndarray:
    g = np.zeros(ntheta * nphi)
    lib().orc_render_grid(_c(a), l_max, int(polar), ntheta, nphi, g)
    return g.reshape(ntheta, nphi)


def find_near_minimum(a, l_max, polar, l_lowpass=6):
    t, p = C.c_double(), C.c_double()
    v = lib().orc_find_near_minimum(_c(a), l_max, int(polar), l_lowpass, C.byref(t), C.byref(p))
    return v, t.value, p.value


def real_maximum(a, l_max, polar):
    """max Re a by the reference's method (l <= 6 start, BFGS2) with the
    gradient in the minimiser's own co-ordinates; (value, theta, phi)."""
    t, p = C.c_double(), C.c_double()
    v = lib().orc_real_maximum(_c(a), l_max, int(polar), C.byref(t), C.byref(p))
    return v, t.value, p.value


def real_minimum_ref(a, l_max, polar):
    """sh_series_real_minimum as the reference runs it (its gradient
    convention; theta, phi unconditioned); (value, theta, phi)."""
    t, p = C.c_double(), C.c_double()
    v = lib().orc_real_minimum_ref(_c(a), l_max, int(polar), C.byref(t), C.byref(p))
    return v, t.value, p.value


def rms_error(measured, exact, l_max) -> float:
    """diagnostics.c:145-175 for two non-polar series of equal l_max."""
    d = np.asarray(exact) - np.asarray(measured)
    return float(np.sqrt(np.real(np.vdot(d, d)) / (4 * np.pi)))
