"""ctypes view of libsphradiometer_b200's C ABI.

Struct layouts follow include/sphradiometer/*.h (themselves the reference's
src/include/sphradiometer/sh_series.h, instrument.h and correlator.h), so
Python code can walk plans and series exactly as C callers do.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsphradiometer_b200.so")


class sh_series(C.Structure):
    _fields_ = [("l_max", C.c_uint), ("polar", C.c_int), ("coeff", C.c_void_p)]


class sh_series_array(C.Structure):
    _fields_ = [("l_max", C.c_uint), ("polar", C.c_int), ("n", C.c_int),
                ("series", C.POINTER(sh_series)), ("coeff", C.c_void_p), ("stride", C.c_int)]


class sh_series_rotation_plan(C.Structure):
    _fields_ = [("l_max", C.c_uint), ("D", C.POINTER(C.c_void_p))]


class gsl_block(C.Structure):
    _fields_ = [("size", C.c_size_t), ("data", C.POINTER(C.c_double))]


class gsl_vector(C.Structure):
    _fields_ = [("size", C.c_size_t), ("stride", C.c_size_t), ("data", C.POINTER(C.c_double)),
                ("block", C.POINTER(gsl_block)), ("owner", C.c_int)]


class instrument(C.Structure):
    _fields_ = [("phase_centre", C.POINTER(gsl_vector)), ("data", C.c_void_p)]


class instrument_array(C.Structure):
    _fields_ = [("instruments", C.POINTER(C.POINTER(instrument))), ("n", C.c_int)]


class correlator_baseline(C.Structure):
    _fields_ = [("instruments", C.POINTER(instrument_array)), ("index_a", C.c_int), ("index_b", C.c_int),
                ("d", C.POINTER(gsl_vector)), ("theta", C.c_double), ("phi", C.c_double)]


class correlator_plan_fd(C.Structure):
    _fields_ = [("baseline", C.POINTER(correlator_baseline)), ("delta_t", C.c_double), ("transient", C.c_int),
                ("delay_product", C.POINTER(sh_series_array)), ("fseries_product", C.c_void_p),
                ("power_1d", C.POINTER(sh_series)), ("rotation_plan", C.POINTER(sh_series_rotation_plan))]


class correlator_plan_td(C.Structure):
    _fields_ = [("baseline", C.POINTER(correlator_baseline)), ("delta_t", C.c_double), ("transient", C.c_int),
                ("proj_a", C.POINTER(sh_series_array)), ("proj_b", C.POINTER(sh_series_array)),
                ("sample_a", C.POINTER(sh_series)), ("sample_b", C.POINTER(sh_series)), ("product", C.POINTER(sh_series)),
                ("power_1d", C.POINTER(sh_series)), ("product_plan", C.c_void_p),
                ("rotation_plan", C.POINTER(sh_series_rotation_plan))]


class correlator_network_baselines(C.Structure):
    _fields_ = [("baselines", C.POINTER(C.POINTER(correlator_baseline))), ("n_baselines", C.c_int)]


class correlator_network_plan_fd(C.Structure):
    _fields_ = [("baselines", C.POINTER(correlator_network_baselines)),
                ("plans", C.POINTER(C.POINTER(correlator_plan_fd)))]


class correlator_network_plan_td(C.Structure):
    _fields_ = [("baselines", C.POINTER(correlator_network_baselines)),
                ("plans", C.POINTER(C.POINTER(correlator_plan_td)))]


class _Cplx(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


_P = C.POINTER
_vp = C.c_void_p
_u, _i, _d, _ll, _sz = C.c_uint, C.c_int, C.c_double, C.c_longlong, C.c_size_t

# name: (restype, argtypes)
SIGNATURES = {
    "sphrad_b200_last_error": (C.c_char_p, []),
    "sphrad_b200_inject_allocation_failure": (_i, [C.c_long]),
    # sh_series basics
    "sh_series_new": (_P(sh_series), [_u, _i]),
    "sh_series_new_zero": (_P(sh_series), [_u, _i]),
    "sh_series_copy": (_P(sh_series), [_P(sh_series)]),
    "sh_series_assign": (_P(sh_series), [_P(sh_series), _P(sh_series)]),
    "sh_series_resize": (_P(sh_series), [_P(sh_series), _u]),
    "sh_series_zero": (_P(sh_series), [_P(sh_series)]),
    "sh_series_set_polar": (_P(sh_series), [_P(sh_series), _i]),
    "sh_series_free": (None, [_P(sh_series)]),
    "sh_series_get": (_Cplx, [_P(sh_series), _u, _i]),
    "sh_series_set": (_Cplx, [_P(sh_series), _u, _i, _Cplx]),
    "sh_series_Y": (_Cplx, [_u, _i, _d, _d]),
    "sh_series_eval": (_Cplx, [_P(sh_series), _d, _d]),
    "sh_series_impulse": (_P(sh_series), [_u, _d, _d]),
    "sh_series_add": (_P(sh_series), [_P(sh_series), _Cplx, _P(sh_series)]),
    "sh_series_scale": (_P(sh_series), [_P(sh_series), _Cplx]),
    "sh_series_conj": (_P(sh_series), [_P(sh_series)]),
    "sh_series_real": (_P(sh_series), [_P(sh_series)]),
    "sh_series_imag": (_P(sh_series), [_P(sh_series)]),
    "sh_series_dot": (_Cplx, [_P(sh_series), _P(sh_series)]),
    "sh_series_wigner_3j": (_d, [_i, _i, _i, _i, _i, _i]),
    "sh_series_to_mesh": (_vp, [_P(sh_series), _P(_i), _P(_i), _P(_P(_d))]),
    "sh_series_from_mesh": (_P(sh_series), [_P(sh_series), _vp]),
    "sh_series_mesh_new": (_vp, [_u, _P(_i), _P(_i), _P(_P(_d)), _P(_P(_d))]),
    "sh_series_product_plan_new": (_vp, [_P(sh_series), _P(sh_series), _P(sh_series)]),
    "sh_series_product_plan_free": (None, [_vp]),
    "sh_series_product": (_P(sh_series), [_P(sh_series), _P(sh_series), _P(sh_series), _vp]),
    "sh_series_real_minimum": (_d, [_P(sh_series), _P(_d), _P(_d)]),
    # rotation
    "euler_rotation_matrix": (_P(_d), [_d, _d, _d]),
    "sh_series_rot_matrix": (_P(_d), [_d, _d]),
    "sh_series_rotation_plan_new": (_P(sh_series_rotation_plan), [_P(sh_series), _P(_d)]),
    "sh_series_rotation_plan_free": (None, [_P(sh_series_rotation_plan)]),
    "sh_series_rotation_plan_copy": (_P(sh_series_rotation_plan), [_P(sh_series_rotation_plan)]),
    "sh_series_rotation_plan_set_l": (_P(sh_series_rotation_plan), [_P(sh_series_rotation_plan), _u]),
    "sh_series_rotation_plan_wigner_D": (_Cplx, [_P(sh_series_rotation_plan), _u, _i, _i]),
    "sh_series_rotate": (_P(sh_series), [_P(sh_series), _P(sh_series), _P(sh_series_rotation_plan)]),
    "sh_series_rotate_z": (_P(sh_series), [_P(sh_series), _P(sh_series), _d]),
    # arrays
    "sh_series_array_new": (_P(sh_series_array), [_i, _u, _i]),
    "sh_series_array_free": (None, [_P(sh_series_array)]),
    "sh_series_array_dotc": (_P(sh_series), [_P(sh_series), _P(sh_series_array), _vp]),
    "sh_series_array_dot": (_P(sh_series), [_P(sh_series), _P(sh_series_array), _vp]),
    "sh_series_array_set_l": (_P(sh_series_array), [_P(sh_series_array), _u]),
    "sh_series_array_forward_fft": (_P(sh_series_array), [_P(sh_series_array)]),
    "sh_series_array_reverse_fft": (_P(sh_series_array), [_P(sh_series_array)]),
    # instruments and correlator
    "instrument_new": (_P(instrument), [_d, _d, _d, _vp]),
    "instrument_free": (None, [_P(instrument)]),
    "instrument_array_new": (_P(instrument_array), [_i]),
    "instrument_array_append": (_P(instrument), [_P(instrument_array), _P(instrument)]),
    "instrument_array_free": (None, [_P(instrument_array)]),
    "correlator_network_baselines_new": (_P(correlator_network_baselines), [_P(instrument_array)]),
    "correlator_network_baselines_free": (None, [_P(correlator_network_baselines)]),
    "correlator_network_l_max": (_u, [_P(correlator_network_baselines), _d]),
    "correlator_baseline_power_l_max_naive": (_u, [_d, _d]),
    "correlator_plan_fd_new": (_P(correlator_plan_fd), [_P(correlator_baseline), _i, _d]),
    "correlator_plan_fd_new_l": (_P(correlator_plan_fd), [_P(correlator_baseline), _i, _d, _u]),
    "correlator_plan_fd_free": (None, [_P(correlator_plan_fd)]),
    "correlator_plan_fd_set_l": (_P(correlator_plan_fd), [_P(correlator_plan_fd), _u]),
    "correlator_network_plan_fd_new": (_P(correlator_network_plan_fd), [_P(correlator_network_baselines), _i, _d]),
    "correlator_network_plan_fd_new_l": (_P(correlator_network_plan_fd), [_P(correlator_network_baselines), _i, _d, _u]),
    "correlator_network_plan_fd_free": (None, [_P(correlator_network_plan_fd)]),
    "correlator_network_plan_fd_set_l": (_P(correlator_network_plan_fd), [_P(correlator_network_plan_fd), _u]),
    "correlator_baseline_integrate_power_fd": (_P(sh_series), [_vp, _vp, _P(correlator_plan_fd)]),
    "correlator_network_integrate_power_fd": (_P(sh_series), [_P(sh_series), _P(_vp), _P(correlator_network_plan_fd)]),
    "sphrad_b200_plan_fd_touch": (None, [_P(correlator_plan_fd)]),
    "correlator_plan_td_new": (_P(correlator_plan_td), [_P(correlator_baseline), _d]),
    "correlator_plan_td_free": (None, [_P(correlator_plan_td)]),
    "correlator_network_plan_td_new": (_P(correlator_network_plan_td), [_P(correlator_network_baselines), _d]),
    "correlator_network_plan_td_free": (None, [_P(correlator_network_plan_td)]),
    "correlator_baseline_integrate_power_td": (_P(sh_series), [_vp, _vp, _vp, _i, _P(correlator_plan_td)]),
    "correlator_network_integrate_power_td": (_P(sh_series), [_P(sh_series), _P(_vp), _i, _P(_vp), _P(correlator_network_plan_td)]),
    "projection_matrix_n_elements": (_i, [_d, _d]),
    "projection_matrix_l_max": (_u, [_d, _d]),
    "projection_matrix_delay": (_P(sh_series_array), [_u, _u, _P(gsl_vector), _d]),
    "projection_delay_element": (_d, [_d, _d, _vp]),
    "sphrad_network_plan_mult_by_projection": (_i, [_P(correlator_network_plan_fd), _d, _vp, _vp, _vp]),
    "correlator_network_plan_mult_by_projection": (_i, [_P(correlator_network_plan_fd), _d, _d, _vp]),
    "sphrad_antenna_response": (_i, [_vp, _vp, _vp, _d, _d, _d, _d]),
    "instrument_new_from_LALDetector": (_P(instrument), [_vp]),
    # precalculated plans on disk
    "make_precalc_directories": (_i, [C.c_char_p, _i]),
    "write_precalc_time_series_length": (_i, [_u, C.c_char_p]),
    "read_precalc_time_series_length": (_i, [_P(_u), C.c_char_p]),
    "write_precalc_correlator_network_plan_fd": (_i, [_P(correlator_network_plan_fd), _P(correlator_network_plan_fd), C.c_char_p]),
    "read_precalc_correlator_network_baselines": (_P(correlator_network_baselines), [_P(instrument_array), C.c_char_p]),
    "read_precalc_correlator_network_plan_fd": (_i, [_P(correlator_network_plan_fd), _P(correlator_network_plan_fd), _P(correlator_network_baselines), _i,
                                                      C.c_char_p]),
    # batched extension
    "sphrad_batch_plan_new": (_vp, [_P(correlator_network_plan_fd), _i]),
    "sphrad_batch_plan_free": (None, [_vp]),
    "sphrad_batch_plan_l_max": (_u, [_vp]),
    "sphrad_batch_plan_bins": (_i, [_vp]),
    "sphrad_batch_workspace_size": (_sz, [_vp, _i]),
    "sphrad_batch_integrate": (_i, [_vp, _vp, _i, _ll, _vp, _vp, _vp, _sz, _vp]),
    "sphrad_batch_integrate_host": (_i, [_vp, _vp, _i, _ll, _vp, _vp]),
    "sphrad_batch_get_split": (_i, [_vp, _i]),
    "sphrad_batch_get_ctas": (_i, [_vp, _i]),
    "sphrad_batch_set_ctas": (_i, [_vp, _i, _i]),
    "sphrad_batch_set_split": (_i, [_vp, _i, _i]),
    "sphrad_batch_autotune": (_i, [_vp, _vp, _i, _ll, _vp, _vp, _sz, _vp]),
    "sphrad_batch_kernels_per_call": (_i, [_vp]),
    "sphrad_batch_pipeline": (_i, [_vp, _i]),
    "sphrad_batch_set_pipeline": (_i, [_vp, _i, _i]),
    # time series to spectra
    "sphrad_fseries_plan_new": (_vp, [_i, _vp]),
    "sphrad_fseries_plan_free": (None, [_vp]),
    "sphrad_tseries_to_fseries": (_i, [_vp, _vp, _i, _ll, _vp, _ll, _vp]),
    "sphrad_tseries_to_fseries_host": (_i, [_vp, _vp, _vp]),
    "sphrad_ctseries_to_fseries": (_i, [_vp, _vp, _i, _ll, _vp, _ll, _vp]),
    "sphrad_ctseries_to_fseries_host": (_i, [_vp, _vp, _vp]),
    "sphrad_generate_alm_skys": (_i, [_P(_P(sh_series)), _P(_P(sh_series)), _P(correlator_network_plan_fd), _P(correlator_network_plan_fd), _P(_vp), _i, _d,
                                      _P(sh_series)]),
    "sphrad_batch_alm_skys_workspace_size": (_sz, [_vp, _vp, _i]),
    "sphrad_batch_generate_alm_skys": (_i, [_vp, _vp, _vp, _vp, _i, _ll, _vp, _vp, _vp, _vp, _vp, _sz, _vp]),
    "sphrad_batch_tseries_workspace_size": (_sz, [_vp, _i]),
    "sphrad_batch_integrate_tseries": (_i, [_vp, _vp, _vp, _i, _ll, _vp, _vp, _vp, _sz, _vp]),
    "sphrad_batch_status": (_i, [_vp]),
    "sphrad_batch_set_wait_limit": (_i, [_vp, C.c_ulonglong]),
    "sphrad_batch_test_withhold_stage": (_i, [_vp, _i]),
    "sphrad_batch_set_timing_events": (_i, [_vp, _vp, _vp]),
    "sphrad_batch_integrate_noalloc": (_i, [_vp, _vp, _i, _ll, _vp, _vp, _vp]),
    "sphrad_batch_integrate_weighted": (_i, [_vp, _vp, _i, _ll, _vp, _vp, _vp, _sz, _vp, _i, _vp]),
    "sphrad_uneven_plan_new": (_vp, [_vp, _i, _d, _vp, _i, _u, _i]),
    "sphrad_uneven_plan_free": (None, [_vp]),
    "sphrad_uneven_set_segments": (_i, [_vp, _i, _vp, _vp, _vp]),
    "sphrad_uneven_layout": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "sphrad_uneven_jobs": (_i, [_vp]),
    "sphrad_uneven_set_split": (_i, [_vp, _i]),
    "sphrad_uneven_autotune": (_i, [_vp, _vp, _vp, _vp]),
    "sphrad_uneven_use_graph": (_i, [_vp, _i]),
    "sphrad_uneven_set_persistent": (_i, [_vp, _i]),
    "sphrad_uneven_persistent": (_i, [_vp]),
    "sphrad_uneven_integrate": (_i, [_vp, _vp, _vp, _vp]),
    "sphrad_uneven_kernels_per_call": (_i, [_vp]),
    "sphrad_sky_grid_new": (_vp, [_u, _i, _i, _i, _i]),
    "sphrad_sky_grid_free": (None, [_vp]),
    "sphrad_sky_grid_rows": (_i, [_vp, _vp]),
    "sphrad_sky_grid_pixels": (C.c_longlong, [_vp]),
    "sphrad_healpix_nside": (_i, [_u]),
    "sphrad_sky_grid_scratch_size": (_sz, [_vp, _i]),
    "sphrad_sky_render": (_i, [_vp, _vp, _i, _u, _vp, _vp, _sz, _vp]),
    "sphrad_sky_grid_argmax": (_i, [_vp, _vp, _i, _u, _u, _vp, _vp, _vp, _sz, _vp]),
    "sphrad_sky_refine_peaks": (_i, [_vp, _i, _u, _vp, _vp, _vp, _vp, _vp]),
    "sphrad_sky_peaks": (_i, [_vp, _i, _u, _vp, _vp, _vp]),
    "sphrad_sky_set_refinement": (_i, [_i]),
    "sphrad_sky_refinement": (_i, []),
    "sphrad_sh_rotate_batch_scratch_size": (_sz, [_u, _i]),
    "sphrad_sh_rotate_batch": (_i, [_vp, _i, _u, _i, _vp, _vp, _i, _vp, _sz, _vp]),
    "sphrad_sh_product_grid_new": (_vp, [_u, _u, _u, _i]),
    "sphrad_sh_product_grid_free": (None, [_vp]),
    "sphrad_sh_product_scratch_size": (_sz, [_vp, _i]),
    "sphrad_sh_product_batch": (_i, [_vp, _vp, _vp, _i, _vp, _vp, _sz, _vp]),
    "sphrad_proposal_new": (_vp, [_i, C.c_ulonglong]),
    "sphrad_proposal_free": (None, [_vp]),
    "sphrad_proposal_n_params": (_sz, []),
    "sphrad_proposal_get_params": (_i, [_vp, _vp]),
    "sphrad_proposal_set_params": (_i, [_vp, _vp]),
    "sphrad_proposal_get_grads": (_i, [_vp, _vp]),
    "sphrad_proposal_sky_features": (_i, [_vp, _vp, _i, _u, _vp, _vp]),
    "sphrad_proposal_load": (_i, [_vp, _vp, _i, _i, _vp]),
    "sphrad_proposal_forward": (_i, [_vp, _i, _i, _vp, _vp]),
    "sphrad_proposal_backward": (_i, [_vp, _i, _vp, _vp]),
    "sphrad_proposal_adam": (_i, [_vp, C.c_float, _vp]),
    "sphrad_proposal_loss": (C.c_float, [_vp, _i]),
    "sphrad_proposal_localise": (_i, [_vp, _vp, _vp, _vp, _i, _u, _d, _d, _d, _vp, _vp, C.POINTER(_i), _vp]),
    "sphrad_proposal_set_mirror": (_i, [_vp, _vp]),
    "sphrad_proposal_status": (_i, [_vp]),
}

_lib = None


def load():
    """Load the in-tree library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m sphradiometer_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            # a symbol this build lacks fails where it is called, not here
            # (tests/test_abi_cpu.py checks that every declared one exists)
            f = getattr(L, name, None)
            if f is None:
                continue
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    e = load().sphrad_b200_last_error()
    return e.decode() if e else ""


def cplx(z: complex) -> _Cplx:
    return _Cplx(float(np.real(z)), float(np.imag(z)))


def series_length(l_max: int, polar: bool) -> int:
    return (l_max + 1) if polar else (l_max + 1) ** 2


def series_to_numpy(p) -> np.ndarray:
    """Copy of a sh_series' coefficients as complex128."""
    s = p.contents
    n = series_length(s.l_max, s.polar)
    buf = (C.c_double * (2 * n)).from_address(s.coeff)
    return np.frombuffer(buf, dtype=np.complex128, count=n).copy()


def numpy_to_series(a, l_max: int, polar: bool):
    L = load()
    p = L.sh_series_new(l_max, int(polar))
    if not p:
        raise MemoryError(last_error())
    a = np.ascontiguousarray(a, np.complex128)
    assert a.size == series_length(l_max, polar)
    C.memmove(p.contents.coeff, a.ctypes.data, a.nbytes)
    return p


def array_to_numpy(p) -> np.ndarray:
    a = p.contents
    n = a.n * a.stride
    buf = (C.c_double * (2 * n)).from_address(a.coeff)
    return np.frombuffer(buf, dtype=np.complex128, count=n).copy().reshape(a.n, a.stride)


def rotation_plan_flat(p) -> np.ndarray:
    """The plan's matrices flattened (matrix l at sum_{k<l}(2k+1)^2)."""
    rp = p.contents
    out = []
    for l in range(1, rp.l_max + 1):
        w = 2 * l + 1
        centre = rp.D[l]
        start = centre - 16 * (w * l + l)
        buf = (C.c_double * (2 * w * w)).from_address(start)
        out.append(np.frombuffer(buf, dtype=np.complex128, count=w * w).copy())
    return np.concatenate(out) if out else np.zeros(0, np.complex128)
