"""sphradiometer_b200: B200-native (sm_100a) full-sky cross-power path.

The product is ``libsphradiometer_b200.so`` (``csrc/``), a drop-in for the
reference's C ABI (``include/sphradiometer/*.h``) plus a batched,
device-resident API (``include/sphradiometer_b200.h``).  This module is the
Python host side over that C ABI, used by the tests and the benchmark; it
holds no numerics of its own, and it raises if the library is missing.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import last_error, load, series_length, series_to_numpy, numpy_to_series, array_to_numpy, rotation_plan_flat

PREC_FP64 = 0
PREC_FP32 = 1
PREC_BF16X3 = 2
PREC_BF16X6 = 3
PRECISIONS = {"fp64": PREC_FP64, "fp32": PREC_FP32, "bf16x3": PREC_BF16X3, "bf16x6": PREC_BF16X6}


class SphradError(RuntimeError):
    pass


def _check(ptr, what: str):
    if not ptr:
        raise SphradError(f"{what} failed: {last_error()}")
    return ptr


class Network:
    """A detector network with its frequency-domain correlation plan.

    ``positions``: n_det x 3 phase centres in light-seconds.  ``l_max``:
    power l_max of every baseline (the plan is built directly at
    min(l_max, native) with ``correlator_network_plan_fd_new_l``); ``None``
    builds at each baseline's native l_max as ``correlator_network_plan_fd_new``
    does.
    """

    def __init__(self, positions, n: int, delta_t: float, l_max: int | None = None):
        L = load()
        self.positions = np.asarray(positions, np.float64)
        self.n, self.delta_t = int(n), float(delta_t)
        self._inst = _check(L.instrument_array_new(0), "instrument_array_new")
        for p in self.positions:
            _check(L.instrument_array_append(self._inst, _check(L.instrument_new(p[0], p[1], p[2], None), "instrument_new")),
                   "instrument_array_append")
        self._bl = _check(L.correlator_network_baselines_new(self._inst), "correlator_network_baselines_new")
        if l_max is None:
            self._plan = _check(L.correlator_network_plan_fd_new(self._bl, self.n, self.delta_t), "correlator_network_plan_fd_new")
        else:
            self._plan = _check(L.correlator_network_plan_fd_new_l(self._bl, self.n, self.delta_t, int(l_max)),
                                "correlator_network_plan_fd_new_l")
        self.n_det = len(self.positions)
        self.n_baselines = self._bl.contents.n_baselines

    @property
    def plan(self):
        return self._plan

    def baseline(self, k: int):
        return self._bl.contents.baselines[k].contents

    def plan_fd(self, k: int):
        return self._plan.contents.plans[k]

    def baseline_l_max(self, k: int) -> int:
        return self.plan_fd(k).contents.power_1d.contents.l_max

    @property
    def l_max(self) -> int:
        return max(self.baseline_l_max(k) for k in range(self.n_baselines))

    def delay_table(self, k: int) -> np.ndarray:
        return array_to_numpy(self.plan_fd(k).contents.delay_product)

    def rotation_flat(self, k: int) -> np.ndarray:
        return rotation_plan_flat(self.plan_fd(k).contents.rotation_plan)

    def set_l(self, l_max: int):
        _check(load().correlator_network_plan_fd_set_l(self._plan, int(l_max)), "correlator_network_plan_fd_set_l")

    def integrate(self, fseries, sky_l_max: int | None = None) -> np.ndarray:
        """correlator_network_integrate_power_fd on one segment: fseries is
        n_det x n (full conjugate-filled spectra).  Returns the sky a_lm."""
        L = load()
        F = [np.ascontiguousarray(f, np.complex128) for f in fseries]
        ptrs = (C.c_void_p * len(F))(*[f.ctypes.data for f in F])
        lm = self.l_max if sky_l_max is None else sky_l_max
        sky = _check(L.sh_series_new_zero(lm, 0), "sh_series_new_zero")
        try:
            _check(L.correlator_network_integrate_power_fd(sky, ptrs, self._plan), "correlator_network_integrate_power_fd")
            return series_to_numpy(sky)
        finally:
            L.sh_series_free(sky)

    def integrate_baseline(self, k: int, a, b) -> np.ndarray:
        L = load()
        a = np.ascontiguousarray(a, np.complex128)
        b = np.ascontiguousarray(b, np.complex128)
        out = _check(L.correlator_baseline_integrate_power_fd(a.ctypes.data, b.ctypes.data, self.plan_fd(k)),
                     "correlator_baseline_integrate_power_fd")
        try:
            return series_to_numpy(out)
        finally:
            L.sh_series_free(out)

    def close(self):
        L = load()
        if getattr(self, "_plan", None):
            L.correlator_network_plan_fd_free(self._plan)
            self._plan = None
        if getattr(self, "_bl", None):
            L.correlator_network_baselines_free(self._bl)
            self._bl = None
        if getattr(self, "_inst", None):
            L.instrument_array_free(self._inst)
            self._inst = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class TimeDomainNetwork:
    """A detector network with its time-domain correlation plan
    (correlator_network_plan_td_new, correlator.c:820-858).

    ``positions``: n_det x 3 phase centres in light-seconds.
    """

    def __init__(self, positions, delta_t: float):
        L = load()
        self.delta_t = float(delta_t)
        self._inst = _check(L.instrument_array_new(0), "instrument_array_new")
        for p in np.asarray(positions, np.float64):
            _check(L.instrument_array_append(self._inst, _check(L.instrument_new(p[0], p[1], p[2], None), "instrument_new")),
                   "instrument_array_append")
        self._bl = _check(L.correlator_network_baselines_new(self._inst), "correlator_network_baselines_new")
        self._plan = _check(L.correlator_network_plan_td_new(self._bl, self.delta_t), "correlator_network_plan_td_new")
        self.n_baselines = self._bl.contents.n_baselines

    def baseline(self, k: int):
        return self._bl.contents.baselines[k].contents

    def plan_td(self, k: int):
        return self._plan.contents.plans[k]

    def transient(self, k: int) -> int:
        return self.plan_td(k).contents.transient

    def power_l_max(self, k: int) -> int:
        return self.plan_td(k).contents.power_1d.contents.l_max

    @property
    def l_max(self) -> int:
        return max(self.power_l_max(k) for k in range(self.n_baselines))

    def projections(self, k: int):
        p = self.plan_td(k).contents
        return array_to_numpy(p.proj_a), array_to_numpy(p.proj_b)

    def rotation_flat(self, k: int) -> np.ndarray:
        return rotation_plan_flat(self.plan_td(k).contents.rotation_plan)

    def integrate(self, tseries, windows, sky_l_max: int | None = None) -> np.ndarray:
        """correlator_network_integrate_power_td: tseries is n_det x n
        samples, windows one array of n - 2 transient weights per baseline.
        Returns the sky a_lm."""
        L = load()
        ts = [np.ascontiguousarray(t, np.float64) for t in tseries]
        ws = [np.ascontiguousarray(w, np.float64) for w in windows]
        tp = (C.c_void_p * len(ts))(*[t.ctypes.data for t in ts])
        wp = (C.c_void_p * len(ws))(*[w.ctypes.data for w in ws])
        lm = self.l_max if sky_l_max is None else sky_l_max
        sky = _check(L.sh_series_new_zero(lm, 0), "sh_series_new_zero")
        try:
            _check(L.correlator_network_integrate_power_td(sky, tp, len(ts[0]), wp, self._plan), "correlator_network_integrate_power_td")
            return series_to_numpy(sky)
        finally:
            L.sh_series_free(sky)

    def integrate_baseline(self, k: int, a, b, window) -> np.ndarray:
        """correlator_baseline_integrate_power_td of baseline k."""
        L = load()
        a = np.ascontiguousarray(a, np.float64)
        b = np.ascontiguousarray(b, np.float64)
        w = np.ascontiguousarray(window, np.float64)
        out = _check(L.correlator_baseline_integrate_power_td(a.ctypes.data, b.ctypes.data, w.ctypes.data, len(a), self.plan_td(k)),
                     "correlator_baseline_integrate_power_td")
        try:
            return series_to_numpy(out)
        finally:
            L.sh_series_free(out)

    def close(self):
        L = load()
        if getattr(self, "_plan", None):
            L.correlator_network_plan_td_free(self._plan)
            self._plan = None
        if getattr(self, "_bl", None):
            L.correlator_network_baselines_free(self._bl)
            self._bl = None
        if getattr(self, "_inst", None):
            L.instrument_array_free(self._inst)
            self._inst = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def generate_alm_skys(net_p: Network, net_n: Network, series, gmst: float, logprior) -> tuple[np.ndarray, np.ndarray]:
    """sphrad_generate_alm_skys (inspiral_sky_map.c:869-1101): series is
    n_det x n complex SNR series, net_p / net_n the networks whose plans were
    multiplied by the projection of each polarisation sign, logprior the
    (L+1)^2 prior coefficients.  Returns (sky_p, sky_n)."""
    L = load()
    z = [np.ascontiguousarray(s, np.complex128) for s in series]
    ptrs = (C.c_void_p * len(z))(*[s.ctypes.data for s in z])
    lp = np.asarray(logprior, np.complex128)
    l_max = int(round(np.sqrt(lp.size))) - 1
    prior = numpy_to_series(lp, l_max, False)
    sp, sn = C.POINTER(_abi.sh_series)(), C.POINTER(_abi.sh_series)()
    try:
        if L.sphrad_generate_alm_skys(C.byref(sp), C.byref(sn), net_p.plan, net_n.plan, ptrs, len(z[0]), float(gmst), prior):
            raise SphradError("sphrad_generate_alm_skys: " + last_error())
        out = (series_to_numpy(sp), series_to_numpy(sn))
        L.sh_series_free(sp)
        L.sh_series_free(sn)
        return out
    finally:
        L.sh_series_free(prior)


def batch_generate_alm_skys(bp_p: "BatchPlan", bp_n: "BatchPlan", fplan: "FseriesPlan", ctseries, gmst=None, logprior=None, stream=None):
    """sphrad_batch_generate_alm_skys: ctseries complex128 CUDA
    [n_det][n_ev][n]; gmst float64 CUDA [n_ev] or None; logprior complex128
    CUDA [(L+1)^2] or None.  Returns (sky_p, sky_n), complex128 CUDA
    [n_ev][(L+1)^2]."""
    import torch
    L = load()
    assert ctseries.is_cuda and ctseries.dtype == torch.complex128 and ctseries.is_contiguous()
    n_det, n_ev, ldt = ctseries.shape
    nq = (bp_p.l_max + 1) ** 2
    sky_p = torch.empty((n_ev, nq), dtype=torch.complex128, device=ctseries.device)
    sky_n = torch.empty_like(sky_p)
    need = L.sphrad_batch_alm_skys_workspace_size(bp_p._p, bp_n._p, n_ev)
    ws = torch.empty(max(need, 16), dtype=torch.uint8, device=ctseries.device)
    st = stream if stream is not None else torch.cuda.current_stream()
    g = gmst.data_ptr() if gmst is not None else None
    pr = logprior.data_ptr() if logprior is not None else None
    if L.sphrad_batch_generate_alm_skys(bp_p._p, bp_n._p, fplan._p, ctseries.data_ptr(), n_ev, ldt, g, pr, sky_p.data_ptr(), sky_n.data_ptr(), ws.data_ptr(),
                                        ws.numel(), st.cuda_stream):
        raise SphradError("sphrad_batch_generate_alm_skys: " + last_error())
    return sky_p, sky_n


def projection_matrix_delay(phase_centre, n: int, l_max: int, delta_t: float) -> np.ndarray:
    """projection_matrix_delay (projection.c:110-131): n x length(l_max,
    polar) coefficients of the sinc delay taps of a phase centre
    (light-seconds); polar when it lies on the z axis."""
    L = load()
    p = np.asarray(phase_centre, np.float64)
    inst = _check(L.instrument_new(p[0], p[1], p[2], None), "instrument_new")
    try:
        arr = _check(L.projection_matrix_delay(int(n), int(l_max), inst.contents.phase_centre, float(delta_t)), "projection_matrix_delay")
        try:
            return array_to_numpy(arr)
        finally:
            L.sh_series_array_free(arr)
    finally:
        L.instrument_free(inst)


class BatchPlan:
    """Batched device-resident integrator over a Network (sphrad_batch_*).

    ``integrate(F, gmst)``: F is a torch complex128 CUDA tensor
    [n_det][n_seg][ld] holding the n/2+1 unique bins of each segment's
    spectrum; gmst an optional float64 CUDA tensor [n_seg].  Returns a
    complex128 CUDA tensor [n_seg][(l_max+1)^2].
    """

    def __init__(self, net: Network, precision: str | int = "bf16x3"):
        self.precision = PRECISIONS.get(precision, precision) if isinstance(precision, str) else int(precision)
        self.net = net
        self._p = _check(load().sphrad_batch_plan_new(net.plan, self.precision), "sphrad_batch_plan_new")
        self.l_max = load().sphrad_batch_plan_l_max(self._p)
        self.bins = load().sphrad_batch_plan_bins(self._p)
        self._ws = None
        self._ws_bytes = 0

    def workspace(self, n_seg: int):
        import torch
        need = load().sphrad_batch_workspace_size(self._p, n_seg)
        if self._ws is None or self._ws_bytes < need:
            self._ws = torch.zeros(max(need, 16), dtype=torch.uint8, device="cuda")
            self._ws_bytes = need
        return self._ws

    def integrate(self, F, gmst=None, out=None, stream=None):
        import torch
        assert F.is_cuda and F.dtype == torch.complex128 and F.dim() == 3 and F.stride(2) == 1
        n_det, n_seg, ld = F.shape
        # the stride of a size-1 dimension carries no layout
        assert (n_seg == 1 or F.stride(1) == ld) and (n_det == 1 or F.stride(0) == n_seg * ld), "spectra must be contiguous [n_det][n_seg][ld]"
        nq = (self.l_max + 1) ** 2
        if out is None:
            out = torch.empty((n_seg, nq), dtype=torch.complex128, device=F.device)
        ws = self.workspace(n_seg)
        st = stream if stream is not None else torch.cuda.current_stream()
        rc = load().sphrad_batch_integrate(self._p, F.data_ptr(), n_seg, ld, gmst.data_ptr() if gmst is not None else None,
                                           out.data_ptr(), ws.data_ptr(), self._ws_bytes, st.cuda_stream)
        if rc:
            raise SphradError("sphrad_batch_integrate: " + last_error())
        return out

    def integrate_tseries(self, fplan: "FseriesPlan", x, gmst=None, out=None, stream=None):
        """Skies from real time series: x a float64 CUDA tensor
        [n_det][n_seg][ldt] (ldt even, >= n), transformed and whitened by
        fplan on the GPU, then integrated (sphrad_batch_integrate_tseries)."""
        import torch
        assert x.is_cuda and x.dtype == torch.float64 and x.dim() == 3 and x.stride(2) == 1
        n_det, n_seg, ldt = x.shape
        assert (n_seg == 1 or x.stride(1) == ldt) and (n_det == 1 or x.stride(0) == n_seg * ldt), "time series must be contiguous [n_det][n_seg][ldt]"
        nq = (self.l_max + 1) ** 2
        if out is None:
            out = torch.empty((n_seg, nq), dtype=torch.complex128, device=x.device)
        need = load().sphrad_batch_tseries_workspace_size(self._p, n_seg)
        if getattr(self, "_tws", None) is None or self._tws.numel() < need:
            self._tws = torch.zeros(max(need, 16), dtype=torch.uint8, device="cuda")
        st = stream if stream is not None else torch.cuda.current_stream()
        rc = load().sphrad_batch_integrate_tseries(self._p, fplan._p, x.data_ptr(), n_seg, ldt, gmst.data_ptr() if gmst is not None else None,
                                                   out.data_ptr(), self._tws.data_ptr(), self._tws.numel(), st.cuda_stream)
        if rc:
            raise SphradError("sphrad_batch_integrate_tseries: " + last_error())
        return out

    def integrate_host(self, F_host: np.ndarray, gmst_host: np.ndarray | None = None, out: np.ndarray | None = None):
        n_det, n_seg, ld = F_host.shape
        assert F_host.flags.c_contiguous and F_host.dtype == np.complex128
        nq = (self.l_max + 1) ** 2
        if out is None:
            out = np.empty((n_seg, nq), np.complex128)
        g = None
        if gmst_host is not None:
            gmst_host = np.ascontiguousarray(gmst_host, np.float64)
            g = gmst_host.ctypes.data
        rc = load().sphrad_batch_integrate_host(self._p, F_host.ctypes.data, n_seg, ld, g, out.ctypes.data)
        if rc:
            raise SphradError("sphrad_batch_integrate_host: " + last_error())
        return out

    def autotune(self, F):
        import torch
        n_det, n_seg, ld = F.shape
        ws = self.workspace(n_seg)
        out = torch.empty((n_seg, (self.l_max + 1) ** 2), dtype=torch.complex128, device=F.device)
        k = load().sphrad_batch_autotune(self._p, F.data_ptr(), n_seg, ld, out.data_ptr(), ws.data_ptr(), self._ws_bytes,
                                         torch.cuda.current_stream().cuda_stream)
        if k < 0:
            raise SphradError("sphrad_batch_autotune: " + last_error())
        return k

    def split(self, n_seg: int) -> int:
        return load().sphrad_batch_get_split(self._p, n_seg)

    def set_split(self, n_seg: int, split: int):
        load().sphrad_batch_set_split(self._p, n_seg, split)

    def pipeline(self, n_seg: int) -> int:
        """Pipeline variant of the tcgen05 contraction for n_seg segments."""
        return load().sphrad_batch_pipeline(self._p, n_seg)

    def set_pipeline(self, n_seg: int, variant: int):
        """Pin the pipeline variant for n_seg (-1 = default)."""
        if load().sphrad_batch_set_pipeline(self._p, n_seg, variant) < 0:
            raise SphradError("sphrad_batch_set_pipeline: " + last_error())

    def ctas(self, n_seg: int) -> int:
        """CTAs of the tcgen05 contraction for n_seg segments."""
        return load().sphrad_batch_get_ctas(self._p, n_seg)

    def set_ctas(self, n_seg: int, ctas: int):
        """Pin the tcgen05 contraction's CTA count for n_seg (0 = default)."""
        if load().sphrad_batch_set_ctas(self._p, n_seg, ctas) < 0:
            raise SphradError("sphrad_batch_set_ctas: " + last_error())

    def kernels_per_call(self) -> int:
        return load().sphrad_batch_kernels_per_call(self._p)

    def status(self) -> int:
        return load().sphrad_batch_status(self._p)

    def close(self):
        if getattr(self, "_p", None):
            load().sphrad_batch_plan_free(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


GRID_GL = 0
GRID_CELL = 1
GRID_HEALPIX = 2


class FseriesPlan:
    """Real time series to (whitened) half spectra on the GPU
    (sphrad_fseries_plan_*, sphrad_tseries_to_fseries)."""

    def __init__(self, n: int, psd: np.ndarray | None = None):
        self.n = int(n)
        self._psd = None if psd is None else np.ascontiguousarray(psd, dtype=np.float64)
        if self._psd is not None:
            assert self._psd.shape == (self.n // 2 + 1,)
        ptr = self._psd.ctypes.data if self._psd is not None else None
        self._p = _check(load().sphrad_fseries_plan_new(self.n, ptr), "sphrad_fseries_plan_new")

    def transform(self, x, out=None, stream=None):
        """x: float64 CUDA tensor [..., n] (rows contiguous); returns
        complex128 [..., n/2 + 1]."""
        import torch
        assert x.is_cuda and x.dtype == torch.float64 and x.shape[-1] == self.n and x.is_contiguous()
        rows = x.numel() // self.n
        if out is None:
            out = torch.empty(tuple(x.shape[:-1]) + (self.n // 2 + 1,), dtype=torch.complex128, device=x.device)
        st = stream if stream is not None else torch.cuda.current_stream()
        if load().sphrad_tseries_to_fseries(self._p, x.data_ptr(), rows, self.n, out.data_ptr(), self.n // 2 + 1, st.cuda_stream):
            raise SphradError("sphrad_tseries_to_fseries: " + last_error())
        return out

    def transform_complex(self, z, out=None, stream=None):
        """z: complex128 CUDA tensor [..., n] (rows contiguous), n <= 8192;
        returns the unnormalised forward DFTs, complex128 [..., n]
        (correlator_ctseries_to_fseries)."""
        import torch
        assert z.is_cuda and z.dtype == torch.complex128 and z.shape[-1] == self.n and z.is_contiguous()
        rows = z.numel() // self.n
        if out is None:
            out = torch.empty_like(z)
        st = stream if stream is not None else torch.cuda.current_stream()
        if load().sphrad_ctseries_to_fseries(self._p, z.data_ptr(), rows, self.n, out.data_ptr(), self.n, st.cuda_stream):
            raise SphradError("sphrad_ctseries_to_fseries: " + last_error())
        return out

    def transform_complex_host(self, z: np.ndarray) -> np.ndarray:
        """One host complex series -> its n-bin spectrum."""
        z = np.ascontiguousarray(z, dtype=np.complex128)
        assert z.shape == (self.n,)
        out = np.empty(self.n, dtype=np.complex128)
        if load().sphrad_ctseries_to_fseries_host(self._p, z.ctypes.data, out.ctypes.data):
            raise SphradError("sphrad_ctseries_to_fseries_host: " + last_error())
        return out

    def transform_host(self, x: np.ndarray) -> np.ndarray:
        """One host series -> the full n-bin spectrum (drop-in for
        correlator_tseries_to_fseries)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        assert x.shape == (self.n,)
        out = np.empty(self.n, dtype=np.complex128)
        if load().sphrad_tseries_to_fseries_host(self._p, x.ctypes.data, out.ctypes.data):
            raise SphradError("sphrad_tseries_to_fseries_host: " + last_error())
        return out

    def close(self):
        if self._p:
            load().sphrad_fseries_plan_free(self._p)
            self._p = None


class SkyGrid:
    """Batched inverse SHT onto a theta x phi grid (sphrad_sky_grid_*).

    ``kind``: "gl" (the reference's Gauss-Legendre mesh rows), "cell"
    (theta_i = pi (i + 1/2) / ntheta), columns phi_j = 2 pi j / nphi; or
    "healpix" (ntheta = nside, nphi ignored: 4 nside - 1 rings, 12 nside^2
    pixels in RING order).  ``render(sky)``: sky a complex128 CUDA tensor
    [n_sky][(L+1)^2] -> float32 [n_sky][ntheta][nphi] (healpix: [n_sky][12
    nside^2]) = Re f.  ``argmax(sky, l_use)`` -> (theta, phi) float64 CUDA
    tensors of each sky's best pixel (not on healpix grids).
    """

    def __init__(self, l_max: int, ntheta: int, nphi: int = 0, kind: str = "cell", fp32: bool = True):
        self.l_max, self.ntheta, self.nphi = int(l_max), int(ntheta), int(nphi)
        self.kind = kind
        k = {"gl": GRID_GL, "cell": GRID_CELL, "healpix": GRID_HEALPIX}[kind]
        self._g = _check(load().sphrad_sky_grid_new(self.l_max, k, self.ntheta, self.nphi, 1 if fp32 else 0), "sphrad_sky_grid_new")
        self.n_rows = load().sphrad_sky_grid_rows(self._g, None)
        self.n_pixels = load().sphrad_sky_grid_pixels(self._g)
        self._scratch = None

    def rows(self) -> np.ndarray:
        th = np.empty(self.n_rows, np.float64)
        load().sphrad_sky_grid_rows(self._g, th.ctypes.data)
        return th

    def _scr(self, n_sky: int):
        import torch
        need = load().sphrad_sky_grid_scratch_size(self._g, n_sky)
        if self._scratch is None or self._scratch.numel() < need:
            self._scratch = torch.empty(max(need, 16), dtype=torch.uint8, device="cuda")
        return self._scratch

    @staticmethod
    def _sky_l(sky) -> int:
        L = int(round(sky.shape[1] ** 0.5)) - 1
        assert (L + 1) ** 2 == sky.shape[1], "sky rows must hold (l_max+1)^2 coefficients"
        return L

    def render(self, sky, out=None):
        import torch
        assert sky.is_cuda and sky.dtype == torch.complex128 and sky.is_contiguous()
        n = sky.shape[0]
        if out is None:
            shape = (n, self.n_pixels) if self.kind == "healpix" else (n, self.ntheta, self.nphi)
            out = torch.empty(shape, dtype=torch.float32, device=sky.device)
        scr = self._scr(n)
        rc = load().sphrad_sky_render(self._g, sky.data_ptr(), n, self._sky_l(sky), out.data_ptr(), scr.data_ptr(), scr.numel(),
                                      torch.cuda.current_stream().cuda_stream)
        if rc:
            raise SphradError("sphrad_sky_render: " + last_error())
        return out

    def argmax(self, sky, l_use: int | None = None):
        import torch
        assert sky.is_cuda and sky.dtype == torch.complex128 and sky.is_contiguous()
        n = sky.shape[0]
        L = self._sky_l(sky)
        th = torch.empty(n, dtype=torch.float64, device=sky.device)
        ph = torch.empty(n, dtype=torch.float64, device=sky.device)
        scr = self._scr(n)
        rc = load().sphrad_sky_grid_argmax(self._g, sky.data_ptr(), n, L, L if l_use is None else int(l_use), th.data_ptr(), ph.data_ptr(),
                                           scr.data_ptr(), scr.numel(), torch.cuda.current_stream().cuda_stream)
        if rc:
            raise SphradError("sphrad_sky_grid_argmax: " + last_error())
        return th, ph

    def close(self):
        if getattr(self, "_g", None):
            load().sphrad_sky_grid_free(self._g)
            self._g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def refine_peaks(sky, theta0, phi0):
    """Local maxima of Re f from (theta0, phi0) (sphrad_sky_refine_peaks).
    Returns (out [n][4] = theta, phi, Re f, angle moved; status [n])."""
    import torch
    n = sky.shape[0]
    L = SkyGrid._sky_l(sky)
    out = torch.empty((n, 4), dtype=torch.float64, device=sky.device)
    st = torch.empty(n, dtype=torch.int32, device=sky.device)
    rc = load().sphrad_sky_refine_peaks(sky.data_ptr(), n, L, theta0.contiguous().data_ptr(), phi0.contiguous().data_ptr(), out.data_ptr(),
                                        st.data_ptr(), torch.cuda.current_stream().cuda_stream)
    if rc:
        raise SphradError("sphrad_sky_refine_peaks: " + last_error())
    return out, st


def sky_peaks(sky):
    """The reference's localisation (l <= 6 mesh search + refinement) of the
    maximum of Re f of every sky (sphrad_sky_peaks)."""
    import torch
    n = sky.shape[0]
    L = SkyGrid._sky_l(sky)
    out = torch.empty((n, 4), dtype=torch.float64, device=sky.device)
    st = torch.empty(n, dtype=torch.int32, device=sky.device)
    rc = load().sphrad_sky_peaks(sky.data_ptr(), n, L, out.data_ptr(), st.data_ptr(), torch.cuda.current_stream().cuda_stream)
    if rc:
        raise SphradError("sphrad_sky_peaks: " + last_error())
    return out, st


# ---- drop-in sh_series helpers over numpy coefficient vectors -------------

def _with_series(coeff: np.ndarray, l_max: int, polar: bool):
    return numpy_to_series(coeff, l_max, polar)


def to_mesh(coeff: np.ndarray, l_max: int, polar: bool = False):
    """sh_series_to_mesh: returns (mesh [nt][nphi] complex, cos theta rows)."""
    L = load()
    s = _with_series(coeff, l_max, polar)
    try:
        nt, npx = C.c_int(), C.c_int()
        x = C.POINTER(C.c_double)()
        m = L.sh_series_to_mesh(s, C.byref(nt), C.byref(npx), C.byref(x))
        if not m:
            raise SphradError("sh_series_to_mesh: " + last_error())
        mesh = np.ctypeslib.as_array((C.c_double * (2 * nt.value * npx.value)).from_address(m)).view(np.complex128).reshape(nt.value, npx.value).copy()
        cx = np.ctypeslib.as_array(x, shape=(nt.value,)).copy()
        libc = C.CDLL(None)
        libc.free(C.c_void_p(m))
        libc.free(C.cast(x, C.c_void_p))
        return mesh, cx
    finally:
        L.sh_series_free(s)


def from_mesh(mesh: np.ndarray, l_max: int, polar: bool = False) -> np.ndarray:
    """sh_series_from_mesh on a [2(l_max+1)]^2 complex mesh."""
    L = load()
    s = _check(L.sh_series_new(l_max, 1 if polar else 0), "sh_series_new")
    try:
        mesh = np.ascontiguousarray(mesh, np.complex128)
        if not L.sh_series_from_mesh(s, mesh.ctypes.data):
            raise SphradError("sh_series_from_mesh: " + last_error())
        return series_to_numpy(s)
    finally:
        L.sh_series_free(s)


def product(a: np.ndarray, la: int, pa: bool, b: np.ndarray, lb: int, pb: bool, ld: int, pd: bool) -> np.ndarray:
    """sh_series_product through a product plan."""
    L = load()
    sa, sb = _with_series(a, la, pa), _with_series(b, lb, pb)
    sd = _check(L.sh_series_new_zero(ld, 1 if pd else 0), "sh_series_new_zero")
    plan = _check(L.sh_series_product_plan_new(sd, sa, sb), "sh_series_product_plan_new")
    try:
        if not L.sh_series_product(sd, sa, sb, plan):
            raise SphradError("sh_series_product: " + last_error())
        return series_to_numpy(sd)
    finally:
        L.sh_series_product_plan_free(plan)
        for s in (sa, sb, sd):
            L.sh_series_free(s)


def real_minimum(coeff: np.ndarray, l_max: int, polar: bool = False):
    """sh_series_real_minimum: (value, theta, phi)."""
    L = load()
    s = _with_series(coeff, l_max, polar)
    try:
        t, p = C.c_double(), C.c_double()
        v = L.sh_series_real_minimum(s, C.byref(t), C.byref(p))
        if v != v:
            raise SphradError("sh_series_real_minimum: " + last_error())
        return v, t.value, p.value
    finally:
        L.sh_series_free(s)


# ---- batched spherical-harmonic algebra ------------------------------------

def rotate_batch(series, R, l_max: int, polar: bool = False, fp32: bool = True, out=None):
    """sphrad_sh_rotate_batch: series complex128 CUDA [n][len], R float64
    CUDA [n][3][3] (or [n][9]) -> complex128 [n][(l_max+1)^2]."""
    import torch
    n = series.shape[0]
    assert series.is_cuda and series.dtype == torch.complex128 and series.is_contiguous()
    R = R.reshape(n, 9).contiguous()
    if out is None:
        out = torch.empty((n, (l_max + 1) ** 2), dtype=torch.complex128, device=series.device)
    need = load().sphrad_sh_rotate_batch_scratch_size(l_max, n)
    scr = torch.empty(max(need, 16), dtype=torch.uint8, device=series.device)
    rc = load().sphrad_sh_rotate_batch(series.data_ptr(), n, l_max, int(polar), R.data_ptr(), out.data_ptr(), int(fp32), scr.data_ptr(), need,
                                       torch.cuda.current_stream().cuda_stream)
    if rc:
        raise SphradError("sphrad_sh_rotate_batch: " + last_error())
    return out


class ProductGrid:
    """Batched pixel-domain products (sphrad_sh_product_*):
    ``multiply(a, b)`` for complex128 CUDA [n][(la+1)^2], [n][(lb+1)^2]."""

    def __init__(self, a_l_max: int, b_l_max: int, dest_l_max: int, fp32: bool = True):
        self.la, self.lb, self.ld = int(a_l_max), int(b_l_max), int(dest_l_max)
        self._g = _check(load().sphrad_sh_product_grid_new(self.la, self.lb, self.ld, int(fp32)), "sphrad_sh_product_grid_new")
        self._scr = None

    def multiply(self, a, b, out=None):
        import torch
        n = a.shape[0]
        if out is None:
            out = torch.empty((n, (self.ld + 1) ** 2), dtype=torch.complex128, device=a.device)
        need = load().sphrad_sh_product_scratch_size(self._g, n)
        if self._scr is None or self._scr.numel() < need:
            self._scr = torch.empty(max(need, 16), dtype=torch.uint8, device=a.device)
        rc = load().sphrad_sh_product_batch(self._g, a.contiguous().data_ptr(), b.contiguous().data_ptr(), n, out.data_ptr(), self._scr.data_ptr(),
                                            self._scr.numel(), torch.cuda.current_stream().cuda_stream)
        if rc:
            raise SphradError("sphrad_sh_product_batch: " + last_error())
        return out

    def close(self):
        if getattr(self, "_g", None):
            load().sphrad_sh_product_grid_free(self._g)
            self._g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- learned peak proposal ---------------------------------------------------

class Proposal:
    """The learned peak proposal (sphrad_proposal_*): an MLP from the l <= 12
    a_lm of a sky to a direction, trained and run by the library's tcgen05
    kernels.  Tensors are CUDA tensors on the current stream."""

    N_FEATURES = 338

    def __init__(self, max_batch: int = 4096, seed: int = 1):
        self.max_batch = int(max_batch)
        self._p = _check(load().sphrad_proposal_new(self.max_batch, int(seed)), "sphrad_proposal_new")

    @staticmethod
    def n_params() -> int:
        return int(load().sphrad_proposal_n_params())

    def params(self) -> np.ndarray:
        out = np.empty(self.n_params(), np.float32)
        if load().sphrad_proposal_get_params(self._p, out.ctypes.data):
            raise SphradError("sphrad_proposal_get_params: " + last_error())
        return out

    def set_params(self, theta: np.ndarray):
        theta = np.ascontiguousarray(theta, np.float32)
        assert theta.size == self.n_params()
        if load().sphrad_proposal_set_params(self._p, theta.ctypes.data):
            raise SphradError("sphrad_proposal_set_params: " + last_error())

    def grads(self) -> np.ndarray:
        import torch
        torch.cuda.synchronize()
        out = np.empty(self.n_params(), np.float32)
        if load().sphrad_proposal_get_grads(self._p, out.ctypes.data):
            raise SphradError("sphrad_proposal_get_grads: " + last_error())
        return out

    @staticmethod
    def _st():
        import torch
        return torch.cuda.current_stream().cuda_stream

    def sky_features(self, sky, out=None):
        import torch
        n = sky.shape[0]
        L = int(round(sky.shape[1] ** 0.5)) - 1
        if out is None:
            out = torch.empty((n, self.N_FEATURES), dtype=torch.float32, device=sky.device)
        if load().sphrad_proposal_sky_features(self._p, sky.data_ptr(), n, L, out.data_ptr(), self._st()):
            raise SphradError("sphrad_proposal_sky_features: " + last_error())
        return out

    def forward(self, features, training: bool = False):
        import torch
        n = features.shape[0]
        feats = features.contiguous()
        if load().sphrad_proposal_load(self._p, feats.data_ptr(), n, int(training), self._st()):
            raise SphradError("sphrad_proposal_load: " + last_error())
        d = torch.empty((n, 3), dtype=torch.float32, device=features.device)
        if load().sphrad_proposal_forward(self._p, n, int(training), d.data_ptr(), self._st()):
            raise SphradError("sphrad_proposal_forward: " + last_error())
        return d

    def train_step(self, features, target, lr: float) -> None:
        """One Adam step on a batch; the loss is read with ``loss``."""
        n = features.shape[0]
        self.forward(features, training=True)
        t = target.contiguous()
        if load().sphrad_proposal_backward(self._p, n, t.data_ptr(), self._st()):
            raise SphradError("sphrad_proposal_backward: " + last_error())
        if lr > 0 and load().sphrad_proposal_adam(self._p, float(lr), self._st()):
            raise SphradError("sphrad_proposal_adam: " + last_error())

    def loss(self, n: int) -> float:
        return float(load().sphrad_proposal_loss(self._p, int(n)))

    def set_mirror(self, normal=None):
        """Normal of the skies' mirror-symmetry plane (3-detector networks), or None."""
        if normal is None:
            load().sphrad_proposal_set_mirror(self._p, None)
        else:
            v = np.ascontiguousarray(normal, np.float64)
            load().sphrad_proposal_set_mirror(self._p, v.ctypes.data)

    def localise(self, vet: "SkyGrid", grid: "SkyGrid", sky, max_move_deg: float = 30.0, basin_deg: float = 6.0, dominance: float = 0.1):
        """Returns (out [n][4], status [n], n_fallback)."""
        import torch
        n = sky.shape[0]
        L = int(round(sky.shape[1] ** 0.5)) - 1
        out = torch.empty((n, 4), dtype=torch.float64, device=sky.device)
        st = torch.empty(n, dtype=torch.int32, device=sky.device)
        nf = C.c_int(0)
        if load().sphrad_proposal_localise(self._p, vet._g, grid._g, sky.data_ptr(), n, L, float(max_move_deg), float(basin_deg), float(dominance),
                                           out.data_ptr(),
                                           st.data_ptr(), C.byref(nf),
                                           self._st()):
            raise SphradError("sphrad_proposal_localise: " + last_error())
        return out, st, nf.value

    def status(self) -> int:
        return load().sphrad_proposal_status(self._p)

    def close(self):
        if getattr(self, "_p", None):
            load().sphrad_proposal_free(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- uneven batches ------------------------------------------------------------

class UnevenPlan:
    """Segments of different DFT lengths, l_max and baseline subsets of one
    network in one call (sphrad_uneven_*).  Spectra and skies are packed
    1-D complex128 CUDA tensors in the layouts ``in_offset`` / ``out_offset``."""

    def __init__(self, positions, delta_t: float, bucket_n, l_max: int, precision: str | int = "bf16x3"):
        pos = np.ascontiguousarray(positions, np.float64)
        self.n_det = pos.shape[0]
        self.bucket_n = np.ascontiguousarray(bucket_n, np.int32)
        self.l_max = int(l_max)
        prec = PRECISIONS.get(precision, precision) if isinstance(precision, str) else int(precision)
        self._p = _check(load().sphrad_uneven_plan_new(pos.ctypes.data, self.n_det, float(delta_t), self.bucket_n.ctypes.data, len(self.bucket_n),
                                                       self.l_max, prec), "sphrad_uneven_plan_new")
        self.n_seg = 0

    def set_segments(self, bucket, mask, l_max):
        b = np.ascontiguousarray(bucket, np.int32)
        m = np.ascontiguousarray(mask, np.uint32)
        l = np.ascontiguousarray(l_max, np.uint32)
        n = len(b)
        if load().sphrad_uneven_set_segments(self._p, n, b.ctypes.data, m.ctypes.data, l.ctypes.data):
            raise SphradError("sphrad_uneven_set_segments: " + last_error())
        self.n_seg = n
        self.in_offset = np.empty(n, np.int64)
        self.out_offset = np.empty(n, np.int64)
        tot = (C.c_longlong(), C.c_longlong())
        load().sphrad_uneven_layout(self._p, self.in_offset.ctypes.data, self.out_offset.ctypes.data, C.byref(tot[0]), C.byref(tot[1]))
        self.in_total, self.out_total = tot[0].value, tot[1].value
        self.seg_l_max = l.copy()

    def jobs(self) -> int:
        return load().sphrad_uneven_jobs(self._p)

    def kernels_per_call(self) -> int:
        return load().sphrad_uneven_kernels_per_call(self._p)

    def set_split(self, split: int):
        load().sphrad_uneven_set_split(self._p, int(split))

    def use_graph(self, on: bool):
        load().sphrad_uneven_use_graph(self._p, int(bool(on)))

    def set_persistent(self, on: bool):
        """One persistent contraction over every job (tcgen05 precisions)
        or one contraction per job (the default)."""
        load().sphrad_uneven_set_persistent(self._p, int(bool(on)))

    def persistent(self) -> bool:
        return bool(load().sphrad_uneven_persistent(self._p))

    def autotune(self, spectra, out=None):
        import torch
        out = self._out(spectra, out)
        if load().sphrad_uneven_autotune(self._p, spectra.data_ptr(), out.data_ptr(), torch.cuda.current_stream().cuda_stream):
            raise SphradError("sphrad_uneven_autotune: " + last_error())

    def _out(self, spectra, out):
        import torch
        assert spectra.is_cuda and spectra.dtype == torch.complex128 and spectra.numel() >= self.in_total
        if out is None:
            out = torch.empty(self.out_total, dtype=torch.complex128, device=spectra.device)
        return out

    def integrate(self, spectra, out=None):
        import torch
        out = self._out(spectra, out)
        if load().sphrad_uneven_integrate(self._p, spectra.data_ptr(), out.data_ptr(), torch.cuda.current_stream().cuda_stream):
            raise SphradError("sphrad_uneven_integrate: " + last_error())
        return out

    def unpack(self, out) -> list:
        o = out.cpu().numpy() if hasattr(out, "cpu") else np.asarray(out)
        return [o[self.out_offset[s]:self.out_offset[s] + (int(self.seg_l_max[s]) + 1) ** 2] for s in range(self.n_seg)]

    def close(self):
        if getattr(self, "_p", None):
            load().sphrad_uneven_plan_free(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
