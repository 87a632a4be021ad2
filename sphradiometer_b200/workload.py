"""Seeded synthetic inputs for the cross-power path.

Host-side numpy generator of detector data (not part of the GPU path and
never timed).  It restates the reference's injection helpers:

* ``gaussian_white_noise``      -- inject.c:48-56
* ``inject_transform_point_source`` -- inject.c:119-152 (FFT fractional
  delay by r.s / dt, periodic)
* ``inject_into``               -- inject.c:187-203
* ``tseries_to_fseries``        -- correlator.c:224-231 (r2c FFT, then the
  negative frequencies filled with conjugates)

plus the coloured-noise / chirp / whitening recipe of the demo front end
(sphradiometer_demo.c:456-460) used by the benchmark workloads.  Random
numbers come from numpy's Philox generator; a segment's seed is the
workload seed xor the segment index.
"""
from __future__ import annotations

import numpy as np

C_LIGHT = 299792458.0
R_EARTH = 6.371e6
R_EARTH_S = R_EARTH / C_LIGHT


def rng_for(seed: int, index: int = 0) -> np.random.Generator:
    return np.random.Generator(np.random.Philox(int(seed) ^ int(index)))


def vector_r_dot_s(v, theta, phi):
    """instrument.c:77-80."""
    return (v[0] * np.cos(phi) + v[1] * np.sin(phi)) * np.sin(theta) + v[2] * np.cos(theta)


def gaussian_white_noise(n: int, variance: float, rng: np.random.Generator) -> np.ndarray:
    return rng.normal(0.0, np.sqrt(variance), n)


def inject_transform_point_source(position, x, dt: float, theta: float, phi: float) -> np.ndarray:
    n = len(x)
    r_dot_s = vector_r_dot_s(position, theta, phi)
    ft = np.fft.rfft(x)
    k = np.arange(n // 2 + 1)
    ft *= np.exp(1j * 2 * np.pi * r_dot_s * k / (dt * n))
    return np.fft.irfft(ft, n)


def inject_into(position, series, injection, dt: float, ra: float, dec: float, gmst: float):
    gha = gmst - ra
    series += inject_transform_point_source(position, injection, dt, np.pi / 2 - dec, -gha)
    return series


def tseries_to_fseries(x) -> np.ndarray:
    n = len(x)
    F = np.zeros(n, np.complex128)
    h = np.fft.rfft(x)
    F[: n // 2 + 1] = h
    for i in range(1, (n + 1) // 2):
        F[n - i] = np.conj(F[i])
    return F


def random_positions(n_det: int, radius: float, rng: np.random.Generator) -> np.ndarray:
    """Detectors at isotropic random points on a sphere of the given radius
    (seconds)."""
    v = rng.normal(size=(n_det, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v * radius


def pair_positions(separation_s: float, rng: np.random.Generator) -> np.ndarray:
    """Two Earth-surface points whose chord is ``separation_s`` seconds."""
    half = np.arcsin(min(1.0, separation_s / (2 * R_EARTH_S)))
    u = rng.normal(size=3)
    u /= np.linalg.norm(u)
    w = rng.normal(size=3)
    w -= u * (w @ u)
    w /= np.linalg.norm(w)
    p0 = R_EARTH_S * (np.cos(half) * u + np.sin(half) * w)
    p1 = R_EARTH_S * (np.cos(half) * u - np.sin(half) * w)
    return np.stack([p0, p1])


def isotropic_direction(rng: np.random.Generator):
    """(theta, phi) uniform on the sphere."""
    return float(np.arccos(rng.uniform(-1, 1))), float(rng.uniform(0, 2 * np.pi))


def psd(f) -> np.ndarray:
    """S(f) = 1e-46 [(f/100)^-4 + 2 + (f/100)^2] on 20-1000 Hz, 0 outside."""
    f = np.asarray(f, np.float64)
    out = np.zeros_like(f)
    band = (f >= 20.0) & (f <= 1000.0)
    x = f[band] / 100.0
    out[band] = 1e-46 * (x ** -4 + 2.0 + x ** 2)
    return out


def chirp(n: int, dt: float, f0: float = 60.0, f1: float = 400.0, duration: float = 0.25) -> np.ndarray:
    """A Tukey-windowed linear chirp f0 -> f1, centred in the segment."""
    t = np.arange(n) * dt
    t0 = 0.5 * n * dt - 0.5 * duration
    tau = t - t0
    on = (tau >= 0) & (tau < duration)
    h = np.zeros(n)
    ph = 2 * np.pi * (f0 * tau[on] + 0.5 * (f1 - f0) * tau[on] ** 2 / duration)
    w = np.sin(np.pi * tau[on] / duration) ** 2
    h[on] = w * np.sin(ph)
    return h


def whitened_segment(positions, n: int, dt: float, theta: float, phi: float, snr: float,
                     rng: np.random.Generator, hermitian: bool = True) -> np.ndarray:
    """One segment for every detector: coloured noise plus a chirp from
    (theta, phi) (Earth-fixed), delayed per detector with the FFT
    fractional delay, then whitened by 1/sqrt(S) in the 20-1000 Hz band.
    Returns n_det x (n/2+1) (hermitian=True) or n_det x n spectra."""
    nd = len(positions)
    k = np.arange(n // 2 + 1)
    f = k / (n * dt)
    S = psd(f)
    inband = S > 0
    wh = np.zeros_like(S)
    wh[inband] = 1.0 / np.sqrt(S[inband])
    # noise with one-sided PSD S: E|X_k|^2 = n S / (2 dt)
    sigma = np.sqrt(S * n / (2 * dt) / 2.0)
    h = chirp(n, dt)
    Hf = np.fft.rfft(h)
    rho2 = 4.0 * np.sum(np.abs(Hf[inband] * dt) ** 2 / S[inband]) / (n * dt)
    h *= snr / np.sqrt(rho2) if rho2 > 0 else 0.0
    out = np.zeros((nd, n // 2 + 1), np.complex128)
    for d in range(nd):
        nz = sigma * (rng.normal(size=k.size) + 1j * rng.normal(size=k.size))
        nz[0] = nz[0].real
        if n % 2 == 0:
            nz[-1] = nz[-1].real
        x = np.fft.irfft(nz, n)
        x += inject_transform_point_source(positions[d], h, dt, theta, phi)
        out[d] = np.fft.rfft(x) * wh
    if hermitian:
        return out
    full = np.zeros((nd, n), np.complex128)
    full[:, : n // 2 + 1] = out
    for i in range(1, (n + 1) // 2):
        full[:, n - i] = np.conj(out[:, i])
    return full


def make_batch(positions, n: int, dt: float, n_seg: int, seed: int, snr_range=(6.0, 30.0)):
    """A batch of whitened segments, vectorised over segments.

    Per segment: an isotropic source direction (Earth-fixed theta, phi), an
    SNR uniform in ``snr_range`` and a GMST uniform in [0, 2 pi).  Each
    detector sees coloured Gaussian noise of PSD S(f) plus the chirp
    delayed by r_det . s (the periodic FFT delay of inject.c:119-152,
    applied as a phase ramp on the chirp's spectrum), whitened by
    1/sqrt(S) in the 20-1000 Hz band.  Returns a dict with ``F``
    (n_det x n_seg x (n/2+1) complex128), ``theta``, ``phi``, ``snr`` and
    ``gmst`` (n_seg each)."""
    rng = rng_for(seed)
    pos = np.asarray(positions, np.float64)
    nd = len(pos)
    K = n // 2 + 1
    k = np.arange(K)
    f = k / (n * dt)
    S = psd(f)
    inband = S > 0
    wh = np.zeros_like(S)
    wh[inband] = 1.0 / np.sqrt(S[inband])
    sigma = np.sqrt(S * n / (2 * dt) / 2.0)
    h = chirp(n, dt)
    Hf = np.fft.rfft(h)
    rho1 = np.sqrt(4.0 * np.sum(np.abs(Hf[inband] * dt) ** 2 / S[inband]) / (n * dt))
    theta = np.arccos(rng.uniform(-1, 1, n_seg))
    phi = rng.uniform(0, 2 * np.pi, n_seg)
    snr = rng.uniform(snr_range[0], snr_range[1], n_seg)
    gmst = rng.uniform(0, 2 * np.pi, n_seg)
    s_hat = np.stack([np.sin(theta) * np.cos(phi), np.sin(theta) * np.sin(phi), np.cos(theta)], axis=1)
    tau = s_hat @ pos.T                                   # n_seg x n_det, r . s
    F = np.empty((nd, n_seg, K), np.complex128)
    amp = snr / rho1
    for d in range(nd):
        nz = sigma[None, :] * (rng.normal(size=(n_seg, K)) + 1j * rng.normal(size=(n_seg, K)))
        nz[:, 0] = nz[:, 0].real
        if n % 2 == 0:
            nz[:, -1] = nz[:, -1].real
        sig = (amp[:, None] * Hf[None, :]) * np.exp(1j * 2 * np.pi * np.outer(tau[:, d], k) / (dt * n))
        if n % 2 == 0:
            sig[:, -1] = sig[:, -1].real   # c2r drops the Nyquist imaginary part
        F[d] = (nz + sig) * wh[None, :]
    return dict(F=F, theta=theta, phi=phi, snr=snr, gmst=gmst)


def make_tseries_batch(positions, n: int, dt: float, n_seg: int, seed: int, snr_range=(6.0, 30.0)):
    """The batch of ``make_batch`` as raw detector time series: coloured
    noise plus the delayed chirp, before any whitening.  Returns a dict
    with ``x`` (n_det x n_seg x n float64), ``psd`` (the one-sided S(k) at
    k / (n dt), k <= n/2, zero outside the 20-1000 Hz band), ``F`` (the
    whitened half spectra rfft(x) / sqrt(S), zero out of band) and ``gmst``."""
    b = make_batch(positions, n, dt, n_seg, seed, snr_range)
    K = n // 2 + 1
    S = psd(np.arange(K) / (n * dt))
    inband = S > 0
    wh = np.zeros_like(S)
    wh[inband] = 1.0 / np.sqrt(S[inband])
    # undo the whitening in band; out of band the raw series carries no power
    U = np.zeros_like(b["F"])
    U[..., inband] = b["F"][..., inband] / wh[inband]
    x = np.fft.irfft(U, n, axis=-1)
    F = np.fft.rfft(x, axis=-1) * wh
    return dict(x=np.ascontiguousarray(x), psd=np.where(inband, S, 0.0), F=F, gmst=b["gmst"])


def pattern_meshes(l_max: int, n_det: int, rng: np.random.Generator):
    """Smooth synthetic stand-ins for the antenna patterns F+ and Fx of
    n_det detectors (quadrupolar in phi, as real patterns are, with a
    per-detector orientation), sampled on the reference's mesh of l_max:
    rows acos x_i for the 2(l_max+1) Gauss-Legendre nodes in decreasing
    order, columns 2 pi j / (2(l_max+1)).  Returns (fplus, fcross), each
    n_det x nt x nt."""
    nt = 2 * (l_max + 1)
    x, _ = np.polynomial.legendre.leggauss(nt)
    th = np.arccos(x[::-1])[:, None]
    ph = 2 * np.pi * np.arange(nt)[None, :] / nt
    c = rng.uniform(0, 2 * np.pi, n_det)
    fp = np.stack([0.5 * (1 + np.cos(th) ** 2) * np.cos(2 * ph + c[k]) + 0.1 * k for k in range(n_det)])
    fc = np.stack([np.cos(th) * np.sin(2 * ph + c[k]) for k in range(n_det)])
    return np.ascontiguousarray(fp), np.ascontiguousarray(fc)


def full_from_half(half, n: int) -> np.ndarray:
    """Hermitian completion of n/2+1 bins to n bins (last axis)."""
    half = np.asarray(half)
    full = np.zeros(half.shape[:-1] + (n,), np.complex128)
    full[..., : n // 2 + 1] = half
    idx = np.arange(1, (n + 1) // 2)
    full[..., n - idx] = np.conj(half[..., idx])
    return full


def make_batch_torch(positions, n: int, dt: float, n_seg: int, seed: int, device="cuda", snr_range=(6.0, 30.0)):
    """make_batch generated on the GPU with torch (same model: isotropic
    Earth-fixed directions, SNR uniform in ``snr_range``, coloured noise,
    the chirp delayed by r_det . s, whitening), for training and evaluation
    sets of many segments.  Returns torch tensors: ``F`` (n_det x n_seg x
    (n/2+1) complex128), ``theta``, ``phi``, ``snr``, ``gmst``."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    pos = torch.as_tensor(np.asarray(positions, np.float64), device=device)
    nd = pos.shape[0]
    K = n // 2 + 1
    k = np.arange(K)
    S = psd(k / (n * dt))
    inband = S > 0
    wh = np.zeros_like(S)
    wh[inband] = 1.0 / np.sqrt(S[inband])
    sigma = np.sqrt(S * n / (2 * dt) / 2.0)
    Hf = np.fft.rfft(chirp(n, dt))
    rho1 = np.sqrt(4.0 * np.sum(np.abs(Hf[inband] * dt) ** 2 / S[inband]) / (n * dt))
    wh_t = torch.as_tensor(wh, device=device)
    sig_t = torch.as_tensor(sigma, device=device)
    Hf_t = torch.as_tensor(Hf, device=device)
    kk = torch.arange(K, dtype=torch.float64, device=device)

    def U(lo, hi):
        return lo + (hi - lo) * torch.rand(n_seg, generator=g, dtype=torch.float64, device=device)

    theta = torch.arccos(U(-1.0, 1.0))
    phi = U(0.0, 2 * np.pi)
    snr = U(snr_range[0], snr_range[1])
    gmst = U(0.0, 2 * np.pi)
    s_hat = torch.stack([torch.sin(theta) * torch.cos(phi), torch.sin(theta) * torch.sin(phi), torch.cos(theta)], dim=1)
    tau = s_hat @ pos.T
    amp = snr / rho1
    F = torch.empty((nd, n_seg, K), dtype=torch.complex128, device=device)
    for d in range(nd):
        re = torch.randn((n_seg, K), generator=g, dtype=torch.float64, device=device)
        im = torch.randn((n_seg, K), generator=g, dtype=torch.float64, device=device)
        im[:, 0] = 0
        if n % 2 == 0:
            im[:, -1] = 0
        nz = torch.complex(re, im) * sig_t[None, :]
        sig = (amp[:, None] * Hf_t[None, :]) * torch.exp(1j * 2 * np.pi * tau[:, d:d + 1] * kk[None, :] / (dt * n))
        if n % 2 == 0:
            sig[:, -1] = sig[:, -1].real
        F[d] = (nz + sig) * wh_t[None, :]
    return dict(F=F, theta=theta, phi=phi, snr=snr, gmst=gmst)


UNEVEN_BUCKETS = (1024, 2048, 4096, 8192, 16384)
UNEVEN_L = (16, 24, 32, 40, 48)


def make_uneven_batch(positions, n_seg: int, seed: int, fs: float = 4096.0, t_range=(0.25, 4.0), l_choices=UNEVEN_L, n_base=(2, 4),
                      buckets=UNEVEN_BUCKETS, snr_range=(6.0, 30.0), device="cuda"):
    """The uneven workload: per segment a duration log-uniform in
    ``t_range`` at ``fs`` (its time series zero-padded to the next DFT length
    of ``buckets``), an l_max from ``l_choices``, 2-4 of the network's
    baselines, and a chirp injection (SNR uniform in ``snr_range``,
    isotropic direction) in coloured, whitened noise.  Returns a dict:
    ``bucket``, ``n_samples``, ``l_max``, ``mask`` (numpy, per segment) and
    ``spectra``: a packed complex128 tensor, segment after segment, each
    [n_det][bucket_n/2 + 1] (the layout sphrad_uneven_layout reports)."""
    import torch
    rng = rng_for(seed)
    pos = np.asarray(positions, np.float64)
    nd = len(pos)
    nbl = nd * (nd - 1) // 2
    dt = 1.0 / fs
    T = np.exp(rng.uniform(np.log(t_range[0]), np.log(t_range[1]), n_seg))
    nsamp = np.maximum(1, np.round(T * fs).astype(np.int64))
    bucket = np.array([int(np.searchsorted(buckets, x)) for x in nsamp])
    bucket = np.minimum(bucket, len(buckets) - 1)
    lmax = rng.choice(np.asarray(l_choices), n_seg).astype(np.uint32)
    mask = np.zeros(n_seg, np.uint32)
    for s in range(n_seg):
        k = int(rng.integers(n_base[0], n_base[1] + 1))
        for b in rng.choice(nbl, size=min(k, nbl), replace=False):
            mask[s] |= np.uint32(1 << int(b))
    spectra_parts = [None] * n_seg
    for bi, nb in enumerate(buckets):
        idx = np.nonzero(bucket == bi)[0]
        if idx.size == 0:
            continue
        b = make_batch_torch(pos, nb, dt, idx.size, seed * 7919 + bi, device=device, snr_range=snr_range)
        F = b["F"]                                              # [nd][S][K]
        x = torch.fft.irfft(F, n=nb, dim=2)
        keep = torch.as_tensor(nsamp[idx], device=device)[None, :, None]
        t = torch.arange(nb, device=device)[None, None, :]
        x = torch.where(t < keep, x, torch.zeros_like(x))
        F = torch.fft.rfft(x, dim=2)
        for r, s in enumerate(idx):
            spectra_parts[s] = F[:, r, :].reshape(-1)
    spectra = torch.cat(spectra_parts)
    return dict(bucket=bucket, n_samples=nsamp, l_max=lmax, mask=mask, spectra=spectra, buckets=np.asarray(buckets))
