"""GPU parity of the time-series-to-spectrum step (the FFTW step ahead of
the correlator, correlator.c:216-231, and the caller's whitening,
sphradiometer_demo.c:456-460) against numpy's FFT, and of the time-series
entry point of the batched integrator against the spectra path and the
oracle.

Tolerances: the FP64 FFT agrees with numpy's to 1e-13 of the largest bin
(both are O(log n) rounding, ~1e-15); skies from time series match skies
from numpy spectra to 1e-12 on the FP64 path, and the oracle to the
bf16x3 bounds of the spectra path (1e-5 over the batch, 3e-5 per sky).
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from sphradiometer_b200 import workload as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def S():
    import torch
    assert torch.cuda.is_available()
    import sphradiometer_b200 as S
    S.load()
    return S


def maxrel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / np.max(np.abs(b)))


@pytest.mark.parametrize("n", [8, 16, 64, 1024, 2048, 4096, 8192, 16384])
def test_transform_matches_numpy(S, n):
    import torch
    rng = np.random.default_rng(n)
    x = rng.normal(size=(3, 5, n))
    p = S.FseriesPlan(n)
    got = p.transform(torch.from_numpy(x).cuda()).cpu().numpy()
    assert got.shape == (3, 5, n // 2 + 1)
    assert maxrel(got, np.fft.rfft(x, axis=-1)) < 1e-13
    p.close()


def test_whitening_and_strided_rows(S):
    """One-sided PSD whitening (bins outside the band zeroed) on rows with
    padded strides, through the C ABI."""
    import torch
    L = S.load()
    n, dt, rows = 4096, 1.0 / 4096, 7
    psd = W.psd(np.arange(n // 2 + 1) / (n * dt))
    wh = np.where(psd > 0, 1.0 / np.sqrt(np.where(psd > 0, psd, 1.0)), 0.0)
    rng = np.random.default_rng(3)
    ldt, ldf = n + 6, n // 2 + 1 + 3
    x = np.zeros((rows, ldt))
    x[:, :n] = rng.normal(size=(rows, n))
    p = S.FseriesPlan(n, psd)
    xd = torch.from_numpy(x).cuda()
    out = torch.zeros((rows, ldf), dtype=torch.complex128, device="cuda")
    assert L.sphrad_tseries_to_fseries(p._p, xd.data_ptr(), rows, ldt, out.data_ptr(), ldf, None) == 0
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    ref = np.fft.rfft(x[:, :n], axis=-1) * wh
    assert maxrel(got[:, : n // 2 + 1], ref) < 1e-13
    assert np.all(got[:, n // 2 + 1:] == 0)
    p.close()


def test_rejects_bad_sizes_and_layouts(S):
    import torch
    L = S.load()
    for n in (0, 4, 100, 3000, 32768):
        assert not L.sphrad_fseries_plan_new(n, None)
    p = S.FseriesPlan(64)
    x = torch.zeros((2, 70), dtype=torch.float64, device="cuda")
    out = torch.zeros((2, 40), dtype=torch.complex128, device="cuda")
    assert L.sphrad_tseries_to_fseries(p._p, x.data_ptr(), 2, 65, out.data_ptr(), 40, None) < 0   # odd row stride
    assert L.sphrad_tseries_to_fseries(p._p, x.data_ptr(), 2, 62, out.data_ptr(), 40, None) < 0   # stride below n
    assert L.sphrad_tseries_to_fseries(p._p, x.data_ptr(), 2, 70, out.data_ptr(), 32, None) < 0   # too few bins
    assert L.sphrad_tseries_to_fseries(p._p, x.data_ptr() + 8, 1, 64, out.data_ptr(), 40, None) < 0  # misaligned
    p.close()


@pytest.mark.parametrize("whiten", [False, True])
def test_host_drop_in_full_spectrum(S, whiten):
    """sphrad_tseries_to_fseries_host: the full n-bin spectrum with the
    upper half conj-mirrored, as correlator_tseries_to_fseries returns."""
    n, dt = 2048, 1.0 / 2048
    rng = np.random.default_rng(5)
    x = rng.normal(size=n)
    psd = W.psd(np.arange(n // 2 + 1) / (n * dt)) if whiten else None
    p = S.FseriesPlan(n, psd)
    got = p.transform_host(x)
    ref = np.fft.fft(x)
    if whiten:
        wh = np.where(psd > 0, 1.0 / np.sqrt(np.where(psd > 0, psd, 1.0)), 0.0)
        ref = ref * np.concatenate([wh, wh[1:-1][::-1]])
    assert maxrel(got, ref) < 1e-13
    p.close()


@pytest.fixture(scope="module")
def c1t(S):
    pos = W.random_positions(3, W.R_EARTH_S, W.rng_for(2))
    n, dt, L = 4096, 1.0 / 4096, 32
    net = S.Network(pos, n, dt, l_max=L)
    b = W.make_tseries_batch(pos, n, dt, 40, seed=91)
    return dict(net=net, b=b, n=n, L=L, pos=pos)


def test_integrate_tseries_fp64_matches_spectra_path(S, c1t):
    import torch
    b = c1t["b"]
    bp = S.BatchPlan(c1t["net"], "fp64")
    fp = S.FseriesPlan(c1t["n"], b["psd"])
    x = torch.from_numpy(b["x"]).cuda()
    g = torch.from_numpy(b["gmst"].copy()).cuda()
    got = bp.integrate_tseries(fp, x, g).cpu().numpy()
    ref = bp.integrate(torch.from_numpy(np.ascontiguousarray(b["F"])).cuda(), g).cpu().numpy()
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-12
    fp.close()
    bp.close()


def test_integrate_tseries_bf16x3_matches_oracle(S, c1t):
    import torch
    b, net, n, L = c1t["b"], c1t["net"], c1t["n"], c1t["L"]
    bp = S.BatchPlan(net, "bf16x3")
    fp = S.FseriesPlan(n, b["psd"])
    x = torch.from_numpy(b["x"]).cuda()
    g = torch.from_numpy(b["gmst"].copy()).cuda()
    got = bp.integrate_tseries(fp, x, g).cpu().numpy()
    # oracle skies from numpy spectra, on the oracle's own plan
    oplan = O.NetworkPlan(c1t["pos"], n, 1.0 / n, L)
    segs = range(0, 40, 4)
    errs, num, den = [], 0.0, 0.0
    for s in segs:
        F = W.full_from_half(b["F"][:, s, :], n)
        ref = O.rotate_z(oplan.integrate(F), L, False, b["gmst"][s])
        errs.append(np.linalg.norm(got[s] - ref) / np.linalg.norm(ref))
        num += np.linalg.norm(got[s] - ref) ** 2
        den += np.linalg.norm(ref) ** 2
    assert np.sqrt(num / den) < 1e-5 and max(errs) < 3e-5, (np.sqrt(num / den), max(errs))
    assert bp.status() == 0
    fp.close()
    bp.close()
