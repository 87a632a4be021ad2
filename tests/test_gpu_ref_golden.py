"""GPU library against the reference itself.

tests/golden/ref_c0.npz and ref_c1.npz hold outputs of the reference's own
C code (compiled unmodified against the project's FFTW/GSL/LAL stand-ins;
tests/golden/make_ref_golden.py).  Here the GPU library, through its C ABI,
is held to them directly:

* delay tables built on the GPU in FP64 (correlator_plan_fd_new + set_l,
  c1's native plan l_max ~547): every 64th bin row and two projections
  over all bins, relative L2 <= 1e-10; rotation plans <= 1e-12;
* the drop-in correlator_network_integrate_power_fd: <= 1e-10;
* the batched path with the GMST rotation fused: FP64 <= 1e-10, FP32
  <= 1e-5, bf16x3 <= 1e-5 over the batch and 3e-5 per sky (the
  split-precision bound); c0 has a single baseline, so the epilogues' lanes
  of absent baselines are exercised.

And the reference's own test programs test/product_validate.c and
test/rotation_validate.c, compiled unmodified against this repository's
include/sphradiometer headers and linked with libsphradiometer_b200.so
(oracle/Makefile "ref" target), run to completion: their assert()s check
products against pointwise products (<= 1e-13 (l1^2 + l2^2)), rotation
matrices, Wigner-D structure and rotated impulses.
"""
import os
import subprocess

import numpy as np
import pytest

from sphradiometer_b200 import workload as W

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
REF_BIN = os.path.join(ROOT, "oracle", "_ref")


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def S():
    import torch
    assert torch.cuda.is_available()
    import sphradiometer_b200 as S
    S.load()
    return S


def golden(name):
    return np.load(os.path.join(GOLDEN, f"ref_{name}.npz"))


def projection_vectors(seed: int, n: int):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(2, n)) + 1j * rng.normal(size=(2, n))


@pytest.mark.parametrize("name", ["c0", "c1"])
def test_gpu_plans_match_reference(S, name):
    g = golden(name)
    n, dt, L = int(g["n"]), float(g["dt"]), int(g["l_max"])
    net = S.Network(g["positions"], n, dt, l_max=L)
    rvec = projection_vectors(int(g["rvec_seed"]), n)
    for k in range(len(g["baselines"])):
        assert net.baseline_l_max(k) == int(g["baselines"][k][4])
        D = net.delay_table(k)
        assert rel(D[::int(g["row_step"])], g[f"D_rows_{k}"]) < 1e-10, k
        assert rel(rvec @ D, g[f"D_proj_{k}"]) < 1e-10, k
        assert rel(net.rotation_flat(k)[::int(g["rot_step"])], g[f"rot_{k}"]) < 1e-12, k
    net.close()


@pytest.mark.parametrize("name", ["c0", "c1"])
def test_gpu_skies_match_reference(S, name):
    import torch
    g = golden(name)
    n, dt, L = int(g["n"]), float(g["dt"]), int(g["l_max"])
    net = S.Network(g["positions"], n, dt, l_max=L)
    nsk = len(g["skies"])
    batch = W.make_batch(g["positions"], n, dt, nsk, seed=int(g["batch_seed"]))
    for s in range(nsk):
        F = W.full_from_half(batch["F"][:, s, :], n)
        assert rel(net.integrate(F), g["skies"][s]) < 1e-10, s
    Fd = torch.from_numpy(np.ascontiguousarray(batch["F"])).cuda()
    gd = torch.from_numpy(np.ascontiguousarray(batch["gmst"])).cuda()
    ref = g["skies_gmst"]
    for prec, tb, ts in (("fp64", 1e-10, 1e-10), ("fp32", 1e-5, 1e-5), ("bf16x3", 1e-5, 3e-5)):
        bp = S.BatchPlan(net, prec)
        sky = bp.integrate(Fd, gd).cpu().numpy()
        assert bp.status() == 0
        assert rel(sky, ref) < tb, prec
        assert max(rel(sky[s], ref[s]) for s in range(nsk)) < ts, prec
        bp.close()
    net.close()


@pytest.mark.parametrize("prog", ["product_validate", "rotation_validate"])
def test_reference_test_programs_against_library(prog):
    exe = os.path.join(REF_BIN, prog)
    if not os.path.exists(exe):
        pytest.skip(f"{prog} not built (make -C oracle ref needs the reference checkout)")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (r.returncode, r.stdout[-2000:], r.stderr[-2000:])
