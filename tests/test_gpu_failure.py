"""Failure detection on the GPU, without faulting it.

* Device-side: every mbarrier wait of the contraction kernels is bounded
  (the bound is a launch argument, sphrad_batch_set_wait_limit).  A test
  hook makes the spectrum producer of the first CTA withhold one stage's
  load, so a consumer's wait on it runs out after the short bound: the call
  returns, sphrad_batch_status reports the wait's code (and clears it), and
  the next call, hook off, is correct.
* Host-side: allocation failures injected into the library's allocations
  (device and host) make correlator_network_plan_fd_new return NULL without
  aborting, as the reference's constructors do (correlator.c:387-399); once
  the injection is spent the same call builds a plan that integrates
  correctly.
"""
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


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


def test_withheld_stage_times_out_and_plan_recovers(S):
    import torch
    pos = W.random_positions(3, W.R_EARTH_S, W.rng_for(2))
    n, dt, L = 4096, 1.0 / 4096, 32
    net = S.Network(pos, n, dt, l_max=L)
    batch = W.make_batch(pos, n, dt, 16, seed=5)
    F = torch.from_numpy(np.ascontiguousarray(batch["F"])).cuda()
    g = torch.from_numpy(batch["gmst"]).cuda()
    bp = S.BatchPlan(net, "bf16x3")
    lib = S.load()
    good = bp.integrate(F, g).cpu().numpy()
    assert bp.status() == 0
    # ~10 ms at the B200's clock; the withheld stage's wait runs out
    assert lib.sphrad_batch_set_wait_limit(bp._p, 20_000_000) == 0
    assert lib.sphrad_batch_test_withhold_stage(bp._p, 1) == 0
    bp.integrate(F, g)
    torch.cuda.synchronize()
    code = bp.status()
    assert code > 0, code
    assert bp.status() == 0  # reading cleared it
    # hook off, default bound: the plan and the context are usable
    assert lib.sphrad_batch_test_withhold_stage(bp._p, -1) == 0
    assert lib.sphrad_batch_set_wait_limit(bp._p, 0) == 0
    again = bp.integrate(F, g).cpu().numpy()
    assert bp.status() == 0
    assert rel(again, good) < 1e-6
    # and against the oracle
    op = O.NetworkPlan(pos, n, dt, L)
    for s in range(4):
        Fs = W.full_from_half(batch["F"][:, s, :], n)
        ref = O.rotate_z(op.integrate(Fs), L, False, batch["gmst"][s])
        assert rel(again[s], ref) < 3e-5
    bp.close()
    net.close()


def test_injected_allocation_failures_make_plan_construction_return_null(S):
    pos = W.random_positions(3, 0.02, W.rng_for(4))
    n, dt, L = 512, 1.0 / 512, 8
    lib = S.load()
    failed = 0
    net = None
    for k in range(1, 400):
        lib.sphrad_b200_inject_allocation_failure(k)
        try:
            net = S.Network(pos, n, dt, l_max=L)
        except S.SphradError:
            failed += 1
            continue
        finally:
            lib.sphrad_b200_inject_allocation_failure(0)
        break
    assert net is not None and failed >= 3, failed
    rng = np.random.default_rng(3)
    Fs = rng.normal(size=(3, n)) + 1j * rng.normal(size=(3, n))
    ref = O.NetworkPlan(pos, n, dt, L).integrate(Fs)
    assert rel(net.integrate(Fs), ref) < 1e-10
    net.close()
