"""GPU parity of uneven batches (segments of different DFT lengths, l_max
and baseline subsets of a 4-detector network in one call) against the
FP64 oracle, per segment: the mean over the segment's own baselines of the
oracle's correlator_baseline_integrate_power_fd at the segment's padded
DFT length (on the oracle's own delay tables and rotation plans),
truncated to the segment's l_max.

Tolerances: bf16x3 contraction, relative L2 <= 1e-5 over the batch and
3e-5 per sky; FP64 contraction 1e-10.  Graph replay and direct launches
differ only in the order of the FP32 atomic split-K sums (<= 1e-6 of the
largest coefficient), other split-K factors, and the persistent launch
against per-job launches, also in how the FP32 sums are grouped (<= 4e-6).
"""
import numpy as np
import pytest

from oracle import oracle as O
from sphradiometer_b200 import workload as W

pytestmark = pytest.mark.gpu

DT = 1.0 / 4096


@pytest.fixture(scope="module")
def S():
    import torch
    assert torch.cuda.is_available()
    import sphradiometer_b200 as S
    S.load()
    return S


def pairs(nd):
    return [(i, j) for i in range(1, nd) for j in range(i)]


def oracle_skies(S, pos, batch, plan, Lplan):
    """Per-segment oracle skies (numpy), in the plan's packed order."""
    nd = len(pos)
    pr = pairs(nd)
    sp = batch["spectra"].cpu().numpy()
    tables = {}
    out = []
    for s in range(len(batch["bucket"])):
        nb = int(batch["buckets"][batch["bucket"][s]])
        if nb not in tables:
            # the oracle's own delay tables and rotation plans, in the same
            # baseline order (i > j, i ascending)
            op = O.NetworkPlan(pos, nb, DT, Lplan)
            tables[nb] = [(b["D"], b["Rot"], b["l"]) for b in op.baselines]
        Ku = nb // 2 + 1
        half = sp[plan.in_offset[s]:plan.in_offset[s] + nd * Ku].reshape(nd, Ku)
        F = W.full_from_half(half, nb)
        ks = [k for k in range(len(pr)) if (int(batch["mask"][s]) >> k) & 1]
        sky = np.zeros(O.length(Lplan, False), np.complex128)
        for k in ks:
            i, j = pr[k]
            D, R, lb = tables[nb][k]
            p = O.baseline_integrate_power_fd(F[i], F[j], D, lb, R)
            sky += O.assign(p, lb, False, Lplan, False) / len(ks)
        out.append(O.assign(sky, Lplan, False, int(batch["l_max"][s]), False))
    return out


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


@pytest.mark.parametrize("prec,tol_batch,tol_sky", [("bf16x3", 1e-5, 3e-5), ("fp64", 1e-10, 1e-10)])
def test_uneven_batch_matches_oracle(S, prec, tol_batch, tol_sky):
    pos = W.random_positions(4, W.R_EARTH_S, W.rng_for(9))
    batch = W.make_uneven_batch(pos, 48, seed=3, t_range=(0.25, 1.0), l_choices=(16, 24, 32), buckets=(1024, 2048, 4096))
    plan = S.UnevenPlan(pos, DT, batch["buckets"], 32, precision=prec)
    plan.set_segments(batch["bucket"], batch["mask"], batch["l_max"])
    assert plan.jobs() >= 2
    got = plan.unpack(plan.integrate(batch["spectra"]))
    ref = oracle_skies(S, pos, batch, plan, 32)
    errs = [rel(g, r) for g, r in zip(got, ref)]
    num = np.sqrt(sum(np.linalg.norm(g - r) ** 2 for g, r in zip(got, ref)))
    den = np.sqrt(sum(np.linalg.norm(r) ** 2 for r in ref))
    assert num / den < tol_batch, num / den
    assert max(errs) < tol_sky, max(errs)
    plan.close()


def test_uneven_graph_split_and_three_detectors(S):
    import torch
    pos = W.random_positions(3, W.R_EARTH_S, W.rng_for(2))
    batch = W.make_uneven_batch(pos, 300, seed=5, t_range=(0.25, 2.0), l_choices=(16, 32), n_base=(1, 3), buckets=(1024, 2048, 4096, 8192))
    plan = S.UnevenPlan(pos, DT, batch["buckets"], 32)
    plan.set_segments(batch["bucket"], batch["mask"], batch["l_max"])
    assert plan.jobs() <= 4  # one sub-network: one job per bucket
    plan.set_persistent(False)
    plan.use_graph(False)
    direct = plan.integrate(batch["spectra"]).clone()
    plan.use_graph(True)
    g1 = plan.integrate(batch["spectra"]).clone()
    g2 = plan.integrate(batch["spectra"]).clone()
    # split-K partial sums meet in FP32 atomics, whose order varies run to run
    scale = float(direct.abs().max())
    assert float((direct - g1).abs().max()) < 1e-6 * scale and float((g1 - g2).abs().max()) < 1e-6 * scale
    plan.autotune(batch["spectra"])
    tuned = plan.integrate(batch["spectra"])
    plan.set_split(1)
    fixed = plan.integrate(batch["spectra"])
    assert float((tuned - fixed).abs().max() / fixed.abs().max()) < 4e-6
    ref = oracle_skies(S, pos, batch, plan, 32)
    got = plan.unpack(tuned)
    assert max(rel(g, r) for g, r in zip(got, ref)) < 3e-5
    plan.close()


def test_uneven_persistent_launch(S):
    """Every job's contraction in one persistent launch (tcgen05
    precisions, the default): one contraction plus one epilogue per job per
    call; the same skies as one launch per job up to the grouping of the
    FP32 sums, and the oracle's within the bf16x3 bounds."""
    pos = W.random_positions(4, W.R_EARTH_S, W.rng_for(9))
    batch = W.make_uneven_batch(pos, 96, seed=21, t_range=(0.25, 2.0), l_choices=(16, 32, 48), buckets=(1024, 2048, 4096, 8192))
    plan = S.UnevenPlan(pos, DT, batch["buckets"], 48)
    plan.set_segments(batch["bucket"], batch["mask"], batch["l_max"])
    assert plan.persistent() and 2 <= plan.jobs() <= 24
    pers = plan.integrate(batch["spectra"]).clone()
    assert plan.kernels_per_call() == 1 + plan.jobs()
    plan.set_persistent(False)
    per_job = plan.integrate(batch["spectra"]).clone()
    assert not plan.persistent()
    plan.set_persistent(True)
    again = plan.integrate(batch["spectra"]).clone()
    scale = float(per_job.abs().max())
    assert float((pers - per_job).abs().max()) < 4e-6 * scale
    assert float((pers - again).abs().max()) < 1e-6 * scale
    got = plan.unpack(pers)
    ref = oracle_skies(S, pos, batch, plan, 48)
    num = np.sqrt(sum(np.linalg.norm(g - r) ** 2 for g, r in zip(got, ref)))
    den = np.sqrt(sum(np.linalg.norm(r) ** 2 for r in ref))
    assert num / den < 1e-5, num / den
    assert max(rel(g, r) for g, r in zip(got, ref)) < 3e-5
    plan.close()


def test_uneven_rejects_empty_segments(S):
    pos = W.random_positions(4, W.R_EARTH_S, W.rng_for(9))
    plan = S.UnevenPlan(pos, DT, [1024], 16)
    with pytest.raises(S.SphradError):
        plan.set_segments([0, 0], [3, 0], [16, 16])
    with pytest.raises(S.SphradError):
        plan.set_segments([0], [3], [20])  # l_max above the plan's
    plan.close()
