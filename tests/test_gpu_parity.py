"""GPU parity of libsphradiometer_b200 against the CPU oracle.

Every test calls the library through its C ABI (ctypes) and compares with
the FP64 oracle on the same seeded inputs.  Tolerances:
* FP64 paths (plans, rotation, the drop-in integrator, the FP64 batch):
  relative L2 <= 1e-10 (rounding differs only in summation order);
* FP32 batch: relative L2 <= 1e-5;
* bf16x3 (tcgen05, hi+lo) batch: relative L2 over the batch <= 1e-5 (the
  accuracy target of the split-precision path), any single sky <= 3e-5;
* bf16x6 (tcgen05, hi+mid+lo) batch: <= 1e-6 for the batch and every sky.
"""
import numpy as np
import pytest

from oracle import oracle as O
from sphradiometer_b200 import workload as W

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def lib():
    import torch
    assert torch.cuda.is_available()
    import sphradiometer_b200 as S
    S.load()
    return S


def c0_positions(seed=1):
    return W.pair_positions(3.0e6 / W.C_LIGHT, W.rng_for(seed))


def c1_positions(seed=2):
    return W.random_positions(3, W.R_EARTH_S, W.rng_for(seed))


# ---------------------------------------------------------------- plans --

def test_rotation_plan_matches_oracle(lib):
    L = lib.load()
    rng = np.random.default_rng(3)
    for l_max in (1, 7, 20, 48):
        g, b, a = rng.uniform(0, 2 * np.pi), np.arccos(rng.uniform(-1, 1)), rng.uniform(0, 2 * np.pi)
        s = L.sh_series_new_zero(l_max, 0)
        R = L.euler_rotation_matrix(g, b, a)
        p = L.sh_series_rotation_plan_new(s, R)
        assert p, lib.last_error()
        got = lib.rotation_plan_flat(p)
        ref = O.rotation_plan(l_max, O.euler_rotation_matrix(g, b, a))
        assert rel_l2(got, ref) < 1e-12
        L.sh_series_rotation_plan_free(p)
        L.sh_series_free(s)


def test_delay_table_matches_oracle(lib):
    pos = c0_positions()
    dt = 1.0 / 2048
    net = lib.Network(pos, 2048, dt, l_max=25)
    d = pos[1] - pos[0]
    ref = O.delay_product(float(np.linalg.norm(d)), dt, 2048, 25)
    got = net.delay_table(0)
    assert got.shape == ref.shape
    assert rel_l2(got, ref) < 1e-10
    net.close()


def test_native_plan_then_set_l_equals_direct_plan(lib):
    """correlator_plan_fd_new + set_l (the reference's route) equals the
    direct correlator_plan_fd_new_l build."""
    pos = W.pair_positions(0.002, W.rng_for(5))
    dt = 1.0 / 1024
    a = lib.Network(pos, 256, dt)            # native l_max
    a.set_l(6)
    b = lib.Network(pos, 256, dt, l_max=6)
    assert a.baseline_l_max(0) == 6 and b.baseline_l_max(0) == 6
    assert np.max(np.abs(a.delay_table(0) - b.delay_table(0))) < 1e-13 * np.max(np.abs(b.delay_table(0)))
    assert np.max(np.abs(a.rotation_flat(0) - b.rotation_flat(0))) < 1e-14
    a.close()
    b.close()


# ------------------------------------------------------------- rotation --

@pytest.mark.parametrize("polar", [True, False])
def test_rotate_matches_oracle(lib, polar):
    L = lib.load()
    rng = np.random.default_rng(11)
    l_max = 20
    n = lib.series_length(l_max, polar)
    a = rng.normal(size=n) + 1j * rng.normal(size=n)
    s = lib.numpy_to_series(a, l_max, polar)
    res = L.sh_series_new(l_max, 0)
    R = L.euler_rotation_matrix(0.3, 1.1, 2.0)
    p = L.sh_series_rotation_plan_new(res, R)
    assert p, lib.last_error()
    assert L.sh_series_rotate(res, s, p), lib.last_error()
    ref = O.rotate(a, l_max, polar, O.rotation_plan(l_max, O.euler_rotation_matrix(0.3, 1.1, 2.0)))
    assert rel_l2(lib.series_to_numpy(res), ref) < 1e-12
    # result == series is refused, as in the reference
    assert not L.sh_series_rotate(res, res, p)
    for x in (s, res):
        L.sh_series_free(x)
    L.sh_series_rotation_plan_free(p)


# ------------------------------------------------------ drop-in integrator --

def test_network_integrate_c0_matches_oracle(lib):
    """c0: two detectors 3000 km apart, 1 s at 2048 Hz, l_max = 25."""
    pos = c0_positions()
    n, dt, L = 2048, 1.0 / 2048, 25
    net = lib.Network(pos, n, dt, l_max=L)
    batch = W.make_batch(pos, n, dt, 1, seed=21)
    F = W.full_from_half(batch["F"][:, 0, :], n)
    got = net.integrate(F)
    b = dict(D=net.delay_table(0), Rot=net.rotation_flat(0))
    ref = O.baseline_integrate_power_fd(F[1], F[0], b["D"], L, b["Rot"])
    assert rel_l2(got, ref) < 1e-10
    # and the oracle's own plan gives the same sky
    ref2 = O.NetworkPlan(pos, n, dt, L).integrate(F)
    assert rel_l2(got, ref2) < 1e-9
    net.close()


def test_baseline_integrate_side_effects(lib):
    """power_1d holds the normalised polar power and fseries_product the
    cross spectrum after the call (correlator.c:681-711)."""
    pos = c0_positions()
    n, dt, L = 512, 1.0 / 512, 8
    net = lib.Network(pos, n, dt, l_max=L)
    rng = np.random.default_rng(4)
    a = rng.normal(size=n) + 1j * rng.normal(size=n)
    b = rng.normal(size=n) + 1j * rng.normal(size=n)
    sky = net.integrate_baseline(0, a, b)
    D = net.delay_table(0)
    p1 = (b * np.conj(a)) @ D / n
    plan = net.plan_fd(0).contents
    assert rel_l2(lib.series_to_numpy(plan.power_1d), p1) < 1e-12
    fsp = np.frombuffer((np.ctypeslib.as_array((__import__("ctypes").c_double * (2 * n)).from_address(plan.fseries_product))),
                        dtype=np.complex128)
    assert rel_l2(fsp, b * np.conj(a)) < 1e-15
    ref = O.rotate(p1, L, True, net.rotation_flat(0))
    assert rel_l2(sky, ref) < 1e-12
    net.close()


def test_mirror_refresh_after_in_place_edit(lib):
    """Writing into delay_product through the library is seen by the next
    integration (fastX.c:485-487 edits plans in place)."""
    L = lib.load()
    pos = c0_positions()
    n, dt = 256, 1.0 / 256
    net = lib.Network(pos, n, dt, l_max=4)
    rng = np.random.default_rng(8)
    F = rng.normal(size=(2, n)) + 1j * rng.normal(size=(2, n))
    first = net.integrate(F)
    dp = net.plan_fd(0).contents.delay_product
    L.sh_series_scale(__import__("ctypes").byref(dp.contents.series[3]), lib._abi.cplx(5.0))
    second = net.integrate(F)
    D = net.delay_table(0)
    ref = O.baseline_integrate_power_fd(F[1], F[0], D, 4, net.rotation_flat(0))
    assert rel_l2(second, ref) < 1e-12
    assert rel_l2(second, first) > 1e-6
    net.close()


# -------------------------------------------------------- batched path --

@pytest.fixture(scope="module")
def c1(lib):
    """c1: 3 detectors on the Earth sphere, 64 x 1 s segments at 4096 Hz,
    l_max = 32."""
    pos = c1_positions()
    n, dt, L = 4096, 1.0 / 4096, 32
    net = lib.Network(pos, n, dt, l_max=L)
    batch = W.make_batch(pos, n, dt, 64, seed=77)
    # oracle skies on the oracle's own delay tables and rotation plans
    oplan = O.NetworkPlan(pos, n, dt, L)
    ref = np.zeros((64, (L + 1) ** 2), np.complex128)
    for s in range(64):
        F = W.full_from_half(batch["F"][:, s, :], n)
        ref[s] = O.rotate_z(oplan.integrate(F), L, False, batch["gmst"][s])
    return dict(net=net, batch=batch, ref=ref, n=n, L=L, oplan=oplan)


def test_c1_delay_tables_and_rotations_match_oracle(lib, c1):
    """The headline plan: 2 R_E-scale baselines at 4096 Hz built directly at
    l_max 32 (native power l_max ~547, 297 taps), against the oracle's own
    correlator_plan_fd_new + set_l restatement (correlator.c:424-519,
    571-591)."""
    net, oplan = c1["net"], c1["oplan"]
    for k, b in enumerate(oplan.baselines):
        assert net.baseline_l_max(k) == b["l"]
        assert rel_l2(net.delay_table(k), b["D"]) < 1e-10, k
        assert rel_l2(net.rotation_flat(k), b["Rot"]) < 1e-12, k


def test_largest_uneven_bucket_delay_table_matches_oracle(lib):
    """The largest bucket of the uneven workload: n = 16384 at 4096 Hz,
    l_max 48, a near-diameter baseline."""
    pos = W.random_positions(4, W.R_EARTH_S, W.rng_for(9))
    n, dt, L = 16384, 1.0 / 4096, 48
    net = lib.Network(pos, n, dt, l_max=L)
    d = pos[3] - pos[0]
    ref = O.delay_product(float(np.linalg.norm(d)), dt, n, L)
    got = net.delay_table(3)
    assert got.shape == ref.shape
    assert rel_l2(got, ref) < 1e-10
    net.close()


# (precision, relative L2 over the whole batch, worst single sky)
TOLS = {"fp64": (1e-10, 1e-10), "fp32": (1e-5, 1e-5), "bf16x3": (1e-5, 3e-5), "bf16x6": (1e-6, 1e-6)}


@pytest.mark.parametrize("prec", ["fp64", "fp32", "bf16x3", "bf16x6"])
def test_batched_matches_oracle(lib, c1, prec):
    import torch
    tol_batch, tol_sky = TOLS[prec]
    bp = lib.BatchPlan(c1["net"], prec)
    F = torch.from_numpy(np.ascontiguousarray(c1["batch"]["F"])).cuda()
    g = torch.from_numpy(c1["batch"]["gmst"]).cuda()
    sky = bp.integrate(F, g).cpu().numpy()
    assert bp.status() == 0
    errs = [rel_l2(sky[s], c1["ref"][s]) for s in range(64)]
    assert rel_l2(sky, c1["ref"]) < tol_batch, (prec, rel_l2(sky, c1["ref"]))
    assert max(errs) < tol_sky, (prec, max(errs))
    # a second call on the re-zeroed workspace gives the same answer
    sky2 = bp.integrate(F, g).cpu().numpy()
    assert rel_l2(sky2, sky) < (1e-12 if prec == "fp64" else 1e-6)
    bp.close()


@pytest.mark.parametrize("prec", ["fp32", "bf16x3", "bf16x6"])
def test_batched_ragged_sizes_and_splits(lib, c1, prec):
    """Segment counts that do not fill a tile, padded rows, every split."""
    import torch
    bp = lib.BatchPlan(c1["net"], prec)
    K = c1["n"] // 2 + 1
    for S in (1, 5, 64):
        Fh = np.zeros((3, S, K + 7), np.complex128)
        Fh[:, :, :K] = c1["batch"]["F"][:, :S, :]
        F = torch.from_numpy(Fh).cuda()
        g = torch.from_numpy(c1["batch"]["gmst"][:S].copy()).cuda()
        for split in (1, 3, 17):
            bp.set_split(S, split)
            sky = bp.integrate(F, g).cpu().numpy()
            assert max(rel_l2(sky[s], c1["ref"][s]) for s in range(S)) < TOLS[prec][1], (S, split)
    assert bp.status() == 0
    bp.close()


@pytest.mark.parametrize("prec,variant", [("bf16x3", 0), ("bf16x3", 1), ("bf16x3", 2), ("bf16x6", 0)])
def test_batched_work_ranges_across_tiles(lib, c1, prec, variant):
    """CTA counts whose (tile, stage) ranges start and end inside tiles:
    one CTA for all 3 tiles (pieces cut at tile boundaries and every 64
    stages), counts that divide nothing, one stage per CTA, and more CTAs
    than stages (idle CTAs), in every pipeline variant (2: X operand in
    tensor memory)."""
    import torch
    bp = lib.BatchPlan(c1["net"], prec)
    S = 300
    idx = np.arange(S) % c1["batch"]["F"].shape[1]
    F = torch.from_numpy(np.ascontiguousarray(c1["batch"]["F"][:, idx, :])).cuda()
    g = torch.from_numpy(c1["batch"]["gmst"][idx].copy()).cuda()
    units = 3 * ((c1["n"] // 2 + 1 + 7) // 8)
    bp.set_pipeline(S, variant)
    assert bp.pipeline(S) == variant
    for ctas in (1, 7, 148, units, units + 29):
        bp.set_ctas(S, ctas)
        assert bp.ctas(S) == ctas
        sky = bp.integrate(F, g).cpu().numpy()
        errs = [rel_l2(sky[s], c1["ref"][idx[s]]) for s in range(S)]
        assert max(errs) < TOLS[prec][1], (ctas, max(errs))
    bp.set_ctas(S, 0)
    bp.set_pipeline(S, -1)
    assert bp.status() == 0
    bp.close()


def test_batched_host_entry_point(lib, c1):
    bp = lib.BatchPlan(c1["net"], "bf16x3")
    Fh = np.ascontiguousarray(c1["batch"]["F"])
    sky = bp.integrate_host(Fh, c1["batch"]["gmst"])
    assert rel_l2(sky, c1["ref"]) < 1e-5
    bp.close()


def test_batched_host_entry_point_in_chunks(lib, c1):
    """1573 segments go through the host path in three chunks on two
    streams (525, 525, 523); twice, so the second call reuses the scratch
    the first left behind."""
    bp = lib.BatchPlan(c1["net"], "bf16x3")
    S = 1573
    idx = np.arange(S) % c1["batch"]["F"].shape[1]
    Fh = np.ascontiguousarray(c1["batch"]["F"][:, idx, :])
    g = np.ascontiguousarray(c1["batch"]["gmst"][idx])
    for _ in range(2):
        sky = bp.integrate_host(Fh, g)
        errs = [rel_l2(sky[s], c1["ref"][idx[s]]) for s in range(S)]
        assert max(errs) < 1e-5
    assert bp.status() == 0
    bp.close()


def test_batched_autotune_keeps_results(lib, c1):
    import torch
    bp = lib.BatchPlan(c1["net"], "bf16x3")
    F = torch.from_numpy(np.ascontiguousarray(c1["batch"]["F"])).cuda()
    k = bp.autotune(F)
    assert k >= 1 and bp.split(64) == k
    g = torch.from_numpy(c1["batch"]["gmst"]).cuda()
    sky = bp.integrate(F, g).cpu().numpy()
    assert rel_l2(sky, c1["ref"]) < 1e-5
    bp.close()
