"""Training and evaluation of the learned peak proposal.

Skies come from the library itself: seeded 3-detector injections
(workload.make_batch_torch) integrated by the batched tcgen05 path in the
Earth frame.  Each sky's label is the plain extremizer's answer: the best
pixel of a 64 x 128 grid of the full sky, refined in FP64 by the library's
refinement (BFGS2 by default, sphrad_sky_set_refinement).
A 3-detector sky is exactly symmetric under reflection through the plane of
its baselines (the delays depend on the source only through r_ij . s), so
its maximum is defined up to that mirror image; labels and comparisons use
the image on the positive side of the plane normal.

Everything runs on the GPU through the library's kernels (integration,
grids, refinement, the MLP's forward, backward and Adam); torch provides
device memory, random numbers for the synthetic data and index shuffles.
"""
from __future__ import annotations

import time

import numpy as np

from . import workload as W

N_SAMPLES = 4096
DT = 1.0 / 4096
L_MAX = 32


def plane_normal(positions) -> np.ndarray:
    p = np.asarray(positions, np.float64)
    nrm = np.cross(p[1] - p[0], p[2] - p[0])
    return nrm / np.linalg.norm(nrm)


def unit(theta, phi):
    import torch
    return torch.stack([torch.sin(theta) * torch.cos(phi), torch.sin(theta) * torch.sin(phi), torch.cos(theta)], dim=1)


def canonical(v, nrm):
    """Mirror image of unit vectors v on the non-negative side of nrm."""
    import torch
    n = torch.as_tensor(nrm, dtype=v.dtype, device=v.device)
    d = v @ n
    return v - 2 * torch.clamp(d, max=0)[:, None] * n[None, :]


def angle(u, v):
    import torch
    c = torch.linalg.cross(u, v, dim=1).norm(dim=1)
    return torch.atan2(c, (u * v).sum(dim=1))


class Generator:
    """Skies of the c1-style network in the Earth frame, with labels."""

    def __init__(self, S, positions, precision: str = "bf16x3", chunk: int = 8192, vet_rows: int = 24):
        self.S = S
        self.positions = np.asarray(positions, np.float64)
        self.net = S.Network(self.positions, N_SAMPLES, DT, l_max=L_MAX)
        self.bp = S.BatchPlan(self.net, precision)
        self.grid = S.SkyGrid(L_MAX, 64, 128, kind="cell", fp32=True)
        self.vet = S.SkyGrid(L_MAX, vet_rows, 2 * vet_rows, kind="cell", fp32=True)
        self.nrm = plane_normal(self.positions)
        self.chunk = chunk

    def skies(self, n: int, seed: int):
        b = W.make_batch_torch(self.positions, N_SAMPLES, DT, n, seed)
        return self.bp.integrate(b["F"]), b

    def grid_search(self, sky):
        """The plain extremizer: best pixel of the 64 x 128 grid, refined."""
        th, ph = self.grid.argmax(sky)
        out, st = self.S.refine_peaks(sky, th, ph)
        return out, st

    def dataset(self, prop, n: int, seed: int):
        """(features [n][338], canonical targets [n][3]) on the device."""
        import torch
        feats = torch.empty((n, prop.N_FEATURES), dtype=torch.float32, device="cuda")
        targets = torch.empty((n, 3), dtype=torch.float32, device="cuda")
        for c0 in range(0, n, self.chunk):
            cn = min(self.chunk, n - c0)
            sky, _ = self.skies(cn, seed * 1000003 + c0)
            out, _ = self.grid_search(sky)
            v = canonical(unit(out[:, 0], out[:, 1]), self.nrm)
            targets[c0:c0 + cn] = v.float()
            prop.sky_features(sky, out=feats[c0:c0 + cn])
        return feats, targets

    def close(self):
        for o in (self.vet, self.grid, self.bp, self.net):
            o.close()


def train(prop, feats, targets, epochs: int = 4, batch: int = 4096, lr: float = 2e-3, seed: int = 0, log=None):
    """Adam with a cosine learning-rate decay over all steps; returns the
    per-epoch mean losses."""
    import torch
    n = feats.shape[0]
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    steps = epochs * (n // batch)
    k = 0
    losses = []
    for ep in range(epochs):
        perm = torch.randperm(n, generator=g, device="cuda")
        acc = 0.0
        for b0 in range(0, n - batch + 1, batch):
            idx = perm[b0:b0 + batch]
            rate = lr * 0.5 * (1 + np.cos(np.pi * k / max(1, steps)))
            prop.train_step(feats[idx], targets[idx], rate)
            acc += prop.loss(batch)
            k += 1
        losses.append(acc / max(1, n // batch))
        if log:
            log(f"epoch {ep}: loss {losses[-1]:.3e}")
    return losses


def evaluate(S, gen: Generator, prop, n: int, seed: int, max_move_deg: float = 30.0, basin_deg: float = 6.0, dominance: float = 0.1, reps: int = 3,
             untrained=None):
    """Learned-proposal localisation against the plain extremizer on fresh
    skies: proposal error, fallback rate, agreement within 0.5 degrees
    (modulo the mirror image) and localisations per second of both; and
    every direction's error against the injected source (modulo the mirror
    image), for the trained network's raw proposals, an untrained network's
    (``untrained``, same architecture, when given), the plain extremizer
    and the proposal localisation."""
    import torch
    sky, inj = gen.skies(n, seed)
    torch.cuda.synchronize()
    ref, _ = gen.grid_search(sky)
    feats = prop.sky_features(sky)
    dirs = torch.cat([prop.forward(feats[c0:c0 + prop.max_batch]) for c0 in range(0, n, prop.max_batch)])
    prop.set_mirror(gen.nrm)
    out, st, nfb = prop.localise(gen.vet, gen.grid, sky, max_move_deg, basin_deg, dominance)
    vr = canonical(unit(ref[:, 0], ref[:, 1]), gen.nrm)
    vo = canonical(unit(out[:, 0], out[:, 1]), gen.nrm)
    vp = canonical(dirs.double(), gen.nrm)
    agree = torch.rad2deg(angle(vo, vr))
    perr = torch.rad2deg(angle(vp, vr))
    # timing: both localisers on the same device skies
    st_ = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st_)
    for _ in range(reps):
        gen.grid_search(sky)
    b.record(st_)
    torch.cuda.synchronize()
    t_grid = a.elapsed_time(b) / 1e3 / reps
    t0 = time.perf_counter()
    for _ in range(reps):
        prop.localise(gen.vet, gen.grid, sky, max_move_deg, basin_deg, dominance)
    torch.cuda.synchronize()
    t_prop = (time.perf_counter() - t0) / reps
    q = torch.quantile(perr.float(), torch.tensor([0.5, 0.9, 0.99], device=perr.device)).cpu().numpy()
    # against the injected source: the sky peaks at the source or opposite
    # to it depending on the delay convention; take the sign the plain
    # extremizer's answers agree with
    src = unit(inj["theta"], inj["phi"])
    qs = torch.tensor([0.5, 0.9], device=perr.device)
    e_plus = torch.rad2deg(angle(vr, canonical(src, gen.nrm)))
    e_minus = torch.rad2deg(angle(vr, canonical(-src, gen.nrm)))
    truth = canonical(src if e_plus.median() <= e_minus.median() else -src, gen.nrm)

    def terr(v):
        e = torch.rad2deg(angle(v, truth)).float()
        return [float(x) for x in torch.quantile(e, qs).cpu().numpy()]

    vs_truth = {"grid_search": terr(vr), "proposal_localisation": terr(vo), "trained_proposal_raw": terr(vp)}
    if untrained is not None:
        du = torch.cat([untrained.forward(feats[c0:c0 + untrained.max_batch]) for c0 in range(0, n, untrained.max_batch)])
        vs_truth["untrained_proposal_raw"] = terr(canonical(du.double(), gen.nrm))
    return {
        "err_vs_injection_deg_p50_p90": vs_truth,
        "skies": n,
        "proposal_err_deg_p50_p90_p99": [float(x) for x in q],
        "fallback_rate": nfb / n,
        "agree_within_0.5deg": float((agree <= 0.5).float().mean()),
        "max_disagreement_deg": float(agree.max()),
        "localisations_per_s_proposal": n / t_prop,
        "localisations_per_s_grid_search": n / t_grid,
    }
