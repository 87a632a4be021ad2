"""Writes tests/golden/ref_c0.npz and ref_c1.npz: outputs of the reference
itself (cannon-zz/sphradiometer's own C, compiled unmodified against the
project's FFTW/GSL/LAL stand-ins by ``make -C oracle ref``) on the c0 and c1
networks, so that tests on machines without the reference checkout can pin
the oracle and the GPU library to it.

    python tests/golden/make_ref_golden.py            # needs oracle/_ref

Per network (reference calls in brackets):
  * the detector positions, n, dt, l_max and each baseline's (i, j, theta,
    phi, l_max) [correlator_network_plan_fd_new + _set_l];
  * each baseline's delay table [plan->delay_product]: every 64th bin row,
    plus two seeded complex projections over all n bins (r @ D), so a test
    checks the whole table through a few numbers;
  * each baseline's rotation plan, every 31st element of the flattened
    matrices [plan->rotation_plan];
  * skies of 4 seeded segments from sphradiometer_b200.workload.make_batch
    [correlator_network_integrate_power_fd], with checksums of their input
    spectra so a test can confirm it regenerated the same inputs;
  * the skies rotated by each segment's GMST [sh_series_rotate_z].

c0: 2 detectors 3000 km apart, 2048 Hz, n = 2048, l_max 25.
c1: 3 detectors on the Earth sphere, 4096 Hz, n = 4096, l_max 32 (the
reference's native plan here has power l_max ~547: about 2 minutes).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref as R  # noqa: E402
from sphradiometer_b200 import workload as W  # noqa: E402

CASES = {
    "c0": dict(pos=lambda: W.pair_positions(3.0e6 / W.C_LIGHT, W.rng_for(1)), n=2048, dt=1.0 / 2048, L=25, seed=21),
    "c1": dict(pos=lambda: W.random_positions(3, W.R_EARTH_S, W.rng_for(2)), n=4096, dt=1.0 / 4096, L=32, seed=77),
}
N_SKIES = 4
ROW_STEP = 64
ROT_STEP = 31


def projection_vectors(n: int):
    rng = np.random.default_rng(12345 + n)
    return rng.normal(size=(2, n)) + 1j * rng.normal(size=(2, n))


def spectra_checksum(F):
    return np.array([F.sum(), (np.abs(F) ** 2).sum()], dtype=np.complex128)


def make(name: str):
    c = CASES[name]
    pos = c["pos"]()
    n, dt, L = c["n"], c["dt"], c["L"]
    net = R.Network(pos, n, dt, L)
    rvec = projection_vectors(n)
    out = dict(positions=pos, n=n, dt=dt, l_max=L, row_step=ROW_STEP, rot_step=ROT_STEP, rvec_seed=12345 + n, batch_seed=c["seed"])
    base = []
    for k in range(net.n_baselines):
        ia, ib, th, ph = net.baseline(k)
        lb = net.baseline_l_max(k)
        base.append([ia, ib, th, ph, lb])
        D = net.delay_table(k)
        out[f"D_rows_{k}"] = D[::ROW_STEP]
        out[f"D_proj_{k}"] = rvec @ D
        out[f"rot_{k}"] = net.rotation_flat(k)[::ROT_STEP]
    out["baselines"] = np.array(base)
    batch = W.make_batch(pos, n, dt, N_SKIES, seed=c["seed"])
    skies, rotated, sums = [], [], []
    for s in range(N_SKIES):
        F = W.full_from_half(batch["F"][:, s, :], n)
        sky = net.integrate(F, L)
        skies.append(sky)
        rotated.append(R.rotate_z(sky, L, False, float(batch["gmst"][s])))
        sums.append(spectra_checksum(F))
    out["skies"] = np.array(skies)
    out["skies_gmst"] = np.array(rotated)
    out["gmst"] = np.asarray(batch["gmst"][:N_SKIES])
    out["spectra_checksums"] = np.array(sums)
    net.close()
    np.savez_compressed(os.path.join(HERE, f"ref_{name}.npz"), **out)
    print(f"wrote ref_{name}.npz")


if __name__ == "__main__":
    if not R.build(quiet=False):
        sys.exit("oracle/_ref is not built and the reference checkout is absent")
    for name in (sys.argv[1:] or list(CASES)):
        make(name)
