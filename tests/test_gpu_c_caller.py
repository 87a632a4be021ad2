"""The drop-in FD path through a compiled C caller.

tests/c/fd_caller.c builds instruments, network baselines and a network
plan and calls correlator_network_integrate_power_fd once per segment, as
the reference's programs do, compiled against include/sphradiometer and
linked with libsphradiometer_b200.so (no Python between the caller and the
library).  Its skies are held to the reference's own outputs on the same
inputs (tests/golden/ref_c0.npz, ref_c1.npz: the reference's C, compiled
from its sources against the project's stand-ins) at relative L2 <= 1e-10.
"""
import os
import struct
import subprocess

import numpy as np
import pytest

from sphradiometer_b200 import workload as W
from test_abi_cpu import c_caller

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


@pytest.mark.parametrize("name", ["c0", "c1"])
def test_c_caller_matches_reference(tmp_path, name):
    g = np.load(os.path.join(ROOT, "tests", "golden", f"ref_{name}.npz"))
    pos = np.asarray(g["positions"], np.float64)
    n, dt, L = int(g["n"]), float(g["dt"]), int(g["l_max"])
    nsk = len(g["skies"])
    batch = W.make_batch(pos, n, dt, nsk, seed=int(g["batch_seed"]))
    inp = tmp_path / "in.bin"
    with open(inp, "wb") as f:
        f.write(struct.pack("<iiiid", len(pos), n, L, nsk, dt))
        f.write(np.ascontiguousarray(pos).tobytes())
        for s in range(nsk):
            for d in range(len(pos)):
                f.write(np.ascontiguousarray(W.full_from_half(batch["F"][d, s, :], n), np.complex128).tobytes())
    exe = c_caller(tmp_path / "fd_caller")
    out = tmp_path / "out.bin"
    r = subprocess.run([exe, str(inp), str(out)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (r.returncode, r.stderr[-2000:])
    skies = np.fromfile(out, np.complex128).reshape(nsk, (L + 1) ** 2)
    for s in range(nsk):
        assert rel(skies[s], g["skies"][s]) < 1e-10, s
