"""Failure detection on the host (no GPU): allocation failures injected
into the library's own allocations (sphrad_b200_inject_allocation_failure)
must make the host-only constructors of the C ABI return NULL -- the
reference's contract (e.g. correlator.c:387-399: free what was built,
return NULL, never abort) -- and leave the library usable."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def L():
    import sphradiometer_b200 as S
    return S.load()


def build_network(L, pos):
    """instrument_new + instrument_array_append for each detector, then
    correlator_network_baselines_new; returns the objects made so far and
    whether every step succeeded."""
    made = []
    arr = L.instrument_array_new(0)
    if not arr:
        return made, False
    made.append(("array", arr))
    for p in pos:
        inst = L.instrument_new(float(p[0]), float(p[1]), float(p[2]), None)
        if not inst:
            return made, False
        if not L.instrument_array_append(arr, inst):
            return made, False
    net = L.correlator_network_baselines_new(arr)
    if not net:
        return made, False
    made.append(("baselines", net))
    return made, True


def free_all(L, made):
    for kind, p in reversed(made):
        if kind == "baselines":
            L.correlator_network_baselines_free(p)
        else:
            L.instrument_array_free(p)


def test_injected_host_allocation_failures_return_null(L):
    pos = np.array([[0.01, 0.0, 0.0], [0.0, 0.012, 0.0], [0.0, 0.0, 0.009]])
    failures = 0
    for k in range(1, 200):
        assert L.sphrad_b200_inject_allocation_failure(k) == 0
        made, ok = build_network(L, pos)
        free_all(L, made)
        if ok:
            break
        failures += 1
    assert L.sphrad_b200_inject_allocation_failure(0) == 0
    assert failures >= 5, failures   # every allocation of the chain was hit once
    made, ok = build_network(L, pos)
    assert ok
    assert made[-1][1].contents.n_baselines == 3  # the object is usable
    free_all(L, made)


def test_injected_failure_in_series_constructors(L):
    for k in (1, 2):
        L.sphrad_b200_inject_allocation_failure(k)
        assert not L.sh_series_new(8, 0)
    L.sphrad_b200_inject_allocation_failure(0)
    s = L.sh_series_new(8, 0)
    assert s
    L.sh_series_free(s)
    L.sphrad_b200_inject_allocation_failure(1)
    assert not L.sh_series_array_new(16, 4, 1)
    L.sphrad_b200_inject_allocation_failure(0)
