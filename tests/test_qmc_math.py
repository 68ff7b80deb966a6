"""CPU checks of the NOCI-QMC arithmetic the GPU kernels use (noci-rs_b200/csrc/qmc_math.cuh,
compiled for the host by tests/cpu_mirror): the Philox4x32-10 generator against the
known-answer vectors published with the algorithm, FRI rounding, the uniform generator and the
propagator shifts (src/stochastic/state.rs:80-162, metric.rs:675-699)."""
import ctypes

import numpy as np
import pytest

import mirror as MR


@pytest.mark.parametrize("ctr,key,expect", [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
])
def test_philox4x32_10_known_answers(ctr, key, expect):
    c = np.array(ctr, np.uint32)
    out = np.zeros(4, np.uint32)
    MR.lib().mir_philox(MR.p(c, ctypes.c_uint32), key[0], key[1], MR.p(out, ctypes.c_uint32))
    assert tuple(int(v) for v in out) == expect


def test_uniforms_are_uniform_and_distinct_per_purpose():
    L = MR.lib()
    out = np.zeros(2)
    u = []
    for i in range(20000):
        L.mir_uniform2(7, 3, i, 2, MR.p(out, ctypes.c_double))
        u.extend(out)
    u = np.array(u)
    assert 0.0 <= u.min() and u.max() < 1.0
    hist, _ = np.histogram(u, bins=20, range=(0, 1))
    assert np.all(np.abs(hist - u.size / 20) < 5 * np.sqrt(u.size / 20))
    L.mir_uniform2(7, 3, 5, 1, MR.p(out, ctypes.c_double))
    a = out.copy()
    L.mir_uniform2(7, 3, 5, 3, MR.p(out, ctypes.c_double))
    assert not np.array_equal(a, out)


@pytest.mark.parametrize("x", [-0.3, 0.1, 0.999, 2.0, -5.0, 0.0])
def test_fri_is_unbiased(x):
    L = MR.lib()
    us = (np.arange(100000) + 0.5) / 100000
    vals = np.array([L.mir_fri(x, 1.0, float(u)) for u in us])
    assert abs(vals.mean() - x) < 2e-5
    assert set(np.unique(vals)) <= ({x} if abs(x) >= 1 or x == 0 else {0.0, np.copysign(1.0, x)})
    assert L.mir_fri(0.3, 0.0, 0.9) == 0.3          # cutoff 0: unchanged


def test_uniform_child_excludes_parent_and_is_flat():
    L = MR.lib()
    n = 7
    for g in range(n):
        us = (np.arange(6000) + 0.5) / 6000
        ch = np.array([L.mir_uniform_child(g, n, float(u)) for u in us])
        assert g not in ch and ch.min() >= 0 and ch.max() < n
        counts = np.bincount(ch, minlength=n)
        assert np.all(counts[np.arange(n) != g] == 1000)
    assert L.mir_attempts(0.0) == 0 and L.mir_attempts(0.2) == 1 and L.mir_attempts(-3.5) == 4


def test_propagator_shifts():
    L = MR.lib()
    dt, es, h, s, n = 0.01, -1.2, -0.7, 0.9, 3.0
    for prop, ident in ((0, 0.0), (1, es), (2, es), (3, 0.0), (4, 0.0)):
        assert L.mir_diagonal_change(prop, dt, es, h, s, n) == pytest.approx(-dt * (h - es * s - ident) * n)
