"""The oracle's per-pixel operators against golden vectors of the reference's own CUDA kernels.

tests/golden/ref_kernels.npz holds the outputs of cudaEM's device kernels (compiled unchanged
from the reference's headers with the constants header in oracle/ref_shim, run on a B200 by
tests/golden/make_golden.py) on the cases of tests/golden/ref_cases.py: the Fresnel
propagator, the k-space probe, the CTF (plain, with a source-point shift, partially coherent),
the annular detector sum and the spline projected potential of a slice.  Here, on the CPU,
the oracle's FP64 restatement of each operator must agree with them.

Bound: relative L2 <= 1e-5 (the reference computes in float).  Probe-aperture pixels whose g^2
lies within float rounding of the threshold are left out, as in the GPU comparison.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(HERE, "golden"))

import ref_cases  # noqa: E402
from conftest import rel_l2  # noqa: E402

GOLD = os.path.join(HERE, "golden", "ref_kernels.npz")
TOL = 1e-5


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def _c(a):
    a = np.asarray(a, np.float64).reshape(-1, 2)
    return a[:, 0] + 1j * a[:, 1]


@pytest.mark.parametrize("name", ref_cases.CASES)
def test_oracle_matches_reference_kernels(gold, name):
    _, inputs = ref_cases.build(name)
    for k, v in inputs.items():
        if isinstance(v, np.ndarray):
            assert np.array_equal(gold[f"{name}__in_{k}"], v), f"{name}: input {k} differs from the fixture's"
    want = gold[f"{name}__out"]
    got, keep = ref_cases.oracle(name)
    if name == "detector":
        assert abs(got[0] - want[0]) <= TOL * abs(want[0])
        return
    if name == "potential":
        assert np.abs(want).max() > 0
        assert rel_l2(got[keep], want.astype(np.float64)[keep]) < TOL
        return
    assert (~keep).sum() <= 8
    assert rel_l2(_c(got)[keep], _c(want)[keep]) < TOL


def test_a_planted_error_is_caught(gold):
    """The comparison is sharp: the oracle's propagator with its slice thickness off by 1e-3 A
    (0.05 %) fails it."""
    p, _ = ref_cases.build("propagator")
    import ctypes as C
    from oracle import oracle as orc
    p.dz = p.dz + 1e-3
    out = np.empty(2 * p.nx * p.ny)
    orc.lib().or_op_propagator(C.byref(p.c()), out.ctypes.data_as(C.POINTER(C.c_double)))
    assert rel_l2(_c(out), _c(gold["propagator__out"])) > TOL


def test_oracle_slice_loop_against_reference_loop_golden():
    """The oracle's composed slice loop against the reference's own loop (its cuFFT plans and load
    callbacks, run on a B200 by tests/golden/make_golden.py loop), sampled at fixed pixels."""
    import ref_loop_cases as rl
    from oracle import oracle as orc
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_loop.npz")
    g = np.load(path)
    for name in rl.CASES:
        p, V, psi0 = rl.build(name)
        want = orc.slice_loop(p, V, psi0)
        idx = g[f"{name}__idx"]
        assert np.array_equal(idx, rl.sample_index(want.shape[1] * want.shape[2]))
        got = g[f"{name}__out"].astype(np.complex128)
        w = want.reshape(want.shape[0], -1)[:, idx]
        assert rel_l2(got, w) < 1e-5, name
        # the whole exit waves' norms, as the reference computed them
        assert np.allclose(g[f"{name}__norm"], np.linalg.norm(want.reshape(want.shape[0], -1), axis=1), rtol=1e-5)
