"""The oracle's composed slice loop against the reference's own loop, through the C ABI.

oracle/_ref/libref_loop.so runs cudaEM's FFT_Dev plans with its cuFFT load callbacks
(fft_dev.cuh, fftcallbacks.cuh, compiled unchanged from the reference tree) in the order of
wave_modulation and wave_modulation_batch (wave_function.cuh:60-87): forward FFT with the
transmission callback, inverse FFT with the propagator callback, the last slice leaving the exit
wave in reciprocal space.  On the same phase slices, incident waves and the propagator of the
reference's own gen_propagator_kernel, the exit waves must agree with the oracle's FP64 loop, and
the engine's detector intensities with the annular sums of the reference's exit waves.

Bound: relative L2 <= 1e-5 (the reference computes in float through cuFFT).
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))

import ref_loop_cases as rl  # noqa: E402
from conftest import rel_l2  # noqa: E402
from oracle import oracle as orc  # noqa: E402

pytestmark = pytest.mark.gpu

TOL = 1e-5


@pytest.fixture(scope="module")
def libs():
    Ll, Lk = orc.ref_loop_lib(), orc.ref_lib()
    if Ll is None or Lk is None:
        pytest.skip("reference shims not built (needs the reference tree at build time)")
    return Ll, Lk


@pytest.mark.parametrize("name", rl.CASES)
def test_reference_loop_matches_oracle(libs, name):
    Ll, Lk = libs
    p, V, psi0 = rl.build(name)
    got = rl.reference(Ll, Lk, name)
    want = orc.slice_loop(p, V, psi0)
    assert got.shape == want.shape
    assert rel_l2(got, want) < TOL


def test_engine_detectors_match_reference_loop(libs, ctx):
    """The engine's STEM forward on the same slices and probes, against the detector sums of the
    reference's exit waves (the same annuli, summed in FP64 by the oracle's detector)."""
    import ctypes as C
    Ll, Lk = libs
    p, V, psi0 = rl.build("probe_batch")
    ref = rl.reference(Ll, Lk, "probe_batch").astype(np.complex128)
    I_ref = np.empty((ref.shape[0], p.n_det))
    for b in range(ref.shape[0]):
        w = np.ascontiguousarray(ref[b])
        out = np.empty(p.n_det)
        orc.lib().or_op_detect(C.byref(p.c()), w.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)),
                               out.ctypes.data_as(C.POINTER(C.c_double)))
        I_ref[b] = out
    pos = np.array([(12.8, 12.8), (11.1, 13.9), (14.6, 10.2), (9.7, 15.3)])
    I = ctx.stem_forward_potential(p, V, 0.9, pos)
    assert rel_l2(I, I_ref) < TOL
