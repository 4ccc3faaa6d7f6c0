"""Cases for the reference's composed slice loop (oracle/_ref/libref_loop.so: the reference's
FFT_Dev plans with its cuFFT load callbacks, in the order of wave_modulation and
wave_modulation_batch) and the oracle's restatement of the same loop (orc.slice_loop).

Each case builds its grid, phase slices and incident waves from fixed seeds.  The golden file
keeps the reference's exit waves at SAMPLE fixed pixels of every wave, so that the fixture stays
small while the comparison still covers the whole spectrum.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import cases  # noqa: E402
from oracle import oracle as orc  # noqa: E402

SAMPLE = 8192


def grid(n=256):
    p, _ = cases.stem_small(n=n)
    p.lx = p.ly = n * 0.1
    p.cond_lens.outer_aper_ang = 0.021
    return p


def build(name):
    """(params, V [S][n][n] float32, psi0 [B][n][n] complex128)."""
    p = grid()
    if name == "plane_wave":
        V = cases.random_phase_slices(p, 12, seed=101, amp=0.5)
        psi0 = np.ones((1, p.ny, p.nx), np.complex128)
    elif name == "probe_batch":
        V = cases.random_phase_slices(p, 8, seed=102, amp=0.5)
        pos = [(12.8, 12.8), (11.1, 13.9), (14.6, 10.2), (9.7, 15.3)]
        psi0 = np.stack([orc.incident(p, x, y, 0.9) for x, y in pos])
    else:
        raise KeyError(name)
    return p, V, psi0


CASES = ["plane_wave", "probe_batch"]


def sample_index(n_pix):
    return np.sort(np.random.default_rng(7).choice(n_pix, size=SAMPLE, replace=False))


def reference(loop_lib, kern_lib, name):
    """The reference's exit waves [B][n][n] (complex64) on the case's inputs, with the propagator
    from its own gen_propagator_kernel."""
    import cudaem_b200 as cb
    p, V, psi0 = build(name)
    lam, _, _ = cb.physics(p.E0)
    P = np.empty(2 * p.nx * p.ny, np.float32)
    f = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))  # noqa: E731
    assert kern_lib.ref_propagator(p.nx, p.ny, p.lx, p.ly, p.dz, 1, lam, f(P)) == 0
    w0 = np.ascontiguousarray(psi0.astype(np.complex64))
    out = np.empty_like(w0)
    rc = loop_lib.ref_slice_loop(p.nx, V.shape[0], f(V), w0.shape[0], f(w0.view(np.float32)), f(P),
                                 f(out.view(np.float32)))
    assert rc == 0, rc
    return out
