"""Inputs of the reference-kernel golden fixtures, and the oracle's side of each comparison.

Each case builds the parameters and inputs of one per-pixel operator the way
tests/test_gpu_reference_kernels.py does, runs the reference's own CUDA kernel on them
(`reference(L, name)`, the shim library oracle/_ref/libref_kernels.so, on a GPU) or the
oracle's restatement (`oracle(name, inputs)`, on the CPU).  make_golden.py stores the
reference outputs in ref_kernels.npz; tests/test_golden.py compares the oracle with them.

Operators (reference file:line of the kernel the shim calls):
  propagator   gen_propagator_kernel   (device_kernels.cuh, the Fresnel propagator)
  probe        Generate_probe          (device_kernels.cuh:363-444)
  ctf_*        apply_CTF_kernel / apply_PCTF_kernel (device_kernels.cuh)
  detector     sum_square_over_Det     (device_kernels.cuh)
  potential    gen_slice_potential_kernel (device_kernels.cuh:28-47)
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

_TESTS = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, _TESTS)
sys.path.insert(0, os.path.dirname(_TESTS))

import cases  # noqa: E402
import cudaem_b200 as cb  # noqa: E402
from oracle import oracle as orc  # noqa: E402

CASES = ["propagator", "probe", "ctf_plain", "ctf_shift", "ctf_pctf", "detector", "potential"]
CTF_VARIANTS = {"ctf_plain": (0, (0.0, 0.0)), "ctf_shift": (0, (0.013, -0.021)), "ctf_pctf": (1, (0.0, 0.0))}


def _f(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _lam(p):
    lam, sig, _ = cb.physics(p.E0)
    return lam, sig


def g2_float(p, shift=(0.0, 0.0)):
    """g^2 of every pixel as the float grid computes it (plus a source-point shift), in float64."""
    dgx, dgy = np.float32(1.0) / np.float32(p.lx), np.float32(1.0) / np.float32(p.ly)
    kx = np.fft.fftfreq(p.nx, 1.0 / p.nx).astype(np.float32) * dgx + np.float32(shift[0])
    ky = np.fft.fftfreq(p.ny, 1.0 / p.ny).astype(np.float32) * dgy + np.float32(shift[1])
    return kx[None, :].astype(np.float64) ** 2 + ky[:, None].astype(np.float64) ** 2


def near(g2, thr, rel=4e-7):
    """Pixels whose g^2 lies within float rounding of a mask threshold."""
    return np.abs(g2 - thr) <= rel * max(thr, 1e-30)


def build(name):
    """Parameters and inputs of one case (deterministic: fixed workloads and seeds)."""
    if name == "propagator":
        p, _ = cases.hrtem_small(n=128)
        p.dz = 1.9525
        return p, {}
    if name == "probe":
        p, _ = cases.stem_small(n=128)
        p.cond_lens.c10 = -35.0
        p.cond_lens.c30 = 1.2e4
        lam, _ = _lam(p)
        thr = float(np.float32(np.sin(p.cond_lens.outer_aper_ang) / lam) ** 2)
        return p, {"thr": thr, "px": p.lx / 2 + 0.37, "py": p.ly / 2 - 0.21, "z0": 0.8}
    if name in CTF_VARIANTS:
        pctf, shift = CTF_VARIANTS[name]
        p, _ = cases.hrtem_small(n=128)
        p.obj_lens.c10 = -60.0
        p.obj_lens.c30 = 5.0e5
        p.obj_lens.dsf_sigma = 25.0
        p.obj_lens.ssf_beta = 0.4e-3
        p.temporal_spatial_incoh = 1
        lam, _ = _lam(p)
        thr = float(np.float32(np.sin(p.obj_lens.outer_aper_ang) / lam) ** 2)
        w = np.random.default_rng(4).standard_normal(2 * p.nx * p.ny).astype(np.float32)
        # pixels on the aperture edge (after the shift) carry no signal, so both masks agree on the rest
        w.reshape(-1, 2)[near(g2_float(p, shift), thr).ravel()] = 0.0
        return p, {"thr": thr, "pctf": pctf, "shift": shift, "w": w}
    if name == "detector":
        p, _ = cases.stem_small(n=128)
        p.set_detectors([(0.012, 0.045)])
        lam, _ = _lam(p)
        lo = float(np.float32(np.sin(0.012) / lam) ** 2)
        hi = float(np.float32(np.sin(0.045) / lam) ** 2)
        w = np.random.default_rng(5).standard_normal(2 * p.nx * p.ny).astype(np.float32)
        g2 = g2_float(p).ravel()
        w.reshape(-1, 2)[near(g2, lo) | near(g2, hi)] = 0.0
        return p, {"lo": lo, "hi": hi, "w": w}
    if name == "potential":
        p, _ = cases.hrtem_small(n=128)
        rng = np.random.default_rng(6)
        n = 24
        x = rng.uniform(3.0, p.lx - 3.0, n).astype(np.float32)
        y = rng.uniform(3.0, p.ly - 3.0, n).astype(np.float32)
        occ = rng.uniform(0.5, 1.0, n).astype(np.float32)
        return p, {"Z": 14, "x": x, "y": y, "occ": occ}
    raise KeyError(name)


def reference(L, name):
    """The reference kernel's output for a case (float32; the detector sum as a float64 scalar)."""
    p, a = build(name)
    lam, sig = _lam(p)
    N = p.nx * p.ny
    if name == "propagator":
        out = np.empty(2 * N, np.float32)
        assert L.ref_propagator(p.nx, p.ny, p.lx, p.ly, p.dz, 1, lam, _f(out)) == 0
        return out
    if name == "probe":
        out = np.empty(2 * N, np.float32)
        assert L.ref_probe(p.nx, p.ny, p.lx, p.ly, lam, p.cond_lens.c10 + a["z0"], p.cond_lens.c30, 0.0, a["thr"],
                           a["px"], a["py"], _f(out)) == 0
        return out
    if name in CTF_VARIANTS:
        out = np.empty(2 * N, np.float32)
        assert L.ref_ctf(p.nx, p.ny, p.lx, p.ly, lam, p.obj_lens.c10, p.obj_lens.c30, 0.0, a["thr"], a["pctf"],
                         p.obj_lens.dsf_sigma, p.obj_lens.ssf_beta, a["shift"][0], a["shift"][1], _f(a["w"]),
                         _f(out)) == 0
        return out
    if name == "detector":
        got = C.c_double()
        assert L.ref_detector(p.nx, p.ny, p.lx, p.ly, a["lo"], a["hi"], _f(a["w"]), C.byref(got)) == 0
        return np.array([got.value])
    if name == "potential":
        R2, c0, c1, c2, c3 = (np.empty(cb.abi.MS_NR) for _ in range(5))
        rmax = C.c_double()
        assert orc.lib().or_spline(C.byref(p.c()), a["Z"], _d(R2), _d(c0), _d(c1), _d(c2), _d(c3),
                                   C.byref(rmax)) == 0
        tab = [t.astype(np.float32) for t in (R2, c0, c1, c2, c3)]
        out = np.empty(N, np.float32)
        n = len(a["x"])
        assert L.ref_potential(p.nx, p.ny, p.lx, p.ly, n, _f(a["x"]), _f(a["y"]), _f(a["occ"]), *(_f(t) for t in tab),
                               rmax.value, sig / np.cos(p.theta), _f(out)) == 0
        return out
    raise KeyError(name)


def oracle(name):
    """The oracle's restatement of a case's operator (float64), and the mask of pixels compared."""
    p, a = build(name)
    N = p.nx * p.ny
    keep = np.ones(N, bool)
    if name == "propagator":
        out = np.empty(2 * N)
        orc.lib().or_op_propagator(C.byref(p.c()), _d(out))
    elif name == "probe":
        out = np.empty(2 * N)
        orc.lib().or_op_probe(C.byref(p.c()), a["px"], a["py"], a["z0"], _d(out))
        keep = ~near(g2_float(p), a["thr"]).ravel()
    elif name in CTF_VARIANTS:
        out = np.empty(2 * N)
        orc.lib().or_op_ctf(C.byref(p.c()), a["pctf"], 0.0, a["shift"][0], a["shift"][1],
                            _d(a["w"].astype(np.float64)), _d(out))
    elif name == "detector":
        out = np.empty(1)
        orc.lib().or_op_detect(C.byref(p.c()), _d(a["w"].astype(np.float64)), _d(out))
        keep = None
    elif name == "potential":
        out = np.empty(N)
        orc.lib().or_op_slice_potential(C.byref(p.c()), a["Z"], len(a["x"]), _f(a["x"]), _f(a["y"]), _f(a["occ"]),
                                        _d(out))
    else:
        raise KeyError(name)
    return out, keep
