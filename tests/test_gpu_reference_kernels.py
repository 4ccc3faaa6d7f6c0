"""The oracle's per-pixel operators against the reference's own CUDA kernels.

The reference cannot be built as shipped, but its device kernels compile unchanged from
their own files with the constants header in oracle/ref_shim (oracle/_ref/libref_kernels.so,
built by `make -C oracle ref` where the reference tree is present).  On the same inputs,
each operator the oracle restates must agree with the reference's float kernel:

  propagator P(k), k-space probe, CTF (with a source-point shift), partially coherent CTF,
  annular detector sum, spline projected potential of a slice.

Bound: relative L2 <= 1e-5 (the reference computes in float).  Aperture and detector
masks are float comparisons of g^2 against a threshold; pixels whose g^2 lies within a
few float ulps of a threshold can fall on either side depending on how a compiler fuses
g_x^2 + g_y^2, so those boundary pixels are excluded (they are counted, and must be few).
"""
import ctypes as C
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import cases  # noqa: E402
import cudaem_b200 as cb  # noqa: E402
from conftest import rel_l2  # noqa: E402
from oracle import oracle as orc  # noqa: E402

pytestmark = pytest.mark.gpu

TOL = 1e-5


@pytest.fixture(scope="module")
def ref():
    L = orc.ref_lib()
    if L is None:
        pytest.skip("reference-kernel shim not built (needs the reference tree at build time)")
    return L


def _f(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _g2_float(p):
    """g^2 of every pixel as the float grid computes it, and its float64 value."""
    dgx, dgy = np.float32(1.0) / np.float32(p.lx), np.float32(1.0) / np.float32(p.ly)
    kx = np.fft.fftfreq(p.nx, 1.0 / p.nx).astype(np.float32)
    ky = np.fft.fftfreq(p.ny, 1.0 / p.ny).astype(np.float32)
    gx, gy = kx * dgx, ky * dgy
    return (gx[None, :].astype(np.float64) ** 2 + gy[:, None].astype(np.float64) ** 2)


def _near(g2, thr, rel=4e-7):
    return np.abs(g2 - thr) <= rel * max(thr, 1e-30)


def _lam(p):
    lam, sig, _ = cb.physics(p.E0)
    return lam, sig


def _c(a):
    return a.reshape(-1, 2)[:, 0] + 1j * a.reshape(-1, 2)[:, 1]


def test_propagator(ref):
    p, _ = cases.hrtem_small(n=128)
    p.dz = 1.9525
    lam, _ = _lam(p)
    got = np.empty(2 * p.nx * p.ny, np.float32)
    assert ref.ref_propagator(p.nx, p.ny, p.lx, p.ly, p.dz, 1, lam, _f(got)) == 0
    want = np.empty(2 * p.nx * p.ny)
    orc.lib().or_op_propagator(C.byref(p.c()), _d(want))
    assert rel_l2(_c(got), _c(want)) < TOL


def test_probe(ref):
    p, _ = cases.stem_small(n=128)
    p.cond_lens.c10 = -35.0
    p.cond_lens.c30 = 1.2e4
    lam, _ = _lam(p)
    thr = np.float32(np.sin(p.cond_lens.outer_aper_ang) / lam) ** 2
    px, py, z0 = p.lx / 2 + 0.37, p.ly / 2 - 0.21, 0.8
    got = np.empty(2 * p.nx * p.ny, np.float32)
    assert ref.ref_probe(p.nx, p.ny, p.lx, p.ly, lam, p.cond_lens.c10 + z0, p.cond_lens.c30, 0.0, float(thr), px, py,
                         _f(got)) == 0
    want = np.empty(2 * p.nx * p.ny)
    orc.lib().or_op_probe(C.byref(p.c()), px, py, z0, _d(want))
    keep = ~_near(_g2_float(p), float(thr)).ravel()
    assert (~keep).sum() <= 8
    assert rel_l2(_c(got)[keep], _c(want)[keep]) < TOL


@pytest.mark.parametrize("pctf,shift", [(0, (0.0, 0.0)), (0, (0.013, -0.021)), (1, (0.0, 0.0))])
def test_ctf(ref, pctf, shift):
    p, _ = cases.hrtem_small(n=128)
    p.obj_lens.c10 = -60.0
    p.obj_lens.c30 = 5.0e5
    p.obj_lens.dsf_sigma = 25.0
    p.obj_lens.ssf_beta = 0.4e-3
    p.temporal_spatial_incoh = 1
    lam, _ = _lam(p)
    thr = np.float32(np.sin(p.obj_lens.outer_aper_ang) / lam) ** 2
    rng = np.random.default_rng(4)
    w = rng.standard_normal(2 * p.nx * p.ny)
    # pixels on the aperture edge (after the shift) carry no signal, so both masks agree on the rest
    dgx, dgy = np.float32(1.0) / np.float32(p.lx), np.float32(1.0) / np.float32(p.ly)
    kx = np.fft.fftfreq(p.nx, 1.0 / p.nx).astype(np.float32) * dgx + np.float32(shift[0])
    ky = np.fft.fftfreq(p.ny, 1.0 / p.ny).astype(np.float32) * dgy + np.float32(shift[1])
    g2 = kx[None, :].astype(np.float64) ** 2 + ky[:, None].astype(np.float64) ** 2
    edge = _near(g2, float(thr)).ravel()
    w.reshape(-1, 2)[edge] = 0.0
    got = np.empty(2 * p.nx * p.ny, np.float32)
    assert ref.ref_ctf(p.nx, p.ny, p.lx, p.ly, lam, p.obj_lens.c10, p.obj_lens.c30, 0.0, float(thr), pctf,
                       p.obj_lens.dsf_sigma, p.obj_lens.ssf_beta, shift[0], shift[1], _f(w.astype(np.float32)),
                       _f(got)) == 0
    want = np.empty(2 * p.nx * p.ny)
    orc.lib().or_op_ctf(C.byref(p.c()), pctf, 0.0, shift[0], shift[1], _d(w.astype(np.float32).astype(np.float64)),
                        _d(want))
    assert rel_l2(_c(got), _c(want)) < TOL


def test_detector(ref):
    p, _ = cases.stem_small(n=128)
    p.set_detectors([(0.012, 0.045)])
    lam, _ = _lam(p)
    lo = np.float32(np.sin(0.012) / lam) ** 2
    hi = np.float32(np.sin(0.045) / lam) ** 2
    rng = np.random.default_rng(5)
    w = rng.standard_normal(2 * p.nx * p.ny).astype(np.float32)
    g2 = _g2_float(p).ravel()
    w.reshape(-1, 2)[_near(g2, float(lo)) | _near(g2, float(hi))] = 0.0
    got = C.c_double()
    assert ref.ref_detector(p.nx, p.ny, p.lx, p.ly, float(lo), float(hi), _f(w), C.byref(got)) == 0
    want = np.empty(1)
    orc.lib().or_op_detect(C.byref(p.c()), _d(w.astype(np.float64)), _d(want))
    assert abs(got.value - want[0]) / want[0] < TOL


def test_slice_potential(ref):
    p, _ = cases.hrtem_small(n=256)
    lam, sig = _lam(p)
    Z = 14
    R2, c0, c1, c2, c3 = (np.empty(cb.abi.MS_NR) for _ in range(5))
    rmax = C.c_double()
    assert orc.lib().or_spline(C.byref(p.c()), Z, _d(R2), _d(c0), _d(c1), _d(c2), _d(c3), C.byref(rmax)) == 0
    rng = np.random.default_rng(6)
    n = 40
    x = rng.uniform(3.0, p.lx - 3.0, n).astype(np.float32)
    y = rng.uniform(3.0, p.ly - 3.0, n).astype(np.float32)
    occ = rng.uniform(0.5, 1.0, n).astype(np.float32)
    got = np.empty(p.nx * p.ny, np.float32)
    tab = [a.astype(np.float32) for a in (R2, c0, c1, c2, c3)]
    assert ref.ref_potential(p.nx, p.ny, p.lx, p.ly, n, _f(x), _f(y), _f(occ), *(_f(t) for t in tab), rmax.value,
                             sig / np.cos(p.theta), _f(got)) == 0
    want = np.empty(p.nx * p.ny)
    orc.lib().or_op_slice_potential(C.byref(p.c()), Z, n, _f(x), _f(y), _f(occ), _d(want))
    assert rel_l2(got, want) < TOL
