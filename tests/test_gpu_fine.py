"""Fine slicing on the GPU against the FP64 oracle.

Every atom contributes to each slice whose integration range reaches it, with its potential
integrated over that slice (64-point Gauss-Legendre in z, FP64 on the device) and re-splined.
Bounds: projected potentials relative L2 <= 2e-6; CBED and HRTEM outputs <= 1e-5.
"""
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
TOL_POT = 2e-6


@pytest.mark.parametrize("wrap,conf,rmax", [(0, 0, 3.0), (1, 1, 3.0), (0, 2, 2.0)])
def test_fine_potentials(ctx, wrap, conf, rmax):
    p, at = cases.hrtem_small(wrap=wrap, nconf=2)
    p.enable_fine_slicing = 1
    p.pot_rmax = rmax
    V = ctx.projected_potential(p, at, conf=conf)
    Vo, _ = orc.potential(p, at, conf)
    assert V.shape == Vo.shape
    assert rel_l2(V, Vo) < TOL_POT


def test_fine_cbed(ctx):
    p, at = cases.cbed_small(nconf=2)
    p.enable_fine_slicing = 1
    out = cb.MulSimulator(ctx=ctx).executionCBED(p, at)
    ref = orc.simulate_cbed(p, at)
    assert rel_l2(out.image_intensity, ref) < TOL


def test_fine_hrtem(ctx):
    p, at = cases.hrtem_small()
    p.enable_fine_slicing = 1
    out = cb.MulSimulator(ctx=ctx).executionTEM(p, at)
    assert rel_l2(out.image_intensity, orc.simulate_tem(p, at)) < TOL


def test_fine_slices_add_up_to_projection(ctx):
    """Summed over slices, the fine-sliced potential approaches the projected one: the slice
    integrals tile each atom's z line.  What is left is the z tail beyond the integration
    radius, and the fixed z quadrature across the 1/r peak of a nucleus, so pixels within
    0.2 A of an atom column are left out."""
    p, at = cases.hrtem_small(nconf=1)
    p.phonon_model = cb.abi.MS_PHONON_STILL
    p.pot_rmax = 5.0
    Vp = ctx.projected_potential(p, at).sum(0)
    p.enable_fine_slicing = 1
    Vf = ctx.projected_potential(p, at).sum(0)
    X, Y = np.meshgrid(np.arange(p.nx) * p.lx / p.nx, np.arange(p.ny) * p.ly / p.ny)
    far = np.ones(X.shape, bool)
    for x, y in set(zip(np.round(at.x, 4), np.round(at.y, 4))):
        far &= (X - x) ** 2 + (Y - y) ** 2 > 0.2 ** 2
    assert far.mean() > 0.9
    assert rel_l2(Vf[far], Vp[far]) < 0.005
