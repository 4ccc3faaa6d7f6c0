"""The five V(r) parameterisations of the reference on the GPU, against the FP64 oracle.

Vr_dVrir_Doyle/Peng/Kirkland/Weickenmeier/Lobato (basic_functions_dev.cuh:102-186) feed the
radial splines of the projected potential.  Every form is passed per element through
ms_params.element_coefs; the GPU potential (spline evaluation on the device) and a full
HRTEM / CBED simulation are compared with the oracle built from the same coefficients.

The coefficients are synthetic: each form's functional shape with magnitudes and decay
lengths chosen to give projected potentials of a realistic size (tens of V*A near a
nucleus).  They are not a published table; parity does not depend on the values, since
engine and oracle read the same ones.

Bounds: relative L2 <= 2e-6 for potentials, <= 1e-5 for simulated images and patterns.
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import cases  # noqa: E402
import cudaem_b200 as cb  # noqa: E402
from cudaem_b200 import _abi as abi  # noqa: E402
from conftest import rel_l2  # noqa: E402
from oracle import oracle as orc  # noqa: E402

pytestmark = pytest.mark.gpu

TOL = 1e-5
TOL_POT = 2e-6


def synthetic_coefs(form: int, Z: int):
    """(cl, cnl) of one element in `form`, scaled with Z."""
    s = float(Z)
    if form in (abi.MS_POT_DOYLE_0_4,):
        return [4.0 * s, 2.2 * s, 0.9 * s, 0.25 * s], [9.0, 2.1, 0.55, 0.12]
    if form in (abi.MS_POT_PENG_0_4, abi.MS_POT_PENG_0_12):
        return [5.0 * s, 2.6 * s, 1.1 * s, 0.4 * s, 0.1 * s], [14.0, 4.0, 1.2, 0.35, 0.09]
    if form == abi.MS_POT_KIRKLAND_0_12:
        # three Yukawa terms cl e^{-cnl r}/r, then three Gaussians cl e^{-cnl r^2}
        return [1.6 * s, 0.9 * s, 0.3 * s, 1.2 * s, 0.5 * s, 0.2 * s], [3.5, 1.4, 0.6, 12.0, 2.5, 0.4]
    if form == abi.MS_POT_WEICKENMEIER_0_12:
        # cl erfc(cnl r)/r
        return [1.0 * s, 0.8 * s, 0.5 * s, 0.3 * s, 0.2 * s, 0.1 * s], [4.0, 2.5, 1.6, 1.1, 0.8, 0.5]
    if form == abi.MS_POT_LOBATO_0_12:
        # cl e^{-cnl r} (2/(cnl r) + 1)
        return [0.9 * s, 0.6 * s, 0.35 * s, 0.2 * s, 0.08 * s], [6.0, 3.2, 1.8, 1.0, 0.55]
    raise ValueError(form)


FORMS = [abi.MS_POT_DOYLE_0_4, abi.MS_POT_PENG_0_4, abi.MS_POT_PENG_0_12, abi.MS_POT_KIRKLAND_0_12,
         abi.MS_POT_WEICKENMEIER_0_12, abi.MS_POT_LOBATO_0_12]


def with_form(p, form, Zs=(8, 22, 38)):
    p.set_element_coefs([(Z, form, *synthetic_coefs(form, Z)) for Z in Zs])
    p.potential_type = form
    return p


@pytest.mark.parametrize("form", FORMS)
def test_projected_potential_form(ctx, form):
    p, at = cases.hrtem_small(nconf=1)
    with_form(p, form)
    V = ctx.projected_potential(p, at, conf=1)
    Vo, _ = orc.potential(p, at, 1)
    assert V.shape == Vo.shape
    assert np.abs(Vo).max() > 0.1        # a non-trivial potential reached the grid
    assert rel_l2(V, Vo) < TOL_POT


@pytest.mark.parametrize("form", FORMS)
def test_projected_potential_form_si(ctx, form):
    p, at = cases.cbed_small(nconf=2)
    with_form(p, form, Zs=(14,))
    V = ctx.projected_potential(p, at, conf=2)
    Vo, _ = orc.potential(p, at, 2)
    assert rel_l2(V, Vo) < TOL_POT


@pytest.mark.parametrize("form", [abi.MS_POT_LOBATO_0_12, abi.MS_POT_WEICKENMEIER_0_12])
def test_hrtem_with_form(ctx, form):
    p, at = cases.hrtem_small()
    with_form(p, form)
    out = cb.MulSimulator(ctx=ctx).executionTEM(p, at)
    assert rel_l2(out.image_intensity, orc.simulate_tem(p, at)) < TOL


@pytest.mark.parametrize("form", [abi.MS_POT_KIRKLAND_0_12, abi.MS_POT_PENG_0_12, abi.MS_POT_DOYLE_0_4])
def test_cbed_with_form(ctx, form):
    p, at = cases.cbed_small(nconf=2)
    with_form(p, form, Zs=(14,))
    out = cb.MulSimulator(ctx=ctx).executionCBED(p, at)
    assert rel_l2(out.image_intensity, orc.simulate_cbed(p, at)) < TOL


def test_mixed_forms_per_element(ctx):
    """Each element in its own form inside one specimen (the reference's per-element table)."""
    p, at = cases.hrtem_small()
    p.set_element_coefs([(8, abi.MS_POT_LOBATO_0_12, *synthetic_coefs(abi.MS_POT_LOBATO_0_12, 8)),
                         (22, abi.MS_POT_KIRKLAND_0_12, *synthetic_coefs(abi.MS_POT_KIRKLAND_0_12, 22)),
                         (38, abi.MS_POT_WEICKENMEIER_0_12, *synthetic_coefs(abi.MS_POT_WEICKENMEIER_0_12, 38))])
    V = ctx.projected_potential(p, at, conf=1)
    Vo, _ = orc.potential(p, at, 1)
    assert rel_l2(V, Vo) < TOL_POT
