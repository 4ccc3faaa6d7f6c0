"""Partially coherent HRTEM imaging against the FP64 oracle (relative L2 <= 1e-5).

* PCTF: the coherent CTF times the spatial/temporal envelope, for each incoherence mode.
* TCC: the incoherent sum over a Gauss-Hermite defocus quadrature and a source-point
  quadrature, for intensities and complex fields.
* A vanishing spread reduces both to the coherent image.
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


def _hrtem(illum, tsi, record=abi.MS_RECORD_INTENSITY, dsf=30.0, beta=0.5e-3, nt=5, ns=3):
    p, at = cases.hrtem_small(record=record)
    p.illumination_model = illum
    p.temporal_spatial_incoh = tsi
    p.obj_lens.dsf_sigma = dsf
    p.obj_lens.ssf_beta = beta
    p.obj_lens.dsf_npoints = nt
    p.obj_lens.ssf_npoints = ns
    return p, at


def _check(ctx, p, at):
    out = cb.MulSimulator(ctx=ctx).executionTEM(p, at)
    ref = orc.simulate_tem(p, at)
    if p.data_record == abi.MS_RECORD_WAVE:
        assert rel_l2(out.image_real + 1j * out.image_imag, ref[0] + 1j * ref[1]) < TOL
        return out.image_real + 1j * out.image_imag
    assert rel_l2(out.image_intensity, ref) < TOL
    return out.image_intensity


@pytest.mark.parametrize("tsi", [abi.MS_TSI_TEMPORAL_SPATIAL, abi.MS_TSI_TEMPORAL, abi.MS_TSI_SPATIAL])
def test_pctf(ctx, tsi):
    p, at = _hrtem(abi.MS_ILLUM_PARTIAL, tsi)
    _check(ctx, p, at)


@pytest.mark.parametrize("tsi,record", [(abi.MS_TSI_TEMPORAL_SPATIAL, abi.MS_RECORD_INTENSITY),
                                        (abi.MS_TSI_TEMPORAL, abi.MS_RECORD_INTENSITY),
                                        (abi.MS_TSI_SPATIAL, abi.MS_RECORD_INTENSITY),
                                        (abi.MS_TSI_TEMPORAL_SPATIAL, abi.MS_RECORD_WAVE)])
def test_tcc(ctx, tsi, record):
    p, at = _hrtem(abi.MS_ILLUM_TCC, tsi, record=record)
    _check(ctx, p, at)


def test_partial_coherence_without_spread_is_coherent(ctx):
    coh = _check(ctx, *_hrtem(abi.MS_ILLUM_COHERENT, abi.MS_TSI_TEMPORAL_SPATIAL))
    pctf = _check(ctx, *_hrtem(abi.MS_ILLUM_PARTIAL, abi.MS_TSI_TEMPORAL_SPATIAL, dsf=0.0, beta=0.0))
    tcc = _check(ctx, *_hrtem(abi.MS_ILLUM_TCC, abi.MS_TSI_TEMPORAL_SPATIAL, dsf=0.0, beta=0.0))
    assert rel_l2(pctf, coh) < 1e-6
    assert rel_l2(tcc, coh) < 1e-6


def test_spread_damps_contrast(ctx):
    """A larger defocus spread lowers the image contrast (the envelope damps high frequencies)."""
    lo = _check(ctx, *_hrtem(abi.MS_ILLUM_PARTIAL, abi.MS_TSI_TEMPORAL, dsf=10.0))
    hi = _check(ctx, *_hrtem(abi.MS_ILLUM_PARTIAL, abi.MS_TSI_TEMPORAL, dsf=80.0))
    assert np.std(hi) < np.std(lo)
