"""Parity of the CUDA engine with the FP64 oracle, through the C ABI.

Bound: relative L2 error <= 1e-5 for every forward output (exit waves,
images, patterns, detector intensities), <= 2e-6 for projected potentials.
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


@pytest.mark.parametrize("wrap", [0, 1])
@pytest.mark.parametrize("conf", [0, 1])
def test_projected_potential(ctx, wrap, conf):
    p, at = cases.hrtem_small(wrap=wrap)
    V = ctx.projected_potential(p, at, conf=conf)
    Vo, _ = orc.potential(p, at, conf)
    assert V.shape == Vo.shape
    assert rel_l2(V, Vo) < TOL_POT


@pytest.mark.parametrize("cells,n,rmax,conf", [((5, 5, 4), 128, 3.0, 1), ((7, 5, 2), 256, 2.3, 0),
                                               ((3, 4, 2), 128, 3.3, 1)])
def test_projected_potential_periodic_images(ctx, cells, n, rmax, conf):
    """Periodic wrap on boxes whose length is not a multiple of the atom-cell size (the cut-off):
    the cell ranges of a pixel block are looked up per periodic image, so no image of an atom
    within the cut-off of the box edges is missed."""
    p, at = cases.hrtem_small(n=n, cells=cells, nconf=2, wrap=1)
    p.pot_rmax = rmax
    V = ctx.projected_potential(p, at, conf=conf)
    Vo, _ = orc.potential(p, at, conf)
    assert V.shape == Vo.shape
    assert rel_l2(V, Vo) < TOL_POT


@pytest.mark.parametrize("n", [128, 256, 512, 1024])
def test_slice_loop_random_phases(ctx, n):
    p, _ = cases.stem_small(n=n)
    p.lx = p.ly = n * 0.12
    S = 5 if n <= 512 else 3
    V = cases.random_phase_slices(p, S, seed=n)
    xy = np.array([[p.lx / 2, p.ly / 2], [p.lx / 3, p.ly / 2 + 0.7]])
    I = ctx.stem_forward_potential(p, V, 0.9, xy)
    Io = orc.stem_forward_potential(p, V, 0.9, xy)
    assert rel_l2(I, Io) < TOL


def test_slice_loop_rectangular(ctx):
    p, _ = cases.stem_small(n=128)
    p.ny = 256
    p.ly = 256 * 0.12
    p.lx = 128 * 0.12
    V = cases.random_phase_slices(p, 4, seed=3)
    xy = np.array([[p.lx / 2, p.ly / 2]])
    assert rel_l2(ctx.stem_forward_potential(p, V, 0.0, xy), orc.stem_forward_potential(p, V, 0.0, xy)) < TOL


@pytest.mark.parametrize("record", [abi.MS_RECORD_INTENSITY, abi.MS_RECORD_WAVE])
def test_hrtem(ctx, record):
    p, at = cases.hrtem_small(record=record)
    out = cb.MulSimulator(ctx=ctx).executionTEM(p, at)
    ref = orc.simulate_tem(p, at)
    if record == abi.MS_RECORD_WAVE:
        got = out.image_real + 1j * out.image_imag
        assert rel_l2(got, ref[0] + 1j * ref[1]) < TOL
    else:
        assert rel_l2(out.image_intensity, ref) < TOL
    assert out.launches > 0


@pytest.mark.parametrize("record", [abi.MS_RECORD_INTENSITY, abi.MS_RECORD_WAVE])
def test_ed(ctx, record):
    p, at = cases.ed_small(record=record)
    out = cb.MulSimulator(ctx=ctx).executionTEM(p, at)
    ref = orc.simulate_tem(p, at)
    if record == abi.MS_RECORD_WAVE:
        assert rel_l2(out.image_real + 1j * out.image_imag, ref[0] + 1j * ref[1]) < TOL
    else:
        assert rel_l2(out.image_intensity, ref) < TOL


@pytest.mark.parametrize("wrap", [0, 1])
def test_cbed_frozen_phonons(ctx, wrap):
    p, at = cases.cbed_small(nconf=3, wrap=wrap)
    out = cb.MulSimulator(ctx=ctx).executionCBED(p, at)
    ref = orc.simulate_cbed(p, at)
    assert rel_l2(out.image_intensity, ref) < TOL


@pytest.mark.parametrize("plain", [False, True])
def test_stem(ctx, plain):
    p, at = cases.stem_small(plain=plain)
    out = cb.MulSimulator(ctx=ctx).executionSTEM(p, at)
    ref = orc.simulate_stem(p, at)
    assert out.stem_intensity.shape == ref.shape
    assert rel_l2(out.stem_intensity, ref) < TOL


def test_stem_batch_sizes_agree(ctx):
    p, at = cases.stem_small(scan=(4, 3), nconf=1)
    res = []
    for b in (1, 5, 12):
        q = p.copy()
        q.probe_batch = b
        res.append(cb.MulSimulator(ctx=ctx).executionSTEM(q, at).stem_intensity)
    assert rel_l2(res[1], res[0]) < 1e-6 and rel_l2(res[2], res[0]) < 1e-6


def test_full_size_cbed_one_configuration(ctx):
    """The measured CBED workload at its real depth and sampling (Si 16x16x60 cells, 1024^2,
    240 slices) for one phonon configuration: FP32 error after 240 slices stays within 1e-5."""
    from cudaem_b200 import workloads as wl
    p, at = wl.cbed_si(nconf=1)
    out = cb.MulSimulator(ctx=ctx).executionCBED(p, at)
    assert out.n_slices == 240
    ref = orc.simulate_cbed(p, at)
    assert rel_l2(out.image_intensity, ref) < TOL


def test_full_size_hrtem(ctx):
    """The measured HRTEM workload (SrTiO3 10x10x20 cells, 512^2, 40 slices, -10 nm, Cs 1 mm)."""
    from cudaem_b200 import workloads as wl
    p, at = wl.hrtem_sto()
    out = cb.MulSimulator(ctx=ctx).executionTEM(p, at)
    ref = orc.simulate_tem(p, at)
    assert rel_l2(out.image_intensity, ref) < TOL


def test_full_size_stem_probes(ctx):
    """Two probes of the measured STEM workload (SrTiO3 16x16x25, 1024^2, 50 slices, ADF 60-200 mrad)."""
    from cudaem_b200 import workloads as wl
    p, at = wl.stem_sto(nconf=1, scan=(2, 1), step=0.8)
    out = cb.MulSimulator(ctx=ctx).executionSTEM(p, at)
    ref = orc.simulate_stem(p, at)
    assert rel_l2(out.stem_intensity, ref) < TOL


def test_thickness(ctx):
    p, at = cases.thickness_small()
    out = cb.ThicknessSimulator(ctx=ctx).run(p, at)
    ref = orc.simulate_thickness(p, at)
    assert out.thickness_frames.shape == ref.shape
    assert rel_l2(out.thickness_frames, ref) < TOL


def test_thickness_convergent_phonons(ctx):
    p, at = cases.thickness_small(nconf=2)
    p.iw_type = abi.MS_IW_CONVERGENT
    p.cond_lens.outer_aper_ang = 0.02
    p.iw_x = p.lx / 2
    p.iw_y = p.ly / 2
    out = cb.ThicknessSimulator(ctx=ctx).run(p, at)
    ref = orc.simulate_thickness(p, at)
    assert rel_l2(out.thickness_frames, ref) < TOL


def test_kernel_limits_survive_switching_specimens(ctx):
    """Launch-size bookkeeping across calls: three-element, one-element, then three-element
    specimens again in one context (the potential kernel's shared memory grows with the number
    of elements) all run and match the oracle."""
    for maker in (cases.hrtem_small, cases.cbed_small, cases.hrtem_small):
        p, at = maker()
        V = ctx.projected_potential(p, at, conf=0)
        Vo, _ = orc.potential(p, at, 0)
        assert rel_l2(V, Vo) < TOL_POT
