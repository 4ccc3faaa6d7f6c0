"""Parity at the largest grid (2048^2) and at the full STEM shape, through the C ABI.

The 2048-point passes use their own team layout (32 threads of 64 points per transform,
one resident block per SM); these tests compare them with the FP64 oracle directly:
a raw slice loop on random phases, a frozen-phonon CBED pattern, and an uneven batch that
mixes 256^2, 1024^2 and 2048^2 instances in one ms_simulate_many call.  The full-size STEM
test runs the ADF workload's own grid and depth (SrTiO3 16x16x25 cells, 1024^2, 50 slices,
ADF 60-200 mrad) on 16 probe positions and 2 phonon configurations.

Bound: relative L2 <= 1e-5 for every output.
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import cases  # noqa: E402
import cudaem_b200 as cb  # noqa: E402
from conftest import rel_l2  # noqa: E402
from cudaem_b200 import workloads as wl  # noqa: E402
from oracle import oracle as orc  # noqa: E402

pytestmark = pytest.mark.gpu

TOL = 1e-5


def test_slice_loop_random_phases_2048(ctx):
    p, _ = cases.stem_small(n=2048)
    p.lx = p.ly = 2048 * 0.12
    V = cases.random_phase_slices(p, 6, seed=2048)
    xy = np.array([[p.lx / 2, p.ly / 2], [p.lx / 3, p.ly / 2 + 0.7], [p.lx / 2 + 5.1, p.ly / 4]])
    I = ctx.stem_forward_potential(p, V, 0.9, xy)
    Io = orc.stem_forward_potential(p, V, 0.9, xy)
    assert rel_l2(I, Io) < TOL


def test_slice_loop_rectangular_2048(ctx):
    """2048 points across, 512 down (and the transpose): each axis keeps its own team layout."""
    for nx, ny in ((2048, 512), (512, 2048)):
        p, _ = cases.stem_small(n=128)
        p.nx, p.ny = nx, ny
        p.lx, p.ly = nx * 0.1, ny * 0.1
        V = cases.random_phase_slices(p, 4, seed=nx + 3 * ny)
        xy = np.array([[p.lx / 2, p.ly / 2]])
        assert rel_l2(ctx.stem_forward_potential(p, V, 0.3, xy), orc.stem_forward_potential(p, V, 0.3, xy)) < TOL


def test_cbed_2048_frozen_phonons(ctx):
    p, at = wl.cbed_si(cells=(8, 8, 4), n=2048, nconf=2)
    out = cb.MulSimulator(ctx=ctx).executionCBED(p, at)
    assert out.n_slices == 16
    ref = orc.simulate_cbed(p, at)
    assert rel_l2(out.image_intensity, ref) < TOL


def test_hrtem_2048(ctx):
    p, at = wl.hrtem_sto(cells=(10, 10, 4), n=2048)
    out = cb.MulSimulator(ctx=ctx).executionTEM(p, at)
    assert rel_l2(out.image_intensity, orc.simulate_tem(p, at)) < TOL


def _uneven_jobs_with_2048():
    jobs = []
    p, at = wl.hrtem_sto(cells=(6, 6, 4), n=256, nconf=1, seed=21)
    p.simulation_type = cb.abi.MS_SIM_CBED
    p.iw_x, p.iw_y = p.lx / 2, p.ly / 2
    p.cond_lens.outer_aper_ang = 0.018
    jobs.append((p, at))
    p, at = wl.cbed_si(cells=(6, 6, 3), n=1024, nconf=1, seed=22)
    p.E0 = 150.0
    p.cond_lens.outer_aper_ang = 0.025
    jobs.append((p, at))
    p, at = wl.cbed_si(cells=(8, 8, 2), n=2048, nconf=1, seed=23)
    p.E0 = 240.0
    p.cond_lens.outer_aper_ang = 0.012
    jobs.append((p, at))
    p, at = wl.hrtem_sto(cells=(10, 10, 5), n=2048, nconf=1, seed=24)
    p.simulation_type = cb.abi.MS_SIM_CBED
    p.E0 = 90.0
    p.iw_x, p.iw_y = p.lx / 2 + 0.4, p.ly / 2
    p.cond_lens.outer_aper_ang = 0.028
    jobs.append((p, at))
    return jobs


def test_uneven_batch_with_2048_instances(ctx):
    jobs = _uneven_jobs_with_2048()
    sim = cb.MulSimulator(ctx=ctx)
    outs, lat = sim.executionMany(jobs)
    assert {p.nx for p, _ in jobs} == {256, 1024, 2048}
    for (p, at), o in zip(jobs, outs):
        ref = orc.simulate_cbed(p, at)
        assert rel_l2(o.image_intensity, ref) < TOL, (p.nx, o.n_slices)
        single = sim.executionCBED(p, at).image_intensity
        assert rel_l2(o.image_intensity, single) < 1e-7
    assert np.all(np.isfinite(lat)) and np.all(lat > 0)


def test_full_size_stem_16_probes_2_configurations(ctx):
    """The ADF workload's grid and depth on 16 of its probe positions (a 4x4 patch of the
    0.2 A scan) and 2 of its 10 phonon configurations, batched in one call."""
    p, at = wl.stem_sto(nconf=2, scan=(4, 4))
    out = cb.MulSimulator(ctx=ctx).executionSTEM(p, at)
    ref = orc.simulate_stem(p, at)
    assert out.stem_intensity.shape == (1, 4, 4)
    assert rel_l2(out.stem_intensity, ref) < TOL
