"""Batched execution forms against the FP64 oracle and against the engine's own single calls.

* Uneven batch (ms_simulate_many): CBED instances of mixed grids, slice counts, beam
  energies, convergence angles and phonon seeds in one call; each pattern within relative
  L2 1e-5 of the oracle and equal to the engine's single-simulation result.
* STEM probe batches replayed from a captured CUDA graph: identical to direct launches.
* Autotuned probe batch: the image does not depend on the batch the tuner picks.
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


def _mixed_jobs():
    jobs = []
    p, at = wl.cbed_si(cells=(2, 2, 4), n=128, nconf=2, seed=5)
    jobs.append((p, at))
    p, at = wl.hrtem_sto(cells=(3, 3, 3), n=256, nconf=1, seed=6)
    p.simulation_type = cb.abi.MS_SIM_CBED
    p.E0 = 200.0
    p.iw_x, p.iw_y = p.lx / 2, p.ly / 2
    p.cond_lens.outer_aper_ang = 0.015
    jobs.append((p, at))
    p, at = wl.cbed_si(cells=(2, 2, 2), n=128, nconf=1, seed=7)
    p.E0 = 120.0
    p.cond_lens.outer_aper_ang = 0.025
    jobs.append((p, at))
    p, at = wl.hrtem_sto(cells=(3, 3, 6), n=128, nconf=1, seed=8)
    p.simulation_type = cb.abi.MS_SIM_CBED
    p.E0 = 80.0
    p.iw_x, p.iw_y = p.lx / 2 + 0.3, p.ly / 2
    p.cond_lens.outer_aper_ang = 0.010
    jobs.append((p, at))
    p, at = wl.cbed_si(cells=(2, 2, 3), n=256, nconf=3, seed=9)
    p.E0 = 250.0
    p.cond_lens.outer_aper_ang = 0.030
    jobs.append((p, at))
    return jobs


def test_uneven_batch_matches_oracle_and_single_calls(ctx):
    jobs = _mixed_jobs()
    sim = cb.MulSimulator(ctx=ctx)
    outs, lat = sim.executionMany(jobs)
    assert len(outs) == len(jobs)
    assert np.all(np.isfinite(lat)) and np.all(lat > 0)
    for (p, at), o in zip(jobs, outs):
        ref = orc.simulate_cbed(p, at)
        assert rel_l2(o.image_intensity, ref) < TOL
        single = sim.executionCBED(p, at).image_intensity
        assert rel_l2(o.image_intensity, single) < 1e-7
    # inside one grid group (the 128^2 instances 0, 2, 3) instances finish in slice-count order
    group = sorted([0, 2, 3], key=lambda i: outs[i].n_slices)
    assert outs[group[0]].n_slices < outs[group[-1]].n_slices
    assert lat[group[0]] <= lat[group[1]] <= lat[group[2]]


def test_uneven_batch_rejects_other_modes(ctx):
    p, at = cases.hrtem_small()
    sim = cb.MulSimulator(ctx=ctx)
    with pytest.raises(cb.MsError):
        sim.executionMany([(p, at)])


def test_stem_graph_replay_identical_to_direct_launches(ctx):
    p, at = cases.stem_small(n=128, scan=(3, 3), batch=2)   # four full batches and a partial one
    sim = cb.MulSimulator(ctx=ctx)
    ctx.set_graphs(True)
    a = sim.executionSTEM(p, at).stem_intensity
    b = sim.executionSTEM(p, at).stem_intensity            # replayed from the cached graphs
    ctx.set_graphs(False)
    c = sim.executionSTEM(p, at).stem_intensity
    ctx.set_graphs(True)
    assert np.array_equal(a, b)
    assert np.array_equal(a, c)
    assert rel_l2(a, orc.simulate_stem(p, at)) < TOL


def test_stem_autotuned_batch(ctx):
    p, at = cases.stem_small(n=128, scan=(12, 8), nconf=1, batch=0)
    sim = cb.MulSimulator(ctx=ctx)
    a = sim.executionSTEM(p, at).stem_intensity
    chosen = ctx.last_probe_batch
    assert chosen in (32, 64)
    q = p.copy()
    q.probe_batch = 7
    b = sim.executionSTEM(q, at).stem_intensity
    assert ctx.last_probe_batch == 7
    assert rel_l2(a, b) < 1e-12
    assert rel_l2(a, orc.simulate_stem(p, at)) < TOL


def test_potential_chunks_overlap_identical(ctx):
    """Potentials computed in chunks on a side stream during the slice loop (the overlap switch)
    give the same pattern as computing them all before the loop (the default)."""
    p, at = cases.cbed_small(n=128, cells=(2, 2, 12), nconf=3)   # about 48 slices: three chunks
    sim = cb.MulSimulator(ctx=ctx)
    ctx.set_potential_overlap(True)
    try:
        a = sim.executionCBED(p, at)
    finally:
        ctx.set_potential_overlap(False)
    assert a.n_slices > 32
    b = sim.executionCBED(p, at)
    assert np.array_equal(a.image_intensity, b.image_intensity)
    assert rel_l2(a.image_intensity, orc.simulate_cbed(p, at)) < TOL
