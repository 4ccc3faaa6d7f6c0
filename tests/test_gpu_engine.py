"""The persistent slice engine (pass-kernel variant 2) against the per-slice launches and the oracle.

The engine runs the row and column steps of every slice of a batch in one launch: resident blocks
take work items in slice order from a ticket counter and wait, bounded, on per-wave slice counters
for the items an item depends on.  It computes the same transforms as the per-slice kernels, so
every output agrees with them to float rounding (relative L2 <= 1e-6) and with the FP64 oracle to
the same tolerance as the per-slice path (1e-5).  Covered: CBED at 128..2048 points with phonon
configurations of different slice counts (items of finished waves skipped), plane-wave HRTEM and
electron diffraction (the first slice runs as separate passes, the engine the rest), the tilted
plane wave, STEM probe batches (a full and a partial batch, the graph replay), an uneven batch of
several grids (instances finish in slice-count order inside a grid group; a rectangular grid runs
in the per-slice kernels beside the engine groups), and a dependency wait that runs out.
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import cases  # noqa: E402
import cudaem_b200 as cb  # noqa: E402
from cudaem_b200 import _abi as abi  # noqa: E402
from cudaem_b200 import workloads as wl  # noqa: E402
from conftest import rel_l2  # noqa: E402
from oracle import oracle as orc  # noqa: E402

pytestmark = pytest.mark.gpu

ENGINE = 2
PER_SLICE = 3
TOL_SAME = 1e-6
TOL_ORACLE = 1e-5


def _both(ctx, fn):
    ref = fn()                      # per-slice launches (the classic kernels)
    ctx.set_pass_kernels(ENGINE)
    try:
        got = fn()                  # one persistent launch per batch
    finally:
        ctx.set_pass_kernels(0)
    return got, ref


@pytest.mark.parametrize("n,nconf", [(128, 3), (256, 5), (512, 3), (1024, 2), (2048, 1)])
def test_cbed_engine_agrees(ctx, n, nconf):
    p, at = cases.cbed_small(n=n, cells=(3, 3, 5), nconf=nconf)
    sim = cb.MulSimulator(ctx=ctx)
    a, b = _both(ctx, lambda: sim.executionCBED(p, at).image_intensity)
    assert rel_l2(a, b) <= TOL_SAME


def test_cbed_engine_matches_oracle(ctx):
    p, at = cases.cbed_small(n=256, nconf=3)
    ctx.set_pass_kernels(ENGINE)
    out = cb.MulSimulator(ctx=ctx).executionCBED(p, at)
    ctx.set_pass_kernels(0)
    assert rel_l2(out.image_intensity, orc.simulate_cbed(p, at)) < TOL_ORACLE


@pytest.mark.parametrize("kind", ["hrtem", "ed", "hrtem_tilted", "hrtem_wave"])
def test_plane_wave_engine(ctx, kind):
    if kind == "ed":
        p, at = cases.ed_small(n=256, nconf=2)
    elif kind == "hrtem_wave":
        p, at = cases.hrtem_small(n=256, nconf=2, record=abi.MS_RECORD_WAVE)
    else:
        p, at = cases.hrtem_small(n=256, nconf=2)
    if kind == "hrtem_tilted":
        p.theta, p.phi = 0.006, 0.7
        p.iw_type = abi.MS_IW_PLANE_TILTED
    sim = cb.MulSimulator(ctx=ctx)
    if kind == "hrtem_wave":
        f = lambda: (lambda o: np.stack([o.image_real, o.image_imag]))(sim.executionTEM(p, at))  # noqa: E731
    else:
        f = lambda: sim.executionTEM(p, at).image_intensity  # noqa: E731
    a, b = _both(ctx, f)
    assert rel_l2(a, b) <= TOL_SAME
    if kind != "hrtem_wave":
        assert rel_l2(a, orc.simulate_tem(p, at)) < TOL_ORACLE


@pytest.mark.parametrize("batch,scan", [(8, (6, 5)), (0, (3, 2))])
def test_stem_engine(ctx, batch, scan):
    p, at = cases.stem_small(n=256, scan=scan, nconf=2, batch=batch)
    sim = cb.MulSimulator(ctx=ctx)
    a, b = _both(ctx, lambda: sim.executionSTEM(p, at).stem_intensity)
    assert rel_l2(a, b) <= TOL_SAME
    assert rel_l2(a, orc.simulate_stem(p, at)) < TOL_ORACLE


def test_stem_engine_more_waves_than_blocks(ctx):
    """272 probes at 128^2 in batches of 256 and 16: the full batch has more column items per slice
    than the launch has resident blocks."""
    p, at = cases.stem_small(n=128, scan=(17, 16), nconf=1, batch=256)
    sim = cb.MulSimulator(ctx=ctx)
    a, b = _both(ctx, lambda: sim.executionSTEM(p, at).stem_intensity)
    assert rel_l2(a, b) <= TOL_SAME


def test_uneven_batch_engine(ctx):
    jobs = [wl.cbed_si(cells=(2, 2, 3), n=256, nconf=2, seed=s) for s in (1, 2)]
    jobs.append(wl.cbed_si(cells=(2, 2, 5), n=128, nconf=1, seed=3))
    jobs.append(wl.cbed_si(cells=(2, 2, 9), n=128, nconf=2, seed=6))
    jobs.append(wl.cbed_si(cells=(2, 2, 4), n=512, nconf=2, seed=4))
    jobs.append(wl.cbed_si(cells=(2, 2, 2), n=1024, nconf=1, seed=5))
    # a rectangular grid: its group runs in the per-slice kernels beside the engine groups
    p, at = wl.cbed_si(cells=(2, 2, 3), n=256, nconf=1, seed=7)
    p.ny = 128
    p.ly = p.ly / 2
    jobs.append((p, at))
    sim = cb.MulSimulator(ctx=ctx)
    ctx.set_pass_kernels(PER_SLICE)
    outs_ref, _ = sim.executionMany(jobs)
    ctx.set_pass_kernels(ENGINE)
    try:
        outs, lat = sim.executionMany(jobs)
    finally:
        ctx.set_pass_kernels(0)
    assert np.all(np.isfinite(lat)) and np.all(lat > 0)
    for o, r in zip(outs, outs_ref):
        assert rel_l2(o.image_intensity, r.image_intensity) <= TOL_SAME
    for i in (2, 6):
        assert rel_l2(outs[i].image_intensity, orc.simulate_cbed(*jobs[i])) < TOL_ORACLE
    # the 128^2 group: the instance with fewer slices is done first
    assert outs[2].n_slices < outs[3].n_slices
    assert lat[2] <= lat[3]


def test_uneven_batch_default_is_the_engine(ctx):
    """By default the uneven batch runs its square grid groups in the engine: identical to form 2."""
    jobs = [wl.cbed_si(cells=(2, 2, 3), n=256, nconf=2, seed=s) for s in (1, 2)]
    jobs.append(wl.cbed_si(cells=(2, 2, 5), n=512, nconf=1, seed=3))
    sim = cb.MulSimulator(ctx=ctx)
    a = [o.image_intensity for o in sim.executionMany(jobs)[0]]
    ctx.set_pass_kernels(ENGINE)
    try:
        b = [o.image_intensity for o in sim.executionMany(jobs)[0]]
    finally:
        ctx.set_pass_kernels(0)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_engine_wait_runs_out_and_context_recovers(ctx):
    """With MS_INJECT_WAIT_TIMEOUT the first wave's column items wait for a row item that no block
    counts; the wait runs out after about a millisecond, the blocks stop, and the call reports
    MS_ERR_TIMEOUT.  The same context then runs the engine normally."""
    p, at = cases.cbed_small(n=256, nconf=2)
    sim = cb.MulSimulator(ctx=ctx)
    ctx.set_pass_kernels(ENGINE)
    try:
        ctx.set_fault_injection(abi.MS_INJECT_WAIT_TIMEOUT)
        with pytest.raises(cb.MsError) as e:
            sim.executionCBED(p, at)
        assert e.value.status == abi.MS_ERR_TIMEOUT
        ctx.set_fault_injection(abi.MS_INJECT_NONE)
        out = sim.executionCBED(p, at)
    finally:
        ctx.set_pass_kernels(0)
    assert rel_l2(out.image_intensity, orc.simulate_cbed(p, at)) < TOL_ORACLE
