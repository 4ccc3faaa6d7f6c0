"""The persistent pipelined slice passes against the classic kernels.

Both kernel forms run the same transform code on the same data; only the scheduling
(persistent blocks, prefetching) and the compiler's contraction of a few products differ,
so every output agrees to float rounding (relative L2 <= 1e-6; the adjoint's loss and
gradients, which carry residuals 30x smaller than the intensities, to 1e-4).  Covered:
square grids 128..2048 (2048 falls back to the classic form), a rectangular grid, more waves than
resident blocks, phonon configurations with different slice counts (items skipped mid-pass), the
row pass on a transmission store at 512 and 1024 points (CBED, thickness series, uneven batch),
the adjoint's conjugate propagator step, and the uneven batch's per-wave potential and
propagator tables.
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

pytestmark = pytest.mark.gpu


TOL = 1e-6


def _close(a, b):
    return rel_l2(a, b) <= TOL


def _both(ctx, fn, ref_variant=0):
    ctx.set_pass_kernels(ref_variant)
    ref = fn()                      # the reference form (classic kernels)
    ctx.set_pass_kernels(1)
    try:
        got = fn()                  # persistent pipelined
    finally:
        ctx.set_pass_kernels(0)
    return got, ref


@pytest.mark.parametrize("nx,ny,n_probe", [(128, 128, 3), (256, 256, 5), (512, 512, 2), (1024, 1024, 2),
                                           (2048, 2048, 1), (256, 512, 3), (512, 128, 2), (256, 256, 301)])
def test_slice_loop_agree(ctx, nx, ny, n_probe):
    p, _ = cases.stem_small(n=128)
    p.nx, p.ny = nx, ny
    p.lx, p.ly = nx * 0.1, ny * 0.1
    p.probe_batch = 256
    V = cases.random_phase_slices(p, 4, seed=nx + ny)
    rng = np.random.default_rng(nx)
    xy = np.stack([p.lx / 2 + rng.uniform(-1, 1, n_probe), p.ly / 2 + rng.uniform(-1, 1, n_probe)], axis=1)
    a, b = _both(ctx, lambda: ctx.stem_forward_potential(p, V, 0.5, xy))
    assert _close(a, b)


@pytest.mark.parametrize("n,nconf", [(256, 5), (512, 3), (1024, 2)])
def test_cbed_phonons_agree(ctx, n, nconf):
    # 512 and 1024 run the row pass on the transmission store in the 12-warp double-buffered form
    p, at = cases.cbed_small(n=n, cells=(3, 3, 5), nconf=nconf)
    sim = cb.MulSimulator(ctx=ctx)
    a, b = _both(ctx, lambda: sim.executionCBED(p, at).image_intensity)
    assert _close(a, b)


@pytest.mark.parametrize("n", [512, 1024])
def test_thickness_agree(ctx, n):
    p, at = cases.thickness_small(n=n)
    sim = cb.ThicknessSimulator(ctx=ctx)
    a, b = _both(ctx, lambda: sim.run(p, at).thickness_frames)
    assert _close(a, b)


def test_adjoint_agree(ctx):
    p, _ = cases.stem_small(n=256)
    p.ckpt_interval = 3
    V = cases.random_phase_slices(p, 7, seed=2, amp=0.4)
    xy = np.array([[p.lx / 2, p.ly / 2], [p.lx / 2 + 0.6, p.ly / 2 - 0.4]])
    T = ctx.stem_forward_potential(p, V, 0.3, xy) * np.float32(1.03)
    a, b = _both(ctx, lambda: ctx.stem_backward(p, V, 0.3, xy, T))
    tol = 1e-4
    assert abs(a[0] - b[0]) <= tol * abs(b[0])
    assert abs(a[2] - b[2]) <= tol * abs(b[2]) and abs(a[3] - b[3]) <= tol * abs(b[3])
    assert rel_l2(a[1], b[1]) <= tol


def test_uneven_batch_agree(ctx):
    jobs = [wl.cbed_si(cells=(2, 2, 3), n=256, nconf=2, seed=s) for s in (1, 2)]
    jobs.append(wl.cbed_si(cells=(2, 2, 5), n=128, nconf=1, seed=3))
    jobs.append(wl.cbed_si(cells=(2, 2, 4), n=512, nconf=2, seed=4))
    jobs.append(wl.cbed_si(cells=(2, 2, 2), n=1024, nconf=1, seed=5))
    sim = cb.MulSimulator(ctx=ctx)
    # the per-slice classic kernels as the reference (the default runs uneven batches in the engine)
    a, b = _both(ctx, lambda: [o.image_intensity for o in sim.executionMany(jobs)[0]], ref_variant=3)
    for x, y in zip(a, b):
        assert _close(x, y)
