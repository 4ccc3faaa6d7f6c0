"""The adjoint (ms_stem_backward) against the FP64 oracle's adjoint and finite differences.

Loss L = sum over probes and detectors of (I - target)^2 on caller phase slices V.
Bounds: loss relative error <= 1e-4 (the targets sit 5 % away from the intensities, so
the residuals carry the FP32 forward error magnified about 20 times); dL/dV relative L2
<= 1e-4 and dL/dC10, dL/dC30 relative error <= 1e-4, against the oracle's adjoint and
against central finite differences (h = 1e-3 relative).
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import cases  # noqa: E402
from conftest import rel_l2  # noqa: E402
from oracle import oracle as orc  # noqa: E402

pytestmark = pytest.mark.gpu

TOL_LOSS = 1e-4
TOL_GRAD = 1e-4


def _problem(n, S, n_probe, seed, ckpt, batch=0):
    p, _ = cases.stem_small(n=n)
    p.set_detectors([(0.0, 0.012), (0.025, 0.06)])
    p.cond_lens.c10 = -30.0
    p.cond_lens.c30 = 2.0e4
    p.ckpt_interval = ckpt
    p.probe_batch = batch
    V = cases.random_phase_slices(p, S, seed=seed, amp=0.4)
    rng = np.random.default_rng(seed)
    xy = p.lx / 2 + rng.uniform(-1.5, 1.5, size=(n_probe, 2))
    z0 = 0.7
    I0 = orc.stem_forward_potential(p, V, z0, xy)
    T = (I0 * (1 + 0.05 * rng.standard_normal(I0.shape))).astype(np.float32)
    return p, V, xy, z0, T


@pytest.mark.parametrize("n,S,n_probe,ckpt,batch", [
    (128, 7, 5, 3, 2),     # three segments, three probe batches (the last one partial)
    (128, 4, 1, 1, 0),     # a checkpoint at every slice
    (256, 9, 3, 4, 0),     # a one-slice last segment
    (256, 6, 2, 8, 0),     # one segment: no recomputation
])
def test_backward_matches_oracle(ctx, n, S, n_probe, ckpt, batch):
    p, V, xy, z0, T = _problem(n, S, n_probe, seed=n + S, ckpt=ckpt, batch=batch)
    loss, gV, g10, g30 = ctx.stem_backward(p, V, z0, xy, T)
    lo, gVo, g10o, g30o = orc.stem_backward(p, V, z0, xy, T)
    assert abs(loss - lo) / lo < TOL_LOSS
    assert rel_l2(gV, gVo) < TOL_GRAD
    assert abs(g10 - g10o) / abs(g10o) < TOL_GRAD
    assert abs(g30 - g30o) / abs(g30o) < TOL_GRAD


def test_checkpoint_interval_does_not_change_gradients(ctx):
    p, V, xy, z0, T = _problem(128, 10, 3, seed=5, ckpt=1)
    ref = ctx.stem_backward(p, V, z0, xy, T)
    for k in (2, 3, 10, 16):
        p.ckpt_interval = k
        got = ctx.stem_backward(p, V, z0, xy, T)
        assert abs(got[0] - ref[0]) <= 1e-12 * abs(ref[0])
        # the segments are recomputed with the same kernels on the same inputs and dL/dV is summed
        # over probes in a fixed order, so the gradient does not depend on the checkpoint spacing
        assert np.array_equal(got[1], ref[1])
        assert abs(got[2] - ref[2]) <= 1e-9 * abs(ref[2])
        assert abs(got[3] - ref[3]) <= 1e-9 * abs(ref[3])


def test_backward_is_reproducible(ctx):
    """Two calls on the same inputs give the same bits (dL/dV is summed over probes in a fixed
    order, not with atomic adds)."""
    p, V, xy, z0, T = _problem(256, 6, 9, seed=31, ckpt=2, batch=4)
    a = ctx.stem_backward(p, V, z0, xy, T)
    b = ctx.stem_backward(p, V, z0, xy, T)
    assert a[0] == b[0] and a[2] == b[2] and a[3] == b[3]
    assert np.array_equal(a[1], b[1])


def test_backward_against_finite_differences(ctx):
    """GPU gradients against central differences of the FP64 forward model (h = 1e-3 relative)."""
    p, V, xy, z0, T = _problem(128, 3, 2, seed=17, ckpt=2)
    loss, gV, g10, g30 = ctx.stem_backward(p, V, z0, xy, T)

    def L(Vx, q=p):
        I = orc.stem_forward_potential(q, Vx, z0, xy)
        return float(np.sum((I - T.astype(np.float64)) ** 2))

    rng = np.random.default_rng(3)
    big = np.argsort(np.abs(gV).ravel())[-64:]
    picks = rng.choice(big, size=8, replace=False)
    fd, an = [], []
    for idx in picks:
        s, iy, ix = np.unravel_index(idx, V.shape)
        h = 1e-3 * max(abs(float(V[s, iy, ix])), 1.0)
        Vp, Vm = V.copy(), V.copy()
        Vp[s, iy, ix] += h
        Vm[s, iy, ix] -= h
        dp = float(Vp[s, iy, ix]) - float(V[s, iy, ix])
        dm = float(V[s, iy, ix]) - float(Vm[s, iy, ix])
        fd.append((L(Vp) - L(Vm)) / (dp + dm))
        an.append(gV[s, iy, ix])
    assert rel_l2(np.array(an), np.array(fd)) < TOL_GRAD
    for name, g in (("c10", g10), ("c30", g30)):
        h = 1e-3 * abs(getattr(p.cond_lens, name))
        qp, qm = p.copy(), p.copy()
        setattr(qp.cond_lens, name, getattr(p.cond_lens, name) + h)
        setattr(qm.cond_lens, name, getattr(p.cond_lens, name) - h)
        fdv = (L(V, qp) - L(V, qm)) / (2 * h)
        assert abs(fdv - g) / abs(fdv) < TOL_GRAD


def test_backward_differentiable_stem_shape(ctx):
    """The differentiable-STEM workload's shape (SrTiO3 10x10 cells, 512^2, 80 slices of
    1.9525 A, 200 kV, 22 mrad, checkpoints every 8 slices) on 4 of its 16 probes, with
    targets from potentials perturbed by 1 % Gaussian noise."""
    from cudaem_b200 import workloads as wl
    p, at, xy = wl.adjoint_sto(n_probe=4)
    V = ctx.projected_potential(p, at, conf=0)
    assert V.shape[0] == 80
    z0 = 0.5 * p.dz
    rng = np.random.default_rng(7)
    Vt = (V + 0.01 * np.abs(V) * rng.standard_normal(V.shape)).astype(np.float32)
    T = ctx.stem_forward_potential(p, Vt, z0, xy)
    loss, gV, g10, g30 = ctx.stem_backward(p, V, z0, xy, T)
    lo, gVo, g10o, g30o = orc.stem_backward(p, V, z0, xy, T)
    assert abs(loss - lo) / lo < 1e-3          # residuals are ~1e-3 of I: the forward error magnified
    assert rel_l2(gV, gVo) < 1e-3
    assert abs(g10 - g10o) / abs(g10o) < 1e-3
    assert abs(g30 - g30o) / abs(g30o) < 1e-3


def test_backward_finite_differences_differentiable_stem_shape(ctx):
    """The differentiable-STEM check at its own shape: SrTiO3 10x10x40 cells, 512^2, 80 slices,
    checkpoints every 8, targets simulated from potentials perturbed by Gaussian noise at 1 % of
    |V|.  GPU gradients against central differences (h = 1e-3 relative) of the FP64 forward loss
    on 64 potential pixels drawn uniformly over all 80 x 512^2, and on C10 and Cs.  Four of the
    workload's 16 probes, so that the 132 FP64 forward evaluations finish in about a minute."""
    from cudaem_b200 import workloads as wl
    p, at, xy = wl.adjoint_sto(n_probe=4)
    V = ctx.projected_potential(p, at, conf=0)
    assert V.shape == (80, 512, 512) and p.ckpt_interval == 8
    z0 = 0.5 * p.dz
    rng = np.random.default_rng(11)
    Vt = (V + 0.01 * np.abs(V) * rng.standard_normal(V.shape)).astype(np.float32)
    T = orc.stem_forward_potential(p, Vt, z0, xy).astype(np.float32)
    loss, gV, g10, g30 = ctx.stem_backward(p, V, z0, xy, T)
    idx = rng.choice(V.size, size=64, replace=False)
    h = 1e-3 * np.maximum(np.abs(V.ravel()[idx]).astype(np.float64), 1e-3)
    fd, f10, f30 = orc.stem_loss_fd(p, V, z0, xy, T, idx, h, 1e-3 * abs(p.cond_lens.c10),
                                    1e-3 * abs(p.cond_lens.c30))
    an = gV.ravel()[idx].astype(np.float64)
    e_pix = rel_l2(an, fd)
    e10, e30 = abs(g10 - f10) / abs(f10), abs(g30 - f30) / abs(f30)
    print(f"differentiable STEM 512^2 x 80 slices: dL/dV on 64 random pixels rel L2 {e_pix:.2e}, "
          f"dL/dC10 {e10:.2e}, dL/dCs {e30:.2e}")
    assert e_pix < TOL_GRAD
    assert e10 < TOL_GRAD
    assert e30 < TOL_GRAD
