"""Named workloads: the synthetic crystal simulations the engine is measured on.

Each function returns (MultisliceParams, Atoms).  Specimens are built from
their unit cells (SrTiO3 perovskite a = 3.905 A, Si diamond a = 5.431 A,
[001]), with Gaussian frozen-phonon displacements drawn from the seed; the
grid box equals the supercell, so the sampling is box / pixels.
"""
from __future__ import annotations

import numpy as np

from . import MultisliceParams, _abi as abi, si_diamond, srtio3

STO_A = 3.905
SI_A = 5.431


def hrtem_sto(cells=(10, 10, 20), n=512, sigma=0.08, nconf=1, seed=42):
    """Plain HRTEM on a plane wave: SrTiO3 [001], 512^2, slices of a/2, 200 kV,
    objective lens defocus -10 nm, Cs 1 mm, 20 mrad aperture."""
    at = srtio3(*cells, sigma=sigma)
    L = cells[0] * STO_A
    p = MultisliceParams(simulation_type=abi.MS_SIM_HRTEM, nx=n, ny=n, lx=L, ly=cells[1] * STO_A, dz=STO_A / 2,
                         E0=200.0, phonon_model=abi.MS_PHONON_FROZEN, pn_nconf=nconf, pn_seed=seed)
    p.obj_lens.c10 = -100.0
    p.obj_lens.c30 = 1.0e7
    p.obj_lens.outer_aper_ang = 0.020
    return p, at


def cbed_si(cells=(16, 16, 60), n=1024, sigma=0.075, nconf=8, seed=42):
    """Batched CBED with frozen phonons: Si [001], 1024^2, slices of 1.358 A, 300 kV,
    20 mrad probe centred on the box."""
    at = si_diamond(*cells, sigma=sigma)
    L = cells[0] * SI_A
    p = MultisliceParams(simulation_type=abi.MS_SIM_CBED, nx=n, ny=n, lx=L, ly=cells[1] * SI_A, dz=1.358,
                         E0=300.0, phonon_model=abi.MS_PHONON_FROZEN, pn_nconf=nconf, pn_seed=seed,
                         iw_x=L / 2, iw_y=cells[1] * SI_A / 2)
    p.cond_lens.outer_aper_ang = 0.020
    return p, at


def stem_sto(cells=(16, 16, 25), n=1024, sigma=0.08, nconf=10, scan=(64, 64), step=0.2, seed=42, batch=0):
    """Batched STEM ADF: SrTiO3 [001], 1024^2, slices of a/2, 200 kV, 22 mrad probe,
    ADF 60-200 mrad, a scan of 0.2 A steps centred on the box."""
    at = srtio3(*cells, sigma=sigma)
    L = cells[0] * STO_A
    p = MultisliceParams(simulation_type=abi.MS_SIM_STEM, nx=n, ny=n, lx=L, ly=cells[1] * STO_A, dz=STO_A / 2,
                         E0=200.0, phonon_model=abi.MS_PHONON_FROZEN, pn_nconf=nconf, pn_seed=seed,
                         scan_nx=scan[0], scan_ny=scan[1], scan_dx=step, scan_dy=step,
                         scan_x0=L / 2 - scan[0] * step / 2, scan_y0=cells[1] * STO_A / 2 - scan[1] * step / 2,
                         probe_batch=batch)
    p.cond_lens.outer_aper_ang = 0.022
    p.set_detectors([(0.060, 0.200)])
    return p, at


def adjoint_sto(cells=(10, 10, 40), n=512, n_probe=16, seed=42):
    """Differentiable STEM: SrTiO3 [001] 10x10x40 cells, 512^2, 80 slices, 16 probes, 200 kV,
    22 mrad, ADF 60-200 mrad.  Returns (params, atoms, probe positions)."""
    at = srtio3(*cells, sigma=0.08)
    L = cells[0] * STO_A
    p = MultisliceParams(simulation_type=abi.MS_SIM_STEM, nx=n, ny=n, lx=L, ly=cells[1] * STO_A, dz=STO_A / 2,
                         E0=200.0, phonon_model=abi.MS_PHONON_STILL, pn_seed=seed, scan_nx=4, scan_ny=4,
                         ckpt_interval=8)
    p.cond_lens.outer_aper_ang = 0.022
    p.cond_lens.c10 = -20.0
    p.cond_lens.c30 = 1.0e4
    p.set_detectors([(0.060, 0.200)])
    rng = np.random.default_rng(seed)
    xy = L / 2 + rng.uniform(-STO_A, STO_A, size=(n_probe, 2))
    return p, at, xy


def uneven_mix(n_sim=64, seed=42):
    """64 simulations drawn from the seed: grid 256^2..2048^2, 10-200 slices of SrTiO3 or Si,
    80-300 kV, 10-30 mrad probes, per-simulation phonon seeds (CBED, one configuration each)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_sim):
        n = int(rng.choice([256, 512, 1024, 2048]))
        sto = bool(rng.integers(0, 2))
        nsl = int(rng.integers(10, 201))
        E0 = float(rng.uniform(80, 300))
        conv = float(rng.uniform(0.010, 0.030))
        a = STO_A if sto else SI_A
        per_cell = 2 if sto else 4
        nc = max(1, int(np.ceil(nsl / per_cell)))
        dx_target = 0.08
        ncell = max(2, int(round(n * dx_target / a)))
        at = srtio3(ncell, ncell, nc, sigma=0.08) if sto else si_diamond(ncell, ncell, nc, sigma=0.075)
        L = ncell * a
        p = MultisliceParams(simulation_type=abi.MS_SIM_CBED, nx=n, ny=n, lx=L, ly=L, dz=a / per_cell, E0=E0,
                             phonon_model=abi.MS_PHONON_FROZEN, pn_nconf=1, pn_seed=int(rng.integers(1, 1 << 30)),
                             iw_x=L / 2, iw_y=L / 2)
        p.cond_lens.outer_aper_ang = conv
        out.append((p, at))
    return out
