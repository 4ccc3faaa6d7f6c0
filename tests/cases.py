"""Small versions of the measured workloads, sized so the FP64 oracle finishes in seconds."""
from __future__ import annotations

import numpy as np

import cudaem_b200 as cb
from cudaem_b200 import _abi as abi
from cudaem_b200 import workloads as wl


def hrtem_small(n=128, cells=(5, 5, 4), nconf=1, record=abi.MS_RECORD_INTENSITY, wrap=0):
    p, at = wl.hrtem_sto(cells=cells, n=n, nconf=nconf)
    p.data_record = record
    p.pot_wrap = wrap
    return p, at


def ed_small(n=128, nconf=2, record=abi.MS_RECORD_INTENSITY):
    p, at = wl.hrtem_sto(cells=(5, 5, 4), n=n, nconf=nconf)
    p.simulation_type = abi.MS_SIM_ED
    p.data_record = record
    return p, at


def cbed_small(n=128, cells=(2, 2, 4), nconf=2, wrap=0):
    p, at = wl.cbed_si(cells=cells, n=n, nconf=nconf)
    p.pot_wrap = wrap
    return p, at


def stem_small(n=128, cells=(4, 4, 3), nconf=2, scan=(3, 2), plain=False, batch=0):
    p, at = wl.stem_sto(cells=cells, n=n, nconf=nconf, scan=scan, step=0.4, batch=batch)
    # detectors inside this small grid's band limit: bright field and an annulus
    p.set_detectors([(0.0, 0.010), (0.030, 0.060)])
    if plain:
        p.exec_mode = abi.MS_EXEC_PLAIN
    return p, at


def thickness_small(n=128, nconf=1):
    p, at = wl.hrtem_sto(cells=(4, 4, 3), n=n, nconf=nconf)
    p.set_detectors([(0.0, 0.020), (0.0, 0.040)])
    p.thick_det = 1
    return p, at


def random_phase_slices(p, S, seed=0, amp=0.6):
    rng = np.random.default_rng(seed)
    V = rng.uniform(0, amp, size=(S, p.ny, p.nx)).astype(np.float32)
    return V
