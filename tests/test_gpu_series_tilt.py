"""Defocus series and beam tilt against the FP64 oracle, through the C ABI.

* Defocus series (ms_simulate_tem_defocus_series; apply_CTF_kernel_batch,
  device_kernels.cuh:469-503): one multislice run imaged at several objective-lens
  defocus values.  Each image within relative L2 1e-5 of the oracle and equal to a
  separate HRTEM call at that defocus.
* Beam tilt theta != 0: the tilted propagator |g - g0|^2 (gen_propagator_kernel,
  device_kernels.cuh:215-234, g0 = gx_0/gy_0 of multislice_params_dev.cuh:201-208) in
  HRTEM, CBED, STEM and the thickness series, and the tilted plane wave of
  Incident_Wave::apply_beam_tilt (incident_wave.cuh:72-78, exp_r_factor_2d,
  device_kernels.cuh:519-533) selected with iw_type MS_IW_PLANE_TILTED.
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
DEFOCI = [-150.0, -40.0, 0.0, 35.0, 120.0]


@pytest.mark.parametrize("nconf", [1, 2])
def test_defocus_series_matches_oracle(ctx, nconf):
    p, at = cases.hrtem_small(nconf=nconf)
    out = cb.MulSimulator(ctx=ctx).executionTEMDefocusSeries(p, at, DEFOCI)
    ref = orc.simulate_tem_series(p, at, DEFOCI)
    assert out.image_intensity.shape == (len(DEFOCI), p.ny, p.nx)
    for i in range(len(DEFOCI)):
        assert rel_l2(out.image_intensity[i], ref[i]) < TOL, DEFOCI[i]


def test_defocus_series_wave_record(ctx):
    p, at = cases.hrtem_small(nconf=2, record=abi.MS_RECORD_WAVE)
    out = cb.MulSimulator(ctx=ctx).executionTEMDefocusSeries(p, at, DEFOCI[:3])
    re, im = orc.simulate_tem_series(p, at, DEFOCI[:3])
    for i in range(3):
        assert rel_l2(out.image_real[i] + 1j * out.image_imag[i], re[i] + 1j * im[i]) < TOL


def test_defocus_series_equals_single_images(ctx):
    """Each image of the series equals an HRTEM call with the objective lens at C10 + df."""
    p, at = cases.hrtem_small(nconf=2)
    sim = cb.MulSimulator(ctx=ctx)
    ser = sim.executionTEMDefocusSeries(p, at, DEFOCI)
    for i, df in enumerate(DEFOCI):
        q = p.copy()
        q.obj_lens.c10 = p.obj_lens.c10 + df
        single = sim.executionTEM(q, at).image_intensity
        assert rel_l2(ser.image_intensity[i], single) < 1e-6, df


def test_defocus_series_rejects_other_modes(ctx):
    sim = cb.MulSimulator(ctx=ctx)
    p, at = cases.hrtem_small()
    p.illumination_model = abi.MS_ILLUM_PARTIAL
    with pytest.raises(cb.MsError):
        sim.executionTEMDefocusSeries(p, at, DEFOCI)
    p, at = cases.cbed_small()
    with pytest.raises(cb.MsError):
        sim.executionTEMDefocusSeries(p, at, DEFOCI)


def _tilt(p, theta=0.006, phi=0.7):
    p.theta = theta
    p.phi = phi
    return p


@pytest.mark.parametrize("iw", [abi.MS_IW_PLANE, abi.MS_IW_PLANE_TILTED])
def test_hrtem_tilted(ctx, iw):
    p, at = cases.hrtem_small(nconf=2)
    _tilt(p)
    p.iw_type = iw
    out = cb.MulSimulator(ctx=ctx).executionTEM(p, at)
    ref = orc.simulate_tem(p, at)
    assert rel_l2(out.image_intensity, ref) < TOL


def test_tilted_incident_wave_differs_from_plane(ctx):
    """The tilted plane wave is a different illumination from the plain plane wave under the same
    tilted propagator (the carrier moves the spectrum by g0)."""
    p, at = cases.ed_small(nconf=1)
    _tilt(p, theta=0.01)
    a = cb.MulSimulator(ctx=ctx).executionTEM(p, at).image_intensity
    p.iw_type = abi.MS_IW_PLANE_TILTED
    b = cb.MulSimulator(ctx=ctx).executionTEM(p, at).image_intensity
    assert rel_l2(b, orc.simulate_tem(p, at)) < TOL
    assert rel_l2(a, b) > 1e-2


def test_cbed_tilted(ctx):
    p, at = cases.cbed_small(nconf=2)
    _tilt(p, theta=0.004, phi=-1.1)
    out = cb.MulSimulator(ctx=ctx).executionCBED(p, at)
    assert rel_l2(out.image_intensity, orc.simulate_cbed(p, at)) < TOL


def test_stem_tilted(ctx):
    p, at = cases.stem_small(nconf=1)
    _tilt(p, theta=0.005, phi=0.3)
    out = cb.MulSimulator(ctx=ctx).executionSTEM(p, at)
    assert rel_l2(out.stem_intensity, orc.simulate_stem(p, at)) < TOL


@pytest.mark.parametrize("iw", [abi.MS_IW_PLANE, abi.MS_IW_PLANE_TILTED])
def test_thickness_tilted(ctx, iw):
    p, at = cases.thickness_small()
    _tilt(p, theta=0.007, phi=2.0)
    p.iw_type = iw
    out = cb.ThicknessSimulator(ctx=ctx).run(p, at)
    assert rel_l2(out.thickness_frames, orc.simulate_thickness(p, at)) < TOL


def test_stem_general_scan_crop(ctx):
    """The reference's general scan (run_STEM_general_simu, scan_simulator.cuh:115-183): the
    12.8 A grid is a window that follows the probe over a 31 A specimen; each window holds the
    displaced atoms within 2 A of it, shifted in, with the probe at its centre.  One position lies
    off the specimen: its window is empty and records the unscattered probe (blank intensity)."""
    from cudaem_b200 import workloads as wl
    p, at = wl.stem_sto(cells=(8, 8, 3), n=128, nconf=2, scan=(3, 2), step=1.3)
    p.lx = p.ly = 12.8
    p.scan_x0 = 9.0
    p.scan_y0 = 14.0
    p.set_detectors([(0.0, 0.010), (0.030, 0.060)])
    p.cond_lens.outer_aper_ang = 0.015
    p.exec_mode = abi.MS_EXEC_GENERAL
    out = cb.MulSimulator(ctx=ctx).executionSTEM(p, at)
    ref = orc.simulate_stem(p, at)
    assert rel_l2(out.stem_intensity, ref) < TOL
    q = p.copy()
    q.scan_nx, q.scan_ny = 1, 1
    q.scan_x0 = q.scan_y0 = -40.0          # far off the specimen: an empty window
    e = cb.MulSimulator(ctx=ctx).executionSTEM(q, at).stem_intensity
    eo = orc.simulate_stem(q, at)
    assert e[0, 0, 0] > 0 and abs(e[0, 0, 0] - eo[0, 0, 0]) <= 1e-6 * eo[0, 0, 0]
    assert e[1, 0, 0] == 0.0 and eo[1, 0, 0] == 0.0


def test_stem_general_scan_matches_window_simulation(ctx):
    """One general-scan position equals a batched STEM simulation of the cropped, shifted atoms
    with the probe at the window centre."""
    from cudaem_b200 import workloads as wl
    p, at = wl.stem_sto(cells=(6, 6, 2), n=128, nconf=1, scan=(1, 1))
    p.phonon_model = abi.MS_PHONON_STILL
    p.lx = p.ly = 12.8
    p.scan_x0, p.scan_y0 = 11.3, 10.2
    p.set_detectors([(0.0, 0.010), (0.030, 0.060)])
    p.exec_mode = abi.MS_EXEC_GENERAL
    g = cb.MulSimulator(ctx=ctx).executionSTEM(p, at).stem_intensity
    xs, ys = np.float32(p.scan_x0 - 6.4), np.float32(p.scan_y0 - 6.4)
    keep = (at.x >= xs - np.float32(2)) & (at.x <= xs + np.float32(12.8) + np.float32(2)) & \
           (at.y >= ys - np.float32(2)) & (at.y <= ys + np.float32(12.8) + np.float32(2))
    cut = cb.Atoms(Z=at.Z[keep], x=at.x[keep] - xs, y=at.y[keep] - ys, z=at.z[keep], sigma=at.sigma[keep],
                   occ=at.occ[keep])
    q = p.copy()
    q.exec_mode = abi.MS_EXEC_BATCHED
    q.scan_x0, q.scan_y0 = 6.4, 6.4
    w = cb.MulSimulator(ctx=ctx).executionSTEM(q, cut).stem_intensity
    assert rel_l2(g, w) < 1e-6
