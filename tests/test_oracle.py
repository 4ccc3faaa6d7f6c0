"""Checks of the FP64 oracle itself (CPU): known answers, physics invariants and
agreement with the independent numpy restatement."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import cases  # noqa: E402
import numpy_twin as tw  # noqa: E402
from conftest import rel_l2  # noqa: E402
from oracle import oracle as orc  # noqa: E402
import cudaem_b200 as cb  # noqa: E402


# relativistic wavelength (A) and interaction constant (rad/(V A)): textbook values
@pytest.mark.parametrize("E0,lam,sig", [(100, 0.037014, 9.2440e-4), (200, 0.025079, 7.2884e-4),
                                        (300, 0.019687, 6.5262e-4)])
def test_physics_known_answers(E0, lam, sig):
    l, s, g = orc.physics(E0)
    assert abs(l - lam) / lam < 5e-5  # table values carry 5 significant digits
    assert abs(s - sig) / sig < 1e-4
    assert abs(g - (1 + E0 / 510.99895)) < 1e-6


def test_det_log_and_gaussian():
    rng = np.random.default_rng(0)
    for s in rng.uniform(1e-12, 1.0, 2000):
        assert abs(orc.det_log(s) - np.log(s)) < 4e-15 * max(1.0, abs(np.log(s)))
    g = np.array([orc.gauss_pair(7, 3, i, 0) for i in range(20000)]).ravel()
    assert abs(g.mean()) < 0.02 and abs(g.var() - 1) < 0.03
    # keyed, not sequential: a different configuration gives an independent draw
    assert orc.gauss_pair(7, 3, 11, 0) != orc.gauss_pair(7, 4, 11, 0)


def test_moliere_projection_known_answer():
    """V_z(R) = 2 sum cl K0(cnl R) and dV_z/dR^2 = -sum cl cnl K1(cnl R)/R for the Yukawa form."""
    from scipy.special import k0, k1
    p, _ = cases.hrtem_small()
    a0, ke, tf = 0.529177210903, 14.399645478425668, 0.88534138
    for Z in (8, 14, 22, 38):
        aTF = tf * a0 * Z ** (-1 / 3)
        for R in (0.01, 0.05, 0.3, 1.0, 2.9):
            Vz, dV = orc.projected(p, Z, R)
            Va = sum(2 * ke * Z * a * k0(b / aTF * R) for a, b in zip((0.35, 0.55, 0.1), (0.3, 1.2, 6.0)))
            dVa = sum(-ke * Z * a * (b / aTF) * k1(b / aTF * R) / R for a, b in zip((0.35, 0.55, 0.1), (0.3, 1.2, 6.0)))
            assert abs(Vz - Va) / Va < 1e-10
            assert abs(dV - dVa) / abs(dVa) < 1e-9


def test_gaussian_form_projection():
    """Doyle/Peng form: V(r) = sum cl exp(-cnl r^2) projects to sum cl sqrt(pi/cnl) exp(-cnl R^2)."""
    from cudaem_b200 import _abi as abi
    p, _ = cases.hrtem_small()
    cl, cnl = [3.0, 1.5, 0.4, 0.1], [2.0, 0.7, 0.2, 0.05]
    p.set_element_coefs([(14, abi.MS_POT_DOYLE_0_4, cl, cnl)])
    for R in (0.02, 0.4, 1.7):
        Vz, _ = orc.projected(p, 14, R)
        Va = sum(c * np.sqrt(np.pi / k) * np.exp(-k * R * R) for c, k in zip(cl, cnl))
        assert abs(Vz - Va) / Va < 1e-10


def test_spline_table_interpolates_projection():
    p, _ = cases.hrtem_small()
    R2, c0, c1, c2, c3, rmax = orc.spline(p, 22)
    # Hermite cubic reproduces node values and is accurate between nodes away from the taper
    for i in (3, 40, 80):
        d = R2[i + 1] - R2[i]
        x = R2[i] + 0.37 * d
        v = ((c3[i] * (x - R2[i]) + c2[i]) * (x - R2[i]) + c1[i]) * (x - R2[i]) + c0[i]
        Vz, _ = orc.projected(p, 22, np.sqrt(x))
        assert abs(v - Vz) / Vz < 1e-5
    assert abs(c0[-1]) < 1e-12 * abs(c0[0])  # tapered to zero at R_max


def test_fft_conventions():
    x = np.random.default_rng(1).standard_normal((64, 128)) + 1j * np.random.default_rng(2).standard_normal((64, 128))
    assert np.abs(orc.fft2(x, -1) - np.fft.fft2(x)).max() < 1e-11
    assert np.abs(orc.fft2(x, +1) - np.fft.ifft2(x) * x.size).max() < 1e-11


def test_hrtem_against_numpy_twin():
    p, at = cases.hrtem_small()
    img = orc.simulate_tem(p, at)
    V, _ = orc.potential(p, at, 1)  # the single frozen-phonon configuration is conf 1
    W = tw.multislice(p, V, np.ones((p.ny, p.nx)))
    assert rel_l2(img, np.abs(tw.ctf_image(p, W)) ** 2) < 1e-12


def test_stem_forward_against_numpy_twin():
    p, _ = cases.stem_small(n=128)
    V = cases.random_phase_slices(p, 4, seed=5).astype(np.float64)
    xy = np.array([[7.0, 8.0], [3.5, 9.25]])
    I = orc.stem_forward_potential(p, V.astype(np.float32), 1.3, xy)
    ref = np.array([tw.detect(p, tw.multislice(p, V.astype(np.float32).astype(np.float64),
                                               tw.probe(p, x, y, 1.3))) for x, y in xy])
    assert rel_l2(I, ref) < 1e-12


def test_parseval_and_vacuum_propagation():
    """With no band limit and pure-phase slices the multislice is unitary up to the reference's
    N scaling, and two vacuum steps of dz equal one of 2 dz."""
    p, _ = cases.stem_small(n=128)
    p.bwl = 0
    psi0 = tw.probe(p, 5.0, 6.0, 0.0)
    V = cases.random_phase_slices(p, 5, seed=9).astype(np.float64)
    W = tw.multislice(p, V, psi0)
    assert abs(np.sum(np.abs(W) ** 2) / (p.nx * p.ny * np.sum(np.abs(psi0) ** 2)) - 1) < 1e-12
    q = p.copy()
    q.dz = 2 * p.dz
    P1, P2 = tw.propagator(p), tw.propagator(q)
    N = p.nx * p.ny
    assert np.abs(P1 * P1 * N - P2).max() < 1e-12


def test_weak_phase_object():
    """A single thin slice with a small phase: exit wave = N(1 + i V) to first order."""
    p, _ = cases.hrtem_small()
    V = (1e-4 * np.random.default_rng(3).standard_normal((1, p.ny, p.nx))).astype(np.float32)
    W = tw.multislice(p, V.astype(np.float64), np.ones((p.ny, p.nx)))
    psi = np.fft.ifft2(W)
    assert np.abs(psi - (1 + 1j * V[0])).max() < 1e-7


def test_adjoint_matches_finite_differences():
    """The oracle's adjoint against central differences of its own forward model."""
    p, _ = cases.stem_small(n=128)
    p.set_detectors([(0.0, 0.012), (0.025, 0.06)])
    p.cond_lens.c10 = -30.0
    p.cond_lens.c30 = 2.0e4
    S = 3
    V = cases.random_phase_slices(p, S, seed=11, amp=0.4)
    xy = np.array([[6.0, 7.0], [8.5, 7.25]])
    z0 = 0.7
    I0 = orc.stem_forward_potential(p, V, z0, xy)
    T = (I0 * (1 + 0.05 * np.random.default_rng(4).standard_normal(I0.shape))).astype(np.float32)
    loss, gV, g10, g30 = orc.stem_backward(p, V, z0, xy, T)

    def L(Vx, q=p):
        I = orc.stem_forward_potential(q, Vx, z0, xy)
        return float(np.sum((I - T.astype(np.float64)) ** 2))

    assert abs(L(V) - loss) / loss < 1e-10
    rng = np.random.default_rng(12)
    # pick pixels where the gradient is large so float32 steps resolve it
    flat = np.argsort(np.abs(gV).ravel())[-6:]
    for idx in flat:
        s, iy, ix = np.unravel_index(idx, V.shape)
        h = 2e-3
        Vp, Vm = V.copy(), V.copy()
        Vp[s, iy, ix] += h
        Vm[s, iy, ix] -= h
        dp, dm = float(Vp[s, iy, ix]) - float(V[s, iy, ix]), float(V[s, iy, ix]) - float(Vm[s, iy, ix])
        fd = (L(Vp) - L(Vm)) / (dp + dm)
        assert abs(fd - gV[s, iy, ix]) / abs(gV[s, iy, ix]) < 1e-4
    for name, g in (("c10", g10), ("c30", g30)):
        h = 1e-3 * (abs(getattr(p.cond_lens, name)) or 1.0)
        qp, qm = p.copy(), p.copy()
        setattr(qp.cond_lens, name, getattr(p.cond_lens, name) + h)
        setattr(qm.cond_lens, name, getattr(p.cond_lens, name) - h)
        fd = (L(V, qp) - L(V, qm)) / (2 * h)
        assert abs(fd - g) / abs(g) < 1e-4
    del rng


def test_gauss_hermite_known_answers():
    """Quadrature of the partial-coherence models: exact nodes for n = 2, 3 and exact moments of
    exp(-x^2) (normalised: <x^2> = 1/2, <x^4> = 3/4, <x^6> = 15/8) up to degree 2n-1."""
    x, w = orc.gauss_hermite(2)
    assert np.allclose(np.sort(x), [-np.sqrt(0.5), np.sqrt(0.5)], atol=1e-14) and np.allclose(w, 0.5)
    x, w = orc.gauss_hermite(3)
    assert np.allclose(np.sort(x), [-np.sqrt(1.5), 0.0, np.sqrt(1.5)], atol=1e-14)
    assert np.allclose(w[np.argsort(x)], [1 / 6, 2 / 3, 1 / 6], atol=1e-14)
    for n in (4, 8, 16, 40, 64):
        x, w = orc.gauss_hermite(n)
        assert abs(w.sum() - 1) < 1e-13
        assert abs(np.dot(w, x ** 2) - 0.5) < 1e-12
        assert abs(np.dot(w, x ** 4) - 0.75) < 1e-11
        assert abs(np.dot(w, x ** 6) - 15 / 8) < 1e-10
        assert abs(np.dot(w, x ** 3)) < 1e-12


def test_fine_slicing_integrates_the_projection():
    """Fine slicing splits an atom's potential over the slices whose integration range reaches it:
    the slice-integrated splines (64-point Gauss-Legendre in z) of all those slices add up to
    the projected spline wherever the integrand is smooth on the slice scale (R >= 0.1 A), up to
    the potential's tail beyond the integration radius (R_max = 6 A here: about 1e-3 absolute for
    Si, 3e-4 relative at R = 2 A)."""
    import ctypes as C
    p, _ = cases.cbed_small()
    p.pot_rmax = 6.0
    L = orc.lib()
    d = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
    R2, c0 = np.empty(128), np.empty(128)
    tmp = [np.empty(128) for _ in range(3)]
    L.or_spline(C.byref(p.c()), 14, d(R2), d(c0), d(tmp[0]), d(tmp[1]), d(tmp[2]), C.byref(C.c_double()))
    dz, za, rint = 1.358, 0.3, 6.0
    tot = np.zeros(128)
    for s in range(-8, 9):
        zs, ze = s * dz, (s + 1) * dz
        zm = 0.5 * (zs + ze)
        if not (min(zm - rint, zs) <= za < max(zm + rint, ze)):
            continue
        f = [np.empty(128) for _ in range(5)]
        L.or_fine_spline_table(C.byref(p.c()), 14, zm - za, dz, *(d(x) for x in f))
        tot += f[1]
    R = np.sqrt(R2)
    sel = (R >= 0.1) & (R <= 2.0)
    assert np.max(np.abs(tot[sel] - c0[sel]) / np.abs(c0[sel])) < 4e-4
    assert np.max(np.abs(tot[sel] - c0[sel])) < 2e-3
    x, w = np.empty(64), np.empty(64)
    L.or_gauss_legendre_half(64, d(x), d(w))
    assert abs(w.sum() - 1) < 1e-13 and abs(np.dot(w, x ** 2) - 1 / 12) < 1e-14 and abs(np.dot(w, x ** 4) - 1 / 80) < 1e-14


def test_defocus_series_equals_shifted_lens():
    """The oracle's defocus series (apply_CTF_kernel_batch restated) equals single HRTEM images with
    the objective lens moved to C10 + df."""
    p, at = cases.hrtem_small(nconf=2)
    dfs = [-80.0, 0.0, 55.0]
    ser = orc.simulate_tem_series(p, at, dfs)
    for i, df in enumerate(dfs):
        q = p.copy()
        q.obj_lens.c10 = p.obj_lens.c10 + df
        assert rel_l2(ser[i], orc.simulate_tem(q, at)) < 1e-12


def test_tilted_plane_wave_vacuum():
    """A tilted plane wave exp(2 pi i g0.(r - L/2)) whose g0 lies on the frequency grid stays a single
    Fourier component through vacuum slices under the tilted propagator: the ED pattern of an empty
    specimen is one bright pixel at g0."""
    from cudaem_b200 import _abi as abi
    p, at = cases.ed_small(nconf=1)
    lam, _, _ = orc.physics(p.E0)
    m = 3
    p.phi = 0.0
    p.theta = float(np.arcsin(m / p.lx * lam))
    p.iw_type = abi.MS_IW_PLANE_TILTED
    far = cb.Atoms(Z=np.array([8], np.int32), x=np.array([0.5], np.float32), y=np.array([0.5], np.float32),
                   z=np.array([0.0], np.float32), sigma=np.zeros(1, np.float32), occ=np.zeros(1, np.float32))
    img = orc.simulate_tem(p, far)
    peak = np.unravel_index(np.argmax(img), img.shape)
    assert peak == (p.ny // 2, p.nx // 2 + m)
    assert img[peak] / img.sum() > 1 - 1e-9


def test_fp32_host_multislice_tracks_fp64():
    """The FP32 host multislice (the CPU baseline's single-precision figure) against the FP64 oracle."""
    p, at = cases.cbed_small(nconf=2)
    assert rel_l2(orc.simulate_cbed_f32(p, at), orc.simulate_cbed(p, at)) < 1e-4
