"""A second, independent restatement of the multislice wave operators in numpy
(FP64, numpy.fft), used only to cross-check the C oracle.

It follows the same reference lines as the oracle: propagator
(device_kernels.cuh:215-234, grid_dev.cuh:307-325, :462-465), probe
(device_kernels.cuh:363-388), CTF (device_kernels.cuh:445-468), annular
detector (device_kernels.cuh:534-579) and the loop (wave_function.cuh:60-73).
Frequency masks use the float32 arithmetic the engine uses.
"""
from __future__ import annotations

import numpy as np

PI = np.pi


def physics(E0_kV):
    h, me, qe, c = 6.62607015e-34, 9.1093837015e-31, 1.602176634e-19, 299792458.0
    E = E0_kV * 1e3
    g = 1 + qe * E / (me * c * c)
    lam = h / np.sqrt(2 * me * qe * E * (1 + qe * E / (2 * me * c * c)))
    sig = 2 * PI * g * me * qe * lam / h ** 2 * 1e-10
    return lam * 1e10, sig, g


def freqs(n, L):
    k = np.where(np.arange(n) < n // 2, np.arange(n), np.arange(n) - n)
    return k / L, (k.astype(np.float32) * (np.float32(1.0) / np.float32(L))).astype(np.float32)


def grids(p):
    fx, fxf = freqs(p.nx, p.lx)
    fy, fyf = freqs(p.ny, p.ly)
    gx, gy = np.meshgrid(fx, fy)
    g2f = (fxf[None, :] * fxf[None, :]).astype(np.float32) + (fyf[:, None] * fyf[:, None]).astype(np.float32)
    return gx, gy, g2f.astype(np.float32)


def thr(ang, lam):
    g = np.float32(np.sin(ang) / lam)
    return np.float32(g * g)


def gate(v):
    return v if abs(v) > 1e-5 else 0.0


def propagator(p):
    lam, _, _ = physics(p.E0)
    gx, gy, _ = grids(p)
    N = p.nx * p.ny
    gmax = min((p.nx // 2) / p.lx, (p.ny // 2) / p.ly)
    gl = 2 * gmax / 3
    alpha = np.log(99.0) / ((gl + 0.25) ** 2 - gl ** 2)
    amp = np.full(gx.shape, 1.0 / N)
    if p.bwl:
        amp = amp / (1 + np.exp(alpha * (gx ** 2 + gy ** 2 - gl ** 2)))
    g0x = np.sin(p.theta) * np.cos(p.phi) / lam
    g0y = np.sin(p.theta) * np.sin(p.phi) / lam
    th = -PI * lam * p.dz * ((gx - g0x) ** 2 + (gy - g0y) ** 2)
    return amp * np.exp(1j * th)


def chi(lens, lam, gx, gy, c10_shift=0.0):
    """C10, C30, C50 only (the rotationally symmetric terms)."""
    g2 = gx ** 2 + gy ** 2
    cc10 = gate(-PI * (lens.c10 + c10_shift) * lam)
    cc30 = gate(-PI * lens.c30 * lam ** 3 / 2)
    cc50 = gate(-PI * lens.c50 * lam ** 5 / 3)
    return cc10 * g2 + cc30 * g2 ** 2 + cc50 * g2 ** 3


def probe(p, px, py, z_init):
    lam, _, _ = physics(p.E0)
    gx, gy, g2f = grids(p)
    L = p.cond_lens
    g2min = thr(L.inner_aper_ang, lam) if L.inner_aper_ang > 0 else np.float32(0)
    g2max = thr(L.outer_aper_ang, lam) if L.outer_aper_ang > 0 else np.float32(np.finfo(np.float32).max)
    A = (g2min <= g2f) & (g2f < g2max)
    ph = chi(L, lam, gx, gy, z_init) - 2 * PI * px * gx - 2 * PI * py * gy
    W = np.where(A, np.exp(1j * ph), 0)
    return np.fft.ifft2(W) * W.size


def multislice(p, V, psi0):
    P = propagator(p)
    N = p.nx * p.ny
    w = psi0.astype(complex)
    S = V.shape[0]
    for s in range(S):
        w = np.fft.fft2(w * np.exp(1j * V[s]))
        if s < S - 1:
            w = np.fft.ifft2(P * w) * N
    return w


def detect(p, W):
    lam, _, _ = physics(p.E0)
    _, _, g2f = grids(p)
    out = []
    a2 = np.abs(W) ** 2
    for d in range(p.n_det):
        m = (thr(p.det_inner[d], lam) <= g2f) & (g2f <= thr(p.det_outer[d], lam))
        out.append(a2[m].sum())
    return np.array(out)


def ctf_image(p, W):
    lam, _, _ = physics(p.E0)
    gx, gy, g2f = grids(p)
    L = p.obj_lens
    g2max = thr(L.outer_aper_ang, lam) if L.outer_aper_ang > 0 else np.float32(np.finfo(np.float32).max)
    g2min = thr(L.inner_aper_ang, lam) if L.inner_aper_ang > 0 else np.float32(0)
    A = (g2min <= g2f) & (g2f < g2max)
    w = np.where(A, W * np.exp(1j * chi(L, lam, gx, gy)), 0)
    return np.fft.ifft2(w) * w.size
