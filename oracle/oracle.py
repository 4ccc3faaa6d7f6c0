"""TEST INFRASTRUCTURE ONLY: ctypes wrapper over the FP64 CPU oracle.

The oracle (ms_oracle.c) restates cudaEM's multislice operators in double
precision on the CPU.  It is the checker for the CUDA engine; the engine
never imports or calls it.  Only tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py use this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libmsoracle.so")
_LIB = None


REF_LIB_PATH = os.path.join(HERE, "_ref", "libref_kernels.so")
REF_TREE = "/root/reference"


def build() -> str:
    subprocess.run(["make", "-C", HERE, "-s"], check=True)
    if os.path.isdir(REF_TREE):
        # the reference's own kernels: built only where the reference tree exists
        subprocess.run(["make", "-C", HERE, "-s", "ref", f"REF={REF_TREE}"], check=True)
    return LIB_PATH


_REF = None


REF_LOOP_PATH = os.path.join(HERE, "_ref", "libref_loop.so")
_REF_LOOP = None


def ref_loop_lib():
    """The reference's composed slice loop through its cuFFT callbacks (oracle/_ref/libref_loop.so),
    or None when it was not built."""
    global _REF_LOOP
    if _REF_LOOP is None and os.path.exists(REF_LOOP_PATH):
        L = C.CDLL(REF_LOOP_PATH)
        P, f, i = C.POINTER, C.c_float, C.c_int
        L.ref_slice_loop.restype = i
        L.ref_slice_loop.argtypes = [i, i, P(f), i, P(f), P(f), P(f)]
        _REF_LOOP = L
    return _REF_LOOP


def ref_lib():
    """The reference-kernel shim (oracle/_ref/libref_kernels.so), or None when it was not built."""
    global _REF
    if _REF is None and os.path.exists(REF_LIB_PATH):
        L = C.CDLL(REF_LIB_PATH)
        P, f, d, i = C.POINTER, C.c_float, C.c_double, C.c_int
        sig = {
            "ref_propagator": [i, i, d, d, d, i, d, P(f)],
            "ref_probe": [i, i, d, d, d, d, d, f, f, d, d, P(f)],
            "ref_ctf": [i, i, d, d, d, d, d, f, f, i, d, d, d, d, P(f), P(f)],
            "ref_detector": [i, i, d, d, f, f, P(f), P(d)],
            "ref_potential": [i, i, d, d, i, P(f), P(f), P(f), P(f), P(f), P(f), P(f), P(f), d, d, P(f)],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.restype = i
            fn.argtypes = args
        _REF = L
    return _REF


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        src = os.path.join(HERE, "ms_oracle.c")
        if not os.path.exists(LIB_PATH) or os.path.getmtime(src) > os.path.getmtime(LIB_PATH):
            build()
        from cudaem_b200 import _abi as abi
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        f, d, i = C.c_float, C.c_double, C.c_int
        sig = {
            "or_physics": (None, [d, P(d), P(d), P(d)]),
            "or_det_log": (d, [d]),
            "or_gauss_pair": (None, [C.c_uint64, i, C.c_int64, i, P(d), P(d)]),
            "or_displace": (None, [P(abi.ms_params), P(abi.ms_atoms), i, P(f), P(f), P(f)]),
            "or_slices": (i, [P(abi.ms_params), P(f), C.c_int64, P(f), i, P(i)]),
            "or_spline": (i, [P(abi.ms_params), i, P(d), P(d), P(d), P(d), P(d), P(d)]),
            "or_projected": (i, [P(abi.ms_params), i, d, P(d), P(d)]),
            "or_potential": (i, [P(abi.ms_params), P(abi.ms_atoms), i, P(d), C.c_int64, P(i), P(d)]),
            "or_fft2": (None, [P(d), i, i, i]),
            "or_simulate_tem": (i, [P(abi.ms_params), P(abi.ms_atoms), P(d), P(d), P(d)]),
            "or_simulate_cbed": (i, [P(abi.ms_params), P(abi.ms_atoms), P(d), P(d), P(d)]),
            "or_simulate_tem_series": (i, [P(abi.ms_params), P(abi.ms_atoms), i, P(d), P(d), P(d), P(d)]),
            "or_simulate_cbed_f32": (i, [P(abi.ms_params), P(abi.ms_atoms), P(d)]),
            "or_slice_loop": (i, [P(abi.ms_params), P(f), i, i, P(d), P(d)]),
            "or_simulate_stem": (i, [P(abi.ms_params), P(abi.ms_atoms), P(d)]),
            "or_simulate_thickness": (i, [P(abi.ms_params), P(abi.ms_atoms), P(d), C.c_int64, P(i)]),
            "or_stem_forward_potential": (i, [P(abi.ms_params), P(f), i, d, P(d), i, P(d)]),
            "or_stem_backward": (i, [P(abi.ms_params), P(f), i, d, P(d), i, P(f), P(d), P(d), P(d), P(d)]),
            "or_stem_loss_fd": (i, [P(abi.ms_params), P(f), i, d, P(d), i, P(f), i, P(C.c_int64), P(d), d, d,
                                    P(d), P(d), P(d)]),
            "or_gauss_hermite": (None, [i, P(d), P(d)]),
            "or_gauss_legendre_half": (None, [i, P(d), P(d)]),
            "or_fine_spline_table": (i, [P(abi.ms_params), i, d, d, P(d), P(d), P(d), P(d), P(d)]),
            "or_op_propagator": (i, [P(abi.ms_params), P(d)]),
            "or_op_probe": (i, [P(abi.ms_params), d, d, d, P(d)]),
            "or_op_ctf": (i, [P(abi.ms_params), i, d, d, d, P(d), P(d)]),
            "or_op_detect": (i, [P(abi.ms_params), P(d), P(d)]),
            "or_op_slice_potential": (i, [P(abi.ms_params), i, C.c_int64, P(f), P(f), P(f), P(d)]),
            "or_set_threads": (None, [i]),
            "or_get_threads": (i, []),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _f(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _i(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def set_threads(n: int) -> None:
    lib().or_set_threads(n)


def threads() -> int:
    return lib().or_get_threads()


def physics(E0):
    a, b, c = C.c_double(), C.c_double(), C.c_double()
    lib().or_physics(E0, C.byref(a), C.byref(b), C.byref(c))
    return a.value, b.value, c.value


def det_log(s: float) -> float:
    return lib().or_det_log(s)


def gauss_pair(seed, conf, atom, stream):
    a, b = C.c_double(), C.c_double()
    lib().or_gauss_pair(seed, conf, atom, stream, C.byref(a), C.byref(b))
    return a.value, b.value


def displace(params, atoms, conf):
    x, y, z = (np.empty(atoms.n, np.float32) for _ in range(3))
    p, a = params.c(), atoms.c()
    lib().or_displace(C.byref(p), C.byref(a), conf, _f(x), _f(y), _f(z))
    return x, y, z


def slices(params, z):
    z = np.ascontiguousarray(z, np.float32)
    p = params.c()
    ns = lib().or_slices(C.byref(p), _f(z), z.size, None, 0, None)
    b = np.empty(ns + 1, np.float32)
    s = np.empty(z.size, np.int32)
    lib().or_slices(C.byref(p), _f(z), z.size, _f(b), b.size, _i(s))
    return b, s


def spline(params, Z):
    arrs = [np.empty(128) for _ in range(5)]
    rmax = C.c_double()
    p = params.c()
    lib().or_spline(C.byref(p), Z, *[_d(a) for a in arrs], C.byref(rmax))
    return (*arrs, rmax.value)


def projected(params, Z, R):
    v, dv = C.c_double(), C.c_double()
    p = params.c()
    lib().or_projected(C.byref(p), Z, R, C.byref(v), C.byref(dv))
    return v.value, dv.value


def potential(params, atoms, conf=0):
    p, a = params.c(), atoms.c()
    ns, zi = C.c_int(), C.c_double()
    lib().or_potential(C.byref(p), C.byref(a), conf, None, 0, C.byref(ns), C.byref(zi))
    V = np.empty((ns.value, params.ny, params.nx))
    rc = lib().or_potential(C.byref(p), C.byref(a), conf, _d(V), V.size, C.byref(ns), C.byref(zi))
    assert rc == 0
    return V, zi.value


def fft2(x: np.ndarray, sign: int) -> np.ndarray:
    y = np.ascontiguousarray(x, np.complex128).copy()
    lib().or_fft2(_d(y.view(np.float64)), y.shape[1], y.shape[0], sign)
    return y


def _img_outputs(params):
    n = (params.ny, params.nx)
    if params.data_record == 1:
        return None, np.empty(n), np.empty(n)
    return np.empty(n), None, None


def simulate_tem(params, atoms):
    img, re, im = _img_outputs(params)
    p, a = params.c(), atoms.c()
    lib().or_simulate_tem(C.byref(p), C.byref(a), _d(img) if img is not None else None,
                          _d(re) if re is not None else None, _d(im) if im is not None else None)
    return img if img is not None else (re, im)


def simulate_tem_series(params, atoms, defocus):
    df = np.ascontiguousarray(defocus, np.float64).ravel()
    n = (df.size, params.ny, params.nx)
    p, a = params.c(), atoms.c()
    if params.data_record == 1:
        re, im = np.empty(n), np.empty(n)
        lib().or_simulate_tem_series(C.byref(p), C.byref(a), df.size, _d(df), None, _d(re), _d(im))
        return re, im
    img = np.empty(n)
    lib().or_simulate_tem_series(C.byref(p), C.byref(a), df.size, _d(df), _d(img), None, None)
    return img


def slice_loop(params, V, psi0):
    """The slice loop alone on phases V [S][ny][nx] and incident waves psi0 [B][ny][nx] (complex):
    the exit waves in reciprocal space, [B][ny][nx] complex128."""
    V = np.ascontiguousarray(V, np.float32)
    psi0 = np.ascontiguousarray(psi0, np.complex128).reshape(-1, params.ny, params.nx)
    out = np.empty_like(psi0)
    p = params.c()
    lib().or_slice_loop(C.byref(p), _f(V), V.shape[0], psi0.shape[0], _d(psi0.view(np.float64)),
                        _d(out.view(np.float64)))
    return out


def incident(params, px, py, z_init):
    """The incident wave (plane wave, or the convergent probe at (px, py) with defocus shift
    z_init), in real space, as complex128 [ny][nx]."""
    W = np.empty((params.ny, params.nx), np.complex128)
    p = params.c()
    lib().or_op_probe(C.byref(p), px, py, z_init, _d(W.view(np.float64)))
    return np.fft.ifft2(W) * W.size


def simulate_cbed_f32(params, atoms):
    """CBED intensity with the multislice loop in FP32 (the CPU baseline's single-precision path)."""
    img = np.empty((params.ny, params.nx))
    p, a = params.c(), atoms.c()
    lib().or_simulate_cbed_f32(C.byref(p), C.byref(a), _d(img))
    return img


def simulate_cbed(params, atoms):
    img, re, im = _img_outputs(params)
    p, a = params.c(), atoms.c()
    lib().or_simulate_cbed(C.byref(p), C.byref(a), _d(img) if img is not None else None,
                           _d(re) if re is not None else None, _d(im) if im is not None else None)
    return img if img is not None else (re, im)


def simulate_stem(params, atoms):
    out = np.empty((params.n_det, params.scan_ny, params.scan_nx))
    p, a = params.c(), atoms.c()
    lib().or_simulate_stem(C.byref(p), C.byref(a), _d(out))
    return out


def simulate_thickness(params, atoms):
    p, a = params.c(), atoms.c()
    nf = C.c_int()
    lib().or_simulate_thickness(C.byref(p), C.byref(a), None, 0, C.byref(nf))
    fr = np.empty((nf.value, params.ny, params.nx))
    rc = lib().or_simulate_thickness(C.byref(p), C.byref(a), _d(fr), fr.size, C.byref(nf))
    assert rc == 0
    return fr


def stem_forward_potential(params, V, z_init, xy):
    V = np.ascontiguousarray(V, np.float32)
    xy = np.ascontiguousarray(xy, np.float64).reshape(-1, 2)
    I = np.empty((xy.shape[0], params.n_det))
    p = params.c()
    lib().or_stem_forward_potential(C.byref(p), _f(V), V.shape[0], z_init, _d(xy), xy.shape[0], _d(I))
    return I


def stem_backward(params, V, z_init, xy, target):
    V = np.ascontiguousarray(V, np.float32)
    xy = np.ascontiguousarray(xy, np.float64).reshape(-1, 2)
    T = np.ascontiguousarray(target, np.float32)
    gV = np.empty(V.shape)
    loss, g10, g30 = C.c_double(), C.c_double(), C.c_double()
    p = params.c()
    lib().or_stem_backward(C.byref(p), _f(V), V.shape[0], z_init, _d(xy), xy.shape[0], _f(T), C.byref(loss),
                           _d(gV), C.byref(g10), C.byref(g30))
    return loss.value, gV, g10.value, g30.value


def stem_loss_fd(params, V, z_init, xy, target, idx, h, h10, h30):
    """Central differences of L = sum (I - target)^2 (FP64 forward) at the flat pixel indices
    `idx` of V (steps h) and for the condenser C10 and C30 (steps h10, h30)."""
    V = np.ascontiguousarray(V, np.float32)
    xy = np.ascontiguousarray(xy, np.float64).reshape(-1, 2)
    T = np.ascontiguousarray(target, np.float32)
    idx = np.ascontiguousarray(idx, np.int64)
    h = np.ascontiguousarray(h, np.float64)
    fd = np.empty(idx.size)
    f10, f30 = C.c_double(), C.c_double()
    p = params.c()
    rc = lib().or_stem_loss_fd(C.byref(p), _f(V), V.shape[0], z_init, _d(xy), xy.shape[0], _f(T), idx.size,
                               idx.ctypes.data_as(C.POINTER(C.c_int64)), _d(h), h10, h30, _d(fd), C.byref(f10),
                               C.byref(f30))
    assert rc == 0
    return fd, f10.value, f30.value


def gauss_hermite(n: int):
    x, w = np.empty(n), np.empty(n)
    lib().or_gauss_hermite(n, _d(x), _d(w))
    return x, w
