"""cudaem_b200 -- a B200-native multislice engine behind cudaEM's simulator surface.

The compute path is libcudaem_b200.so (hand-written sm_100a CUDA kernels and a
C++ host layer behind a C ABI, include/cudaem_b200.h).  This module is the
Python mirror of the reference's C++ interface:

    reference (cudaEM)                          here
    mulSimulator::executionTEM  (simulator.cu:8)   MulSimulator.executionTEM
    mulSimulator::executionCBED (simulator.cu:20)  MulSimulator.executionCBED
    mulSimulator::executionSTEM (simulator.cu:31)  MulSimulator.executionSTEM
    Thickness_simulator::Thickness_multiGPU        ThicknessSimulator.run
    multislice_params<float>                       MultisliceParams
    output_Multi_Data<float>                       OutputMultiData
    Atom_Coord_Data<float>                         Atoms

There is no CPU fallback: if the library is missing or no GPU is present the
calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _abi as abi

__all__ = ["MsError", "Atoms", "MultisliceParams", "OutputMultiData", "Context", "MulSimulator",
           "ThicknessSimulator", "build_crystal", "srtio3", "si_diamond", "lib", "library_path", "physics"]

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB: Optional[C.CDLL] = None


def library_path() -> str:
    return os.path.join(_HERE, "libcudaem_b200.so")


def lib() -> C.CDLL:
    """The loaded engine library; raises if it has not been built."""
    global _LIB
    if _LIB is None:
        path = library_path()
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is not built: run `python -m cudaem_b200.build` (nvcc, sm_100a)")
        _LIB = abi.bind(C.CDLL(path))
    return _LIB


class MsError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{abi.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def _check(st: int, ctx_handle=None) -> None:
    if st != abi.MS_OK:
        msg = lib().ms_last_error(ctx_handle)
        raise MsError(st, msg.decode() if msg else "")


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def physics(E0_kV: float) -> tuple[float, float, float]:
    """(wavelength A, interaction constant rad/(V A), gamma) at E0_kV."""
    lam, sig, gam = C.c_double(), C.c_double(), C.c_double()
    _check(lib().ms_physics(E0_kV, C.byref(lam), C.byref(sig), C.byref(gam)))
    return lam.value, sig.value, gam.value


# ---------------------------------------------------------------------------
# specimen
# ---------------------------------------------------------------------------
@dataclass
class Atoms:
    """Atom_Coord_Data<float>: Z, x, y, z (A), per-axis thermal sigma (A), occupancy."""
    Z: np.ndarray
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    sigma: np.ndarray
    occ: np.ndarray

    def __post_init__(self):
        self.Z = np.ascontiguousarray(self.Z, dtype=np.int32)
        for n in ("x", "y", "z", "sigma", "occ"):
            setattr(self, n, np.ascontiguousarray(getattr(self, n), dtype=np.float32))

    @property
    def n(self) -> int:
        return int(self.Z.shape[0])

    def c(self) -> abi.ms_atoms:
        return abi.ms_atoms(self.n, _iptr(self.Z), _fptr(self.x), _fptr(self.y), _fptr(self.z), _fptr(self.sigma),
                            _fptr(self.occ))


def build_crystal(basis_Z: Sequence[int], basis_frac: Sequence[Sequence[float]], a: float, b: float, c: float,
                  na: int, nb: int, nc: int, sigma: float, occ: float = 1.0) -> Atoms:
    """A slab of na x nb x nc unit cells (ms_build_crystal)."""
    L = lib()
    bz = np.ascontiguousarray(basis_Z, dtype=np.int32)
    bf = np.ascontiguousarray(basis_frac, dtype=np.float64).reshape(-1)
    n = C.c_int64()
    _check(L.ms_build_crystal(len(bz), _iptr(bz), _dptr(bf), a, b, c, na, nb, nc, sigma, occ, C.byref(n), None,
                              None, None, None, None, None))
    Z = np.empty(n.value, np.int32)
    arr = [np.empty(n.value, np.float32) for _ in range(5)]
    _check(L.ms_build_crystal(len(bz), _iptr(bz), _dptr(bf), a, b, c, na, nb, nc, sigma, occ, C.byref(n), _iptr(Z),
                              *[_fptr(x) for x in arr]))
    return Atoms(Z, *arr)


SRTIO3_BASIS = ([38, 22, 8, 8, 8], [(0, 0, 0), (0.5, 0.5, 0.5), (0.5, 0.5, 0), (0.5, 0, 0.5), (0, 0.5, 0.5)])
SI_BASIS = ([14] * 8, [(0, 0, 0), (0.5, 0.5, 0), (0.5, 0, 0.5), (0, 0.5, 0.5), (0.25, 0.25, 0.25),
                       (0.75, 0.75, 0.25), (0.75, 0.25, 0.75), (0.25, 0.75, 0.75)])


def srtio3(na: int, nb: int, nc: int, sigma: float = 0.08, a: float = 3.905) -> Atoms:
    """SrTiO3 cubic perovskite [001] slab."""
    return build_crystal(SRTIO3_BASIS[0], SRTIO3_BASIS[1], a, a, a, na, nb, nc, sigma)


def si_diamond(na: int, nb: int, nc: int, sigma: float = 0.075, a: float = 5.431) -> Atoms:
    """Si diamond [001] slab (8-atom conventional cell)."""
    return build_crystal(SI_BASIS[0], SI_BASIS[1], a, a, a, na, nb, nc, sigma)


# ---------------------------------------------------------------------------
# parameters and outputs
# ---------------------------------------------------------------------------
class MultisliceParams:
    """multislice_params<float>: a thin wrapper around the ms_params struct.

    Attributes of ms_params read and write through (params.nx = 512, ...);
    lenses are params.cond_lens / params.obj_lens (ms_lens structs)."""

    def __init__(self, **kw):
        object.__setattr__(self, "_p", abi.ms_params())
        object.__setattr__(self, "_coefs", None)
        lib().ms_default_params(C.byref(self._p))
        for k, v in kw.items():
            setattr(self, k, v)

    def __getattr__(self, k):
        return getattr(self._p, k)

    def __setattr__(self, k, v):
        if k == "detectors":
            self.set_detectors(v)
        elif k == "element_coefs":
            self.set_element_coefs(v)
        else:
            setattr(self._p, k, v)

    def set_detectors(self, dets: Sequence[tuple[float, float]]) -> None:
        """Annular detectors as (inner, outer) semi-angles in rad."""
        if len(dets) > abi.MS_MAX_DET:
            raise ValueError("too many detectors")
        self._p.n_det = len(dets)
        for i, (a, b) in enumerate(dets):
            self._p.det_inner[i] = a
            self._p.det_outer[i] = b

    def set_element_coefs(self, coefs: Sequence[tuple[int, int, Sequence[float], Sequence[float]]]) -> None:
        """Per-element V(r) tables: (Z, form, cl[6], cnl[6])."""
        arr = (abi.ms_element_coef * max(1, len(coefs)))()
        for i, (Z, form, cl, cnl) in enumerate(coefs):
            arr[i].Z = Z
            arr[i].form = form
            for j in range(abi.MS_MAX_COEF):
                arr[i].cl[j] = cl[j] if j < len(cl) else 0.0
                arr[i].cnl[j] = cnl[j] if j < len(cnl) else 1.0
        object.__setattr__(self, "_coefs", arr)
        self._p.element_coefs = C.cast(arr, C.POINTER(abi.ms_element_coef))
        self._p.n_element_coefs = len(coefs)

    def copy(self) -> "MultisliceParams":
        q = MultisliceParams()
        C.memmove(C.byref(q._p), C.byref(self._p), C.sizeof(abi.ms_params))
        if self._coefs is not None:
            object.__setattr__(q, "_coefs", self._coefs)
        return q

    def c(self) -> abi.ms_params:
        return self._p

    def validate(self) -> None:
        """multislice_params::validate_parameters."""
        _check(lib().ms_validate_params(C.byref(self._p)))


@dataclass
class OutputMultiData:
    """output_Multi_Data<float>."""
    image_intensity: Optional[np.ndarray] = None
    image_real: Optional[np.ndarray] = None
    image_imag: Optional[np.ndarray] = None
    stem_intensity: Optional[np.ndarray] = None
    thickness_frames: Optional[np.ndarray] = None
    row: int = 0
    col: int = 0
    n_slices: int = 0
    interval_x: float = 0.0
    interval_y: float = 0.0
    total_intensity: float = 0.0
    device_ms: float = 0.0
    launches: int = 0


class Context:
    """One GPU, one stream (ms_create / ms_destroy)."""

    def __init__(self, device: int = 0):
        self.handle = C.c_void_p()
        _check(lib().ms_create(C.byref(self.handle), device))

    def close(self) -> None:
        if self.handle:
            lib().ms_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def check(self, st: int) -> None:
        _check(st, self.handle)

    @property
    def last_device_ms(self) -> float:
        return lib().ms_last_device_ms(self.handle)

    @property
    def last_launch_count(self) -> int:
        return lib().ms_last_launch_count(self.handle)

    @property
    def last_probe_batch(self) -> int:
        return lib().ms_last_probe_batch(self.handle)

    def set_graphs(self, enable: bool) -> None:
        self.check(lib().ms_set_graphs(self.handle, 1 if enable else 0))

    def set_pass_kernels(self, variant: int) -> None:
        """0 (default): classic per-slice passes, the slice engine for uneven batches; 1: persistent
        pipelined passes; 2: the persistent slice engine everywhere; 3: per-slice passes everywhere."""
        self.check(lib().ms_set_pass_kernels(self.handle, variant))

    def set_transmission_store(self, enable: bool) -> None:
        """True (default): slices kept as t = exp(i sigma V); False: as sigma V (t formed in the row step)."""
        self.check(lib().ms_set_transmission_store(self.handle, 1 if enable else 0))

    def set_tile_shape(self, shape: int) -> None:
        """-1: autotuned per grid and batch (default); else bit 0 narrow rows, bit 1 narrow columns."""
        self.check(lib().ms_set_tile_shape(self.handle, int(shape)))

    @property
    def last_tile_shape(self) -> int:
        return lib().ms_last_tile_shape(self.handle)

    def set_tune_cache(self, path: Optional[str]) -> None:
        """JSON file keeping the autotuner's choices across contexts (None: in the context only)."""
        self.check(lib().ms_set_tune_cache(self.handle, path.encode() if path else None))

    def set_fault_injection(self, what: int) -> None:
        """Host-side fault injection for failure-path tests (abi.MS_INJECT_*)."""
        self.check(lib().ms_set_fault_injection(self.handle, int(what)))

    def set_potential_overlap(self, enable: bool) -> None:
        """False: all potentials before the slice loop (default); True: 16-slice chunks on a side
        stream beside the slice passes.  Identical results."""
        self.check(lib().ms_set_potential_overlap(self.handle, 1 if enable else 0))

    def set_profiling(self, enable: bool) -> None:
        self.check(lib().ms_set_profiling(self.handle, 1 if enable else 0))

    def profile_reset(self) -> None:
        self.check(lib().ms_profile_reset(self.handle))

    def profile(self, kernel: str) -> tuple[int, float]:
        """(launches, total device ms) of one kernel class since the last reset."""
        n, t = C.c_int64(), C.c_double()
        self.check(lib().ms_profile_get(self.handle, kernel.encode(), C.byref(n), C.byref(t)))
        return n.value, t.value

    def set_stream(self, stream_ptr: Optional[int]) -> None:
        self.check(lib().ms_set_stream(self.handle, C.c_void_p(stream_ptr) if stream_ptr else None))

    @property
    def stream(self) -> int:
        return lib().ms_get_stream(self.handle) or 0

    # -- low-level entry points ------------------------------------------------
    def projected_potential(self, params: MultisliceParams, atoms: Atoms, conf: int = 0) -> np.ndarray:
        """Sigma-scaled projected potentials [n_slices, ny, nx] of configuration conf (rad)."""
        ns = C.c_int()
        p, a = params.c(), atoms.c()
        self.check(lib().ms_projected_potential(self.handle, C.byref(p), C.byref(a), conf, None, 0, 0, C.byref(ns)))
        V = np.empty((ns.value, params.ny, params.nx), np.float32)
        self.check(lib().ms_projected_potential(self.handle, C.byref(p), C.byref(a), conf, _fptr(V), V.size, 0,
                                                C.byref(ns)))
        return V

    def stem_forward_potential(self, params: MultisliceParams, V: np.ndarray, z_init: float,
                               probe_xy: np.ndarray) -> np.ndarray:
        V = np.ascontiguousarray(V, np.float32)
        xy = np.ascontiguousarray(probe_xy, np.float64).reshape(-1, 2)
        I = np.empty((xy.shape[0], params.n_det), np.float32)
        p = params.c()
        self.check(lib().ms_stem_forward_potential(self.handle, C.byref(p), _fptr(V), V.shape[0], 0, z_init,
                                                   _dptr(xy), xy.shape[0], _fptr(I)))
        return I

    def stem_backward(self, params: MultisliceParams, V: np.ndarray, z_init: float, probe_xy: np.ndarray,
                      target: np.ndarray):
        V = np.ascontiguousarray(V, np.float32)
        xy = np.ascontiguousarray(probe_xy, np.float64).reshape(-1, 2)
        T = np.ascontiguousarray(target, np.float32)
        gV = np.empty_like(V)
        loss, g10, g30 = C.c_double(), C.c_double(), C.c_double()
        p = params.c()
        self.check(lib().ms_stem_backward(self.handle, C.byref(p), _fptr(V), V.shape[0], 0, z_init, _dptr(xy),
                                          xy.shape[0], _fptr(T), C.byref(loss), _fptr(gV), C.byref(g10),
                                          C.byref(g30)))
        return loss.value, gV, g10.value, g30.value


def displace_atoms(params: MultisliceParams, atoms: Atoms, conf: int) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Frozen-phonon coordinates of configuration conf (host, bit-identical to the device path)."""
    x, y, z = (np.empty(atoms.n, np.float32) for _ in range(3))
    p, a = params.c(), atoms.c()
    _check(lib().ms_displace_atoms(C.byref(p), C.byref(a), conf, _fptr(x), _fptr(y), _fptr(z)))
    return x, y, z


def build_slices(params: MultisliceParams, atoms: Atoms, conf: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """Slice planes and each atom's slice (Slice_Generator::calculate)."""
    ns = C.c_int()
    p, a = params.c(), atoms.c()
    _check(lib().ms_build_slices(C.byref(p), C.byref(a), conf, C.byref(ns), None, 0, None))
    b = np.empty(ns.value + 1, np.float32)
    s = np.empty(atoms.n, np.int32)
    _check(lib().ms_build_slices(C.byref(p), C.byref(a), conf, C.byref(ns), _fptr(b), b.size, _iptr(s)))
    return b, s


# ---------------------------------------------------------------------------
# simulators (mulSimulator, Thickness_simulator)
# ---------------------------------------------------------------------------
class MulSimulator:
    """mulSimulator (simulator.cu:8-49) on one B200."""

    def __init__(self, device: int = 0, ctx: Optional[Context] = None):
        self.ctx = ctx if ctx is not None else Context(device)

    def _out(self, params: MultisliceParams, kind: str) -> tuple[OutputMultiData, abi.ms_output]:
        o = OutputMultiData()
        co = abi.ms_output()
        if kind == "image":
            if params.data_record == abi.MS_RECORD_WAVE:
                o.image_real = np.empty((params.ny, params.nx), np.float32)
                o.image_imag = np.empty((params.ny, params.nx), np.float32)
                co.image_real, co.image_imag = _fptr(o.image_real), _fptr(o.image_imag)
            else:
                o.image_intensity = np.empty((params.ny, params.nx), np.float32)
                co.image_intensity = _fptr(o.image_intensity)
        elif kind == "stem":
            o.stem_intensity = np.empty((params.n_det, params.scan_ny, params.scan_nx), np.float32)
            co.stem_intensity = _fptr(o.stem_intensity)
        return o, co

    def _finish(self, o: OutputMultiData, co: abi.ms_output) -> OutputMultiData:
        o.row, o.col, o.n_slices = co.row, co.col, co.n_slices
        o.interval_x, o.interval_y, o.total_intensity = co.interval_x, co.interval_y, co.total_intensity
        o.device_ms = self.ctx.last_device_ms
        o.launches = self.ctx.last_launch_count
        return o

    def executionTEM(self, params: MultisliceParams, atoms: Atoms) -> OutputMultiData:
        o, co = self._out(params, "image")
        p, a = params.c(), atoms.c()
        self.ctx.check(lib().ms_simulate_tem(self.ctx.handle, C.byref(p), C.byref(a), C.byref(co)))
        return self._finish(o, co)

    def executionTEMDefocusSeries(self, params: MultisliceParams, atoms: Atoms,
                                  defocus: Sequence[float]) -> OutputMultiData:
        """HRTEM images at objective-lens defocus C10 + defocus[i] from one multislice run
        (ms_simulate_tem_defocus_series); the image arrays are [n_defocus][ny][nx]."""
        df = np.ascontiguousarray(defocus, np.float64).ravel()
        shape = (df.size, params.ny, params.nx)
        if params.data_record == abi.MS_RECORD_WAVE:
            o = OutputMultiData(image_real=np.empty(shape, np.float32), image_imag=np.empty(shape, np.float32))
        else:
            o = OutputMultiData(image_intensity=np.empty(shape, np.float32))
        co = abi.ms_output()
        for name in ("image_intensity", "image_real", "image_imag"):
            arr = getattr(o, name)
            if arr is not None:
                setattr(co, name, arr.ctypes.data_as(C.POINTER(C.c_float)))
        p, a = params.c(), atoms.c()
        self.ctx.check(lib().ms_simulate_tem_defocus_series(self.ctx.handle, C.byref(p), C.byref(a), df.size,
                                                           df.ctypes.data_as(C.POINTER(C.c_double)), C.byref(co)))
        return self._finish(o, co)

    def executionCBED(self, params: MultisliceParams, atoms: Atoms) -> OutputMultiData:
        o, co = self._out(params, "image")
        p, a = params.c(), atoms.c()
        self.ctx.check(lib().ms_simulate_cbed(self.ctx.handle, C.byref(p), C.byref(a), C.byref(co)))
        return self._finish(o, co)

    def executionSTEM(self, params: MultisliceParams, atoms: Atoms) -> OutputMultiData:
        o, co = self._out(params, "stem")
        p, a = params.c(), atoms.c()
        self.ctx.check(lib().ms_simulate_stem(self.ctx.handle, C.byref(p), C.byref(a), C.byref(co)))
        return self._finish(o, co)


    def executionMany(self, jobs: Sequence[tuple[MultisliceParams, Atoms]]) -> tuple[list[OutputMultiData], np.ndarray]:
        """Uneven batch (ms_simulate_many): CBED simulations of mixed grids and slice counts in one
        call.  Returns the outputs and each instance's completion time in ms from the call's start."""
        n = len(jobs)
        cp = (abi.ms_params * n)()
        ca = (abi.ms_atoms * n)()
        co = (abi.ms_output * n)()
        outs = []
        for i, (params, atoms) in enumerate(jobs):
            C.memmove(C.byref(cp[i]), C.byref(params.c()), C.sizeof(abi.ms_params))
            ca[i] = atoms.c()
            o = OutputMultiData(image_intensity=np.empty((params.ny, params.nx), np.float32))
            co[i].image_intensity = _fptr(o.image_intensity)
            outs.append(o)
        lat = np.zeros(n, np.float64)
        self.ctx.check(lib().ms_simulate_many(self.ctx.handle, n, cp, ca, co, _dptr(lat)))
        for i in range(n):
            self._finish(outs[i], co[i])
        return outs, lat


class ThicknessSimulator(MulSimulator):
    """Thickness_simulator (thickness_simulator.cuh:88-138)."""

    def run(self, params: MultisliceParams, atoms: Atoms) -> OutputMultiData:
        b, _ = build_slices(params, atoms, 0)
        nf = b.size - 1
        o = OutputMultiData(thickness_frames=np.empty((nf, params.ny, params.nx), np.float32))
        co = abi.ms_output()
        co.thickness_frames = _fptr(o.thickness_frames)
        co.thickness_capacity = o.thickness_frames.size
        p, a = params.c(), atoms.c()
        self.ctx.check(lib().ms_simulate_thickness(self.ctx.handle, C.byref(p), C.byref(a), C.byref(co)))
        return self._finish(o, co)
