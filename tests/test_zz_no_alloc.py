"""The allocation-free STEM forward entry point.

ms_stem_forward_potential_noalloc serves callers that cannot let the library
call cudaMalloc (their own memory manager owns the device, or the
synchronisation an allocation implies is not acceptable in their loop).  It
keeps all of its scratch in a fixed array inside the library and takes the
potentials and the output in the caller's device memory.  These tests call it
through the C ABI twice in a row and compare each result with the allocating
entry point ms_stem_forward_potential, at the parity tolerance used for every
forward output (relative L2 <= 1e-5).

This file is named to be collected last, so a failure here leaves every other
test already run.
"""
import ctypes as C
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import cases  # noqa: E402
import cudaem_b200 as cb  # noqa: E402
from cudaem_b200 import _abi as abi  # noqa: E402
from conftest import rel_l2  # noqa: E402

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _noalloc(params, Vd, S, z_init, xy, Id, stream):
    p = params.c()
    xy = np.ascontiguousarray(xy, np.float64)
    st = cb.lib().ms_stem_forward_potential_noalloc(C.c_void_p(stream), C.byref(p), C.c_void_p(Vd.data_ptr()), S,
                                                    z_init, xy.ctypes.data_as(C.POINTER(C.c_double)),
                                                    xy.shape[0], C.c_void_p(Id.data_ptr()))
    return st


@pytest.mark.parametrize("n,ny,n_probe", [(256, 256, 7), (1024, 1024, 6), (512, 256, 5)])
def test_noalloc_matches_allocating_entry_point(n, ny, n_probe):
    import torch

    p, _ = cases.stem_small(n=n)
    p.ny = ny
    p.lx, p.ly = n * 0.1, ny * 0.1
    S = 5 if n <= 256 else 3
    V = cases.random_phase_slices(p, S, seed=n)
    rng = np.random.default_rng(n)
    xy = np.array([p.lx / 2, p.ly / 2]) + rng.uniform(-2.0, 2.0, size=(n_probe, 2))
    z_init = 0.8
    with cb.Context(0) as ctx:
        ref = ctx.stem_forward_potential(p, V, z_init, xy)
    Vd = torch.from_numpy(V).cuda()
    Id = torch.empty((n_probe, p.n_det), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):  # two calls in a row: the shared scratch must not carry state between calls
        Id.fill_(float("nan"))
        st = _noalloc(p, Vd, S, z_init, xy, Id, stream)
        assert st == abi.MS_OK, cb.lib().ms_last_error(None).decode()
        torch.cuda.synchronize()
        got = Id.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert rel_l2(got, ref) < TOL


_COLD_START = r"""
import ctypes as C, os, sys
import numpy as np
import torch
sys.path.insert(0, os.environ["MS_TEST_DIR"])
import cases
import cudaem_b200 as cb
from conftest import rel_l2
p, _ = cases.stem_small(n=256)
p.lx = p.ly = 25.6
V = cases.random_phase_slices(p, 4, seed=9)
xy = np.array([[12.8, 12.8], [11.0, 13.5], [14.1, 12.2]])
Vd = torch.from_numpy(V).cuda()
Id = torch.empty((3, p.n_det), dtype=torch.float32, device="cuda")
stream = torch.cuda.current_stream().cuda_stream
got = []
for _ in range(2):
    st = cb.lib().ms_stem_forward_potential_noalloc(C.c_void_p(stream), C.byref(p.c()), C.c_void_p(Vd.data_ptr()),
                                                    4, 0.5, xy.ctypes.data_as(C.POINTER(C.c_double)), 3,
                                                    C.c_void_p(Id.data_ptr()))
    assert st == 0, cb.lib().ms_last_error(None)
    torch.cuda.synchronize()
    got.append(Id.cpu().numpy().copy())
with cb.Context(0) as ctx:   # the allocating entry point only after the allocation-free calls
    ref = ctx.stem_forward_potential(p, V, 0.5, xy)
for g in got:
    assert np.all(np.isfinite(g)) and rel_l2(g, ref) < 1e-5, rel_l2(g, ref)
print("cold start ok")
"""


def test_noalloc_first_call_in_a_fresh_process():
    """The allocation-free entry point as the first engine call of a process: its set-up (the
    scratch array's address, the FFT constants, the kernels' shared-memory limits) runs on its
    own, before any context of the allocating API exists."""
    import subprocess

    env = dict(os.environ, MS_TEST_DIR=os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _COLD_START], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "cold start ok" in r.stdout


def test_noalloc_rejects_bad_arguments():
    import torch

    p, _ = cases.stem_small(n=256)
    Vd = torch.zeros((2, 256, 256), dtype=torch.float32, device="cuda")
    Id = torch.empty((1, p.n_det), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    q = p.copy()
    q.nx = q.ny = 4096   # refused by the parameter check, which caps each axis at 2048 (the array's limit)
    assert _noalloc(q, Vd, 2, 0.0, np.zeros((1, 2)), Id, stream) == abi.MS_ERR_UNSUPPORTED
    assert b"2048" in cb.lib().ms_last_error(None) or b"power" in cb.lib().ms_last_error(None)
    # a success clears the message of the failed call
    xy = np.array([[12.8, 12.8]])
    assert _noalloc(p, Vd, 2, 0.0, xy, Id, stream) == abi.MS_OK
    assert cb.lib().ms_last_error(None) == b""
    st = cb.lib().ms_stem_forward_potential_noalloc(C.c_void_p(stream), C.byref(p.c()), None, 2, 0.0,
                                                    np.zeros(2).ctypes.data_as(C.POINTER(C.c_double)), 1,
                                                    C.c_void_p(Id.data_ptr()))
    assert st == abi.MS_ERR_INVALID_ARG
