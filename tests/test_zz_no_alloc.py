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


@pytest.mark.parametrize("n,n_probe", [(256, 7), (1024, 6)])
def test_noalloc_matches_allocating_entry_point(n, n_probe):
    import torch

    p, _ = cases.stem_small(n=n)
    p.lx = p.ly = n * 0.1
    S = 5 if n <= 256 else 3
    V = cases.random_phase_slices(p, S, seed=n)
    rng = np.random.default_rng(n)
    xy = p.lx / 2 + rng.uniform(-2.0, 2.0, size=(n_probe, 2))
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


def test_noalloc_rejects_bad_arguments():
    import torch

    p, _ = cases.stem_small(n=256)
    Vd = torch.zeros((2, 256, 256), dtype=torch.float32, device="cuda")
    Id = torch.empty((1, p.n_det), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    q = p.copy()
    q.nx = q.ny = 4096
    assert _noalloc(q, Vd, 2, 0.0, np.zeros((1, 2)), Id, stream) == abi.MS_ERR_UNSUPPORTED
    assert b"2048" in cb.lib().ms_last_error(None) or b"power" in cb.lib().ms_last_error(None)
    st = cb.lib().ms_stem_forward_potential_noalloc(C.c_void_p(stream), C.byref(p.c()), None, 2, 0.0,
                                                    np.zeros(2).ctypes.data_as(C.POINTER(C.c_double)), 1,
                                                    C.c_void_p(Id.data_ptr()))
    assert st == abi.MS_ERR_INVALID_ARG
