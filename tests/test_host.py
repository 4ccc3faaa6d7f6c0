"""Host-side product code against the oracle (CPU only): phonon displacement,
slicing, crystal slabs, parameter validation and the C ABI surface."""
import ctypes as C
import os
import re
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import cases  # noqa: E402
import cudaem_b200 as cb  # noqa: E402
from cudaem_b200 import _abi as abi  # noqa: E402
from cudaem_b200 import workloads as wl  # noqa: E402
from oracle import oracle as orc  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("conf", [0, 1, 2, 7])
def test_displacement_bit_identical_to_oracle(conf):
    p, at = cases.cbed_small(cells=(3, 3, 3), nconf=8)
    got = cb.displace_atoms(p, at, conf)
    ref = orc.displace(p, at, conf)
    for g, r in zip(got, ref):
        assert np.array_equal(g, r)
    if conf == 0:
        assert np.array_equal(got[0], at.x)


def test_displacement_statistics():
    p, at = cases.cbed_small(cells=(8, 8, 8), nconf=2)
    x, y, z = cb.displace_atoms(p, at, 1)
    for d in (x - at.x, y - at.y, z - at.z):
        assert abs(d.std() - 0.075) < 0.004 and abs(d.mean()) < 0.004


def test_phonon_axes_flags():
    p, at = cases.cbed_small(cells=(2, 2, 2), nconf=2)
    p.pn_dim_z = 0
    x, y, z = cb.displace_atoms(p, at, 1)
    assert np.array_equal(z, at.z) and not np.array_equal(x, at.x)


@pytest.mark.parametrize("border", [-1, 0, 1, 2])
@pytest.mark.parametrize("conf", [0, 3])
@pytest.mark.parametrize("fine", [0, 1])
def test_slicing_bit_identical_to_oracle(border, conf, fine):
    p, at = cases.hrtem_small(cells=(3, 3, 6), nconf=4)
    p.slice_border = border
    p.enable_fine_slicing = fine
    b, s = cb.build_slices(p, at, conf)
    _, _, z = orc.displace(p, at, conf)
    bo, so = orc.slices(p, z)
    assert np.array_equal(b, bo) and np.array_equal(s, so)
    assert np.all(np.diff(b) > 0)
    if fine:   # the planes extend one integration radius beyond the atoms on either side
        assert s.min() > 0 and s.max() < b.size - 2
    else:
        assert s.min() >= 0 and s.max() == b.size - 2


@pytest.mark.parametrize("name,expected", [("hrtem", 40), ("cbed", 240), ("stem", 50), ("adjoint", 80)])
def test_workload_slice_counts(name, expected):
    """The measured workloads' specimens slice into the stated number of slices."""
    if name == "hrtem":
        p, at = wl.hrtem_sto()
    elif name == "cbed":
        p, at = wl.cbed_si()
    elif name == "stem":
        p, at = wl.stem_sto()
    else:
        p, at, _ = wl.adjoint_sto()
    for conf in ((0,) if name == "adjoint" else (1, 2)):
        b, _ = cb.build_slices(p, at, conf)
        assert b.size - 1 == expected


def test_crystal_builder():
    at = cb.srtio3(2, 3, 4)
    assert at.n == 5 * 24
    assert set(np.unique(at.Z)) == {8, 22, 38}
    assert np.isclose(at.x.max(), 1.5 * 3.905, atol=1e-5) and np.isclose(at.z.max(), 3.5 * 3.905, atol=1e-5)
    si = cb.si_diamond(1, 1, 1)
    assert si.n == 8
    assert np.allclose(np.sort(si.z), np.array([0, 0, 0.25, 0.25, 0.5, 0.5, 0.75, 0.75]) * 5.431, atol=1e-5)


@pytest.mark.parametrize("field,value,status", [
    ("nx", 100, abi.MS_ERR_UNSUPPORTED), ("ny", 4096, abi.MS_ERR_UNSUPPORTED), ("dz", 0.0, abi.MS_ERR_INVALID_ARG),
    ("E0", -1.0, abi.MS_ERR_INVALID_ARG), ("enable_fine_slicing", 2, abi.MS_ERR_INVALID_ARG),
    ("illumination_model", 9, abi.MS_ERR_INVALID_ARG), ("temporal_spatial_incoh", 7, abi.MS_ERR_INVALID_ARG),
    ("gpu_num", 2, abi.MS_ERR_UNSUPPORTED),
    ("n_det", 9, abi.MS_ERR_INVALID_ARG), ("phonon_model", 2, abi.MS_ERR_INVALID_ARG),
    ("simulation_type", 9, abi.MS_ERR_INVALID_ARG)])
def test_validation_status_codes(field, value, status):
    p, _ = cases.hrtem_small()
    setattr(p, field, value)
    st = cb.lib().ms_validate_params(C.byref(p.c()))
    assert st == status
    assert len(cb.lib().ms_last_error(None)) > 0
    with pytest.raises(cb.MsError):
        p.validate()


def test_default_params_validate():
    p, _ = cases.hrtem_small()
    p.validate()
    q = cb.MultisliceParams()
    q.validate()


def test_header_symbols_exported():
    """Every entry point include/cudaem_b200.h declares is exported by the library."""
    hdr = open(os.path.join(ROOT, "include", "cudaem_b200.h")).read()
    decl = set(re.findall(r"^\s*(?:const char\s*\*|int|void\s*\*?|double|int64_t|ms_status)\s+\**(ms_\w+)\s*\(",
                          hdr, re.M))
    assert len(decl) >= 20
    L = cb.lib()
    for s in sorted(decl):
        assert hasattr(L, s), s
        assert s in abi.PROTOTYPES, s
    assert L.ms_abi_version() == 2
    assert b"sm_100a" in L.ms_version()


def test_struct_layouts(tmp_path):
    """The ctypes mirrors match the C layout of include/cudaem_b200.h field by field: a small C
    program compiled from the header prints every struct's size and every field's offset."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    structs = [abi.ms_lens, abi.ms_element_coef, abi.ms_atoms, abi.ms_params, abi.ms_output]
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "cudaem_b200.h"', "int main(void) {"]
    expect = []
    for st in structs:
        nm = st.__name__
        lines.append(f'printf("%zu\\n", sizeof({nm}));')
        expect.append(C.sizeof(st))
        for f in st._fields_:
            lines.append(f'printf("%zu\\n", offsetof({nm}, {f[0]}));')
            expect.append(getattr(st, f[0]).offset)
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    subprocess.run([cc, "-I", inc, str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert got == expect


def test_no_device_is_reported():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    assert cb.lib().ms_create(C.byref(h), 0) == abi.MS_ERR_NO_DEVICE


@pytest.mark.parametrize("name", ["ms_set_graphs", "ms_set_pass_kernels", "ms_set_tile_shape", "ms_set_transmission_store",
                                  "ms_set_potential_overlap",
                                  "ms_set_profiling"])
def test_context_switches_reject_a_null_context(name):
    """The context switches check their handle before touching any device state."""
    assert getattr(cb.lib(), name)(None, 1) == abi.MS_ERR_INVALID_ARG


def test_tune_cache_rejects_a_null_context():
    assert cb.lib().ms_set_tune_cache(None, b"tune.json") == abi.MS_ERR_INVALID_ARG
