"""Writes ref_kernels.npz: the outputs of the reference's own CUDA kernels on the cases of
ref_cases.py, as golden vectors that pin the oracle's per-pixel operators on the CPU.

Needs a GPU and the reference-kernel shim (oracle/_ref/libref_kernels.so, built by
`make -C oracle ref` where the reference tree is present).  Run from the repository root:

    python tests/golden/make_golden.py [output.npz]        # ref_kernels.npz
    python tests/golden/make_golden.py loop [output.npz]   # ref_loop.npz (the composed slice loop)

Inputs are rebuilt from fixed workloads and seeds by ref_cases.build, and stored beside the
outputs so that a change in the case builders is caught instead of silently compared.
"""
from __future__ import annotations

import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import ref_cases  # noqa: E402
from oracle import oracle as orc  # noqa: E402


def main_loop(out_path: str) -> None:
    """ref_loop.npz: the reference's composed slice loop on ref_loop_cases, sampled."""
    import ref_loop_cases as rl
    Lk, Ll = orc.ref_lib(), orc.ref_loop_lib()
    if Lk is None or Ll is None:
        raise SystemExit("reference shims not built: make -C oracle ref (needs the reference tree)")
    arrays = {}
    for name in rl.CASES:
        out = rl.reference(Ll, Lk, name)
        idx = rl.sample_index(out.shape[1] * out.shape[2])
        arrays[f"{name}__idx"] = idx
        arrays[f"{name}__out"] = out.reshape(out.shape[0], -1)[:, idx]
        arrays[f"{name}__norm"] = np.linalg.norm(out.reshape(out.shape[0], -1).astype(np.complex128), axis=1)
    np.savez_compressed(out_path, **arrays)
    print(f"wrote {out_path}: {len(arrays)} arrays, {os.path.getsize(out_path)} bytes")


def main(out_path: str) -> None:
    L = orc.ref_lib()
    if L is None:
        raise SystemExit("reference-kernel shim not built: make -C oracle ref (needs the reference tree)")
    arrays = {}
    for name in ref_cases.CASES:
        arrays[f"{name}__out"] = ref_cases.reference(L, name)
        _, a = ref_cases.build(name)
        for k, v in a.items():
            if isinstance(v, np.ndarray):
                arrays[f"{name}__in_{k}"] = v
    np.savez_compressed(out_path, **arrays)
    print(f"wrote {out_path}: {len(arrays)} arrays, {os.path.getsize(out_path)} bytes")


if __name__ == "__main__":
    here = os.path.dirname(os.path.abspath(__file__))
    if len(sys.argv) > 1 and sys.argv[1] == "loop":
        main_loop(sys.argv[2] if len(sys.argv) > 2 else os.path.join(here, "ref_loop.npz"))
    else:
        main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(here, "ref_kernels.npz"))
