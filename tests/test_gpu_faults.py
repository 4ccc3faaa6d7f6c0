"""Failure paths on the GPU without a GPU fault.

The tile loads of the column passes complete on a shared-memory barrier whose wait is bounded.
With MS_INJECT_WAIT_TIMEOUT the kernels wait for bytes that never arrive (a transfer count that
nothing satisfies); the wait runs out after about a millisecond, the kernel records it and
returns, and the call reports MS_ERR_TIMEOUT.  The same context then runs the simulation
normally and matches the FP64 oracle.
"""
import os
import sys

import pytest

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import cases  # noqa: E402
import cudaem_b200 as cb  # noqa: E402
from cudaem_b200 import _abi as abi  # noqa: E402
from conftest import rel_l2  # noqa: E402
from oracle import oracle as orc  # noqa: E402

pytestmark = pytest.mark.gpu


def test_bounded_wait_runs_out_and_context_recovers():
    p, at = cases.cbed_small(n=256, nconf=2)
    with cb.Context(0) as ctx:
        sim = cb.MulSimulator(ctx=ctx)
        ctx.set_fault_injection(abi.MS_INJECT_WAIT_TIMEOUT)
        with pytest.raises(cb.MsError) as e:
            sim.executionCBED(p, at)
        assert e.value.status == abi.MS_ERR_TIMEOUT
        ctx.set_fault_injection(abi.MS_INJECT_NONE)
        out = sim.executionCBED(p, at)
        assert rel_l2(out.image_intensity, orc.simulate_cbed(p, at)) < 1e-5


def test_fault_injection_rejects_unknown_codes():
    with cb.Context(0) as ctx:
        with pytest.raises(cb.MsError):
            ctx.set_fault_injection(7)


def test_allocation_failure_and_context_recovers():
    """Every device allocation of the call fails (as cudaMalloc out of memory): the call reports
    MS_ERR_OUT_OF_MEMORY; the same context then allocates and runs normally."""
    p, at = cases.cbed_small(n=128, nconf=2)
    with cb.Context(0) as ctx:
        sim = cb.MulSimulator(ctx=ctx)
        ctx.set_fault_injection(abi.MS_INJECT_ALLOC_FAIL)
        with pytest.raises(cb.MsError) as e:
            sim.executionCBED(p, at)
        assert e.value.status == abi.MS_ERR_OUT_OF_MEMORY
        ctx.set_fault_injection(abi.MS_INJECT_NONE)
        out = sim.executionCBED(p, at)
        assert rel_l2(out.image_intensity, orc.simulate_cbed(p, at)) < 1e-5


def test_allocation_failure_mid_stem_batches():
    """A STEM call fails part-way on a grown buffer (a larger scan needs larger batch buffers than
    the call before it): MS_ERR_OUT_OF_MEMORY, and the context then completes the larger scan."""
    small, at = cases.stem_small(n=128, scan=(2, 1), nconf=1, batch=0)
    large, _ = cases.stem_small(n=128, scan=(6, 5), nconf=1, batch=0)
    with cb.Context(0) as ctx:
        sim = cb.MulSimulator(ctx=ctx)
        sim.executionSTEM(small, at)          # buffers sized for two probes
        ctx.set_fault_injection(abi.MS_INJECT_ALLOC_FAIL)
        with pytest.raises(cb.MsError) as e:
            sim.executionSTEM(large, at)
        assert e.value.status == abi.MS_ERR_OUT_OF_MEMORY
        ctx.set_fault_injection(abi.MS_INJECT_NONE)
        out = sim.executionSTEM(large, at)
        assert rel_l2(out.stem_intensity, orc.simulate_stem(large, at)) < 1e-5
