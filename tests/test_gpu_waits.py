"""Bounded waits and failed allocations, exercised on the GPU without a fault.

The reference waits for its fence without a bound (src/vulkan.cpp:306).  Here
every wait is bounded, and these tests make the bounds run out:

* device: a kernel's first wait for its own asynchronous work (the harmonic
  kernel's bulk staging copies, the tensor-core pass 1's MMAs) with a poll
  bound of 0 gives up at once; the template's status word gets
  STATUS_WAIT_TIMEOUT, the run reports BRP_E_RESULT, the kernel drains its
  copies / MMAs with the full bound before the CTA leaves, and the next run
  with the default bound is clean and equal to an undisturbed run;
* host: a run with a deadline of 0 s returns BRP_E_TIMEOUT while the GPU
  finishes; the next run first waits for that work and succeeds;
* allocation: a failed device allocation during the toplist pre-filter's
  set-up (a host-side fake of cudaMalloc failing) leaves the filter off, and a
  later set-up succeeds and filters correctly.
"""
import numpy as np
import pytest

import brp_b200 as B
from brp_b200 import synth
from brp_b200._lib import lib

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small():
    return synth.bank_workload("waits", [1 << 18], [6], [1], seed=41, f0=800.0, sigmas=(5.0,))


def make_bank(wl, **configure):
    bank = B.Bank(wl.n, [len(x) for x in wl.series], len(wl.templates), 8192)
    for s, x in enumerate(wl.series):
        bank.set_series(s, x)
    if configure:
        bank.configure(wl.n[0], **configure)
    return bank


def test_device_wait_expiry_is_reported_and_the_next_run_is_clean(small):
    wl = small
    bank = make_bank(wl)
    ref, _, _ = bank.run(wl.templates, wl.series_of)
    assert sum(len(c) for c in ref) > 0
    bank.set_wait_limits(device_polls=0)
    with pytest.raises(B.BrpError) as e:
        bank.run(wl.templates, wl.series_of)
    # BRP_E_RESULT: Bank.run_flat attaches the per-template status words
    assert "no valid result" in str(e.value)
    assert all(s & B.STATUS_WAIT_TIMEOUT for s in e.value.status)
    bank.set_wait_limits()  # defaults again
    got, counts, status = bank.run(wl.templates, wl.series_of)
    assert not status.any()
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)
    bank.close()


def test_device_wait_expiry_tensor_core_pass1():
    """The tensor-core pass 1 (config 113, n = 3*2^21) gives up its MMA wait at
    once, drains the MMAs, frees its tensor memory and reports the timeout."""
    wl = synth.bank_workload("waits-tc", [3 << 21], [2], [1], seed=43)
    bank = make_bank(wl, pass1=113, pass2=0, group=2, chains=1)
    ref, _, _ = bank.run(wl.templates, wl.series_of)
    bank.set_wait_limits(device_polls=0)
    with pytest.raises(B.BrpError) as e:
        bank.run(wl.templates, wl.series_of)
    assert all(s & B.STATUS_WAIT_TIMEOUT for s in e.value.status)
    bank.set_wait_limits()
    got, _, status = bank.run(wl.templates, wl.series_of)
    assert not status.any()
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)
    bank.close()


def test_context_wait_limits(small):
    """brp::GPU's context: the device wait expiry reaches the result slot's
    error word (GPU::candidates throws there, src/vulkan.cpp:333)."""
    p = small.templates[0]
    x = small.series[0]
    g = B.GPU(p, x, 192, 0, 1, stockham=True, packed=True)
    g.set_template(p)
    g.run()
    ref = g.candidates()
    g.set_wait_limits(device_polls=0)
    g.run()
    with pytest.raises(B.BrpError) as e:
        g.candidates()
    assert e.value.status == 2
    g.set_wait_limits()
    g.run()
    assert np.array_equal(g.candidates(), ref)
    g.close()


def test_host_deadline_expiry_then_next_run_succeeds():
    """A 128-template bank at n = 2^22 with a 0 s host deadline: the run
    returns BRP_E_TIMEOUT at its first poll while the GPU still works; with the
    default deadline the next run waits for that work first and succeeds."""
    import torch
    wl = synth.bank_workload("deadline", [1 << 22], [128], [1], seed=45)
    bank = make_bank(wl)
    ref, _, _ = bank.run(wl.templates, wl.series_of)
    bank.set_wait_limits(host_seconds=0.0)
    with pytest.raises(B.BrpError) as e:
        bank.run(wl.templates, wl.series_of)
    assert e.value.status == 3
    # an upload now must not touch the buffer the late run may still read
    bank.set_series(0, wl.series[0])
    bank.set_wait_limits()
    got, _, status = bank.run(wl.templates, wl.series_of)
    assert not status.any()
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)
    # and once more after an explicit synchronisation of the device
    bank.set_wait_limits(host_seconds=0.0)
    with pytest.raises(B.BrpError):
        bank.run(wl.templates, wl.series_of)
    torch.cuda.synchronize()
    bank.set_wait_limits()
    got, _, status = bank.run(wl.templates, wl.series_of)
    assert not status.any() and all(np.array_equal(a, b) for a, b in zip(got, ref))
    bank.close()


def test_failed_filter_allocation_leaves_the_filter_off(small):
    wl = small
    bank = make_bank(wl)
    full, _, _ = bank.run(wl.templates, wl.series_of)
    L = lib()
    try:
        for after in (1, 3, 9):  # fail the first, a middle and the last device allocation of the set-up
            L.brp_cuda_debug_fail_allocation(after)
            with pytest.raises(B.BrpError) as e:
                bank.set_toplist_filter(100)
            assert e.value.status == 1 and "cudaMalloc failed" in str(e.value)
            L.brp_cuda_debug_fail_allocation(0)
            got, _, _ = bank.run(wl.templates, wl.series_of)  # filter still off: every candidate
            assert all(np.array_equal(a, b) for a, b in zip(got, full))
    finally:
        L.brp_cuda_debug_fail_allocation(0)
    bank.set_toplist_filter(100)
    kept, counts, status = bank.run(wl.templates, wl.series_of)
    assert not status.any()
    top_full = B.Toplist().fold(wl.templates, wl.orbits, full).final()
    top_kept = B.Toplist().fold(wl.templates, wl.orbits, kept).final()
    assert top_full.tobytes() == top_kept.tobytes()
    bank.close()


def test_failed_context_allocation_is_an_error():
    p = B.parameters(1 << 16, (1 << 16) - 17, 0.3, 3600.0, 1.1, synth.DT)
    x = synth.make_series((1 << 16) - 17, 3)
    L = lib()
    try:
        L.brp_cuda_debug_fail_allocation(4)
        with pytest.raises(B.BrpError) as e:
            B.GPU(p, x, 192, 0, 1, stockham=True, packed=True)
        assert "cudaMalloc failed" in str(e.value)
    finally:
        L.brp_cuda_debug_fail_allocation(0)
    g = B.GPU(p, x, 192, 0, 1, stockham=True, packed=True)
    g.set_template(p)
    g.run()
    g.close()
