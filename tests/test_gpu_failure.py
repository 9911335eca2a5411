"""Failure detection on the GPU without a fault: the error paths are made to run by the library's own
injection switch (fsg_set_fault), never by a bad address, a trap or an endless wait.

* A staging wait that runs out: every chunk of line records expects 16 bytes more than its bulk copies
  deliver, so its mbarrier phase never completes; the bounded wait (1 ms here) gives up, the kernel
  drains its copies and returns, and the call reports FSG_E_TIMEOUT.
* A device allocation that fails: allocations above a cap are refused as on an exhausted device
  (FSG_E_NOMEM).
After each, the same context runs normally again and reproduces a fresh context's result bit for bit."""
import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu


def small_case(fsg):
    from fastspec_b200 import workloads as W
    st, meta = H.load_atm("solar")
    w0, w1, dstep = 5000.0, 5004.0, 0.005
    co = H.contopac_on(meta, fsg.make_grid(0, w0, w1, dstep) + w0)
    lines = fsg.LineList.from_arrays(W.atomic_lines(600, w0, w1, W.SEED0 + 80).arrays())

    def make():
        C = fsg.Context(vmicro=1.0)
        C.set_grid(0, w0, w1, dstep)
        C.set_atmosphere(st)
        C.set_contopac(co)
        x, w, _ = fsg.mu_quadrature(1, 7)
        C.set_mu(x, w)
        return C
    return make, lines


def test_staging_wait_runs_out_and_the_context_recovers(fsg):
    make, lines = small_case(fsg)
    ref = make()
    want = ref.lineop_calc(lines)["lineopac"]
    _, _, want_flux, _ = ref.radtran()
    ref.close()
    C = make()
    C.set_fault(fsg.FAULT_COPY_TIMEOUT, 1.0)
    with pytest.raises(fsg.FsgError) as e:
        C.lineop_calc(lines)
    assert "(-6)" in str(e.value) and "bound" in str(e.value), str(e.value)          # FSG_E_TIMEOUT
    C.set_fault(fsg.FAULT_NONE)
    C.lineop_reset()
    got = C.lineop_calc(lines)["lineopac"]
    _, _, flux, _ = C.radtran()
    assert np.array_equal(got, want) and np.array_equal(flux, want_flux)
    C.close()


def test_refused_allocation_and_the_context_recovers(fsg):
    make, lines = small_case(fsg)
    C = make()
    C.set_fault(fsg.FAULT_ALLOC_LIMIT, 4096)
    with pytest.raises(fsg.FsgError) as e:
        C.lineop_calc(lines)
    assert "(-3)" in str(e.value) and "allocation" in str(e.value), str(e.value)    # FSG_E_NOMEM
    C.set_fault(fsg.FAULT_NONE)
    C.lineop_reset()
    got = C.lineop_calc(lines)["lineopac"]
    ref = make()
    assert np.array_equal(got, ref.lineop_calc(lines)["lineopac"])
    ref.close()
    C.close()


def test_fault_switch_rejects_bad_values(fsg):
    make, _ = small_case(fsg)
    C = make()
    for kind, value in ((fsg.FAULT_COPY_TIMEOUT, 0.0), (fsg.FAULT_COPY_TIMEOUT, 5000.0), (fsg.FAULT_ALLOC_LIMIT, 0.0),
                        (99, 1.0)):
        with pytest.raises(fsg.FsgError):
            C.set_fault(kind, value)
    C.close()
