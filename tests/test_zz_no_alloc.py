"""fsg_locprf_pp_noalloc: the LocPrfPP entry point for callers that cannot allocate device
memory (hosts whose device memory belongs to their own pool allocator).  It must give the
same intensities as the allocating entry point fsg_locprf_pp, call after call, while the
work arrays it shares across calls keep the previous call's contents.  This file is collected
last so that a failure here leaves every other test already run."""
import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu


def test_noalloc_locprf_matches_allocating_entry_point(fsg):
    import torch
    lib = fsg.lib()
    st, _ = H.load_atm("solar")
    rhox = np.asarray(st["rhox"], np.float64)
    nt = len(rhox)
    x = np.array([1.0, 0.8, 0.55, 0.3, 0.1])
    C = fsg.Context()
    rng = np.random.default_rng(77)
    dev = torch.device("cuda", 0)
    for call in range(2):          # the second call runs on work arrays holding the first's data
        nprof = 300 + 50 * call
        xki = 10 ** rng.uniform(-3, 2, (nprof, nt)) * np.linspace(1, 40, nt)
        src = 1e14 * (1 + rng.uniform(0, 1, (nprof, nt))) * np.linspace(1, 3, nt)
        ref = C.locprf_pp(x, xki, src, rhox)
        d = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in
             (("xmu", x), ("xki", xki), ("src", src), ("rhox", rhox))}
        out = torch.full((nprof, len(x)), np.nan, dtype=torch.float64, device=dev)
        rc = lib.fsg_locprf_pp_noalloc(nprof, len(x), d["xmu"].data_ptr(), nt, d["xki"].data_ptr(),
                                       d["src"].data_ptr(), d["rhox"].data_ptr(), out.data_ptr(), None)
        assert rc == 0
        got = out.cpu().numpy()
        # same kernel, same inputs: identical values (the tolerance of the solver tests is 1e-10)
        np.testing.assert_allclose(got, ref, rtol=1e-10, atol=0)
        assert np.array_equal(got, ref)


def test_noalloc_rejects_sizes_beyond_its_work_array(fsg):
    import torch
    lib = fsg.lib()
    nt, nmu = 100, 3
    nprof = (1 << 20) // (3 * nt) + 1
    dev = torch.device("cuda", 0)
    buf = torch.zeros(16, dtype=torch.float64, device=dev)
    p = buf.data_ptr()
    assert lib.fsg_locprf_pp_noalloc(nprof, nmu, p, nt, p, p, p, p, None) == -1


def _noalloc_vs_allocating(fsg, lib, dev, stream, seed):
    """One call of each entry point on device dev (current while it runs), the no-allocation one on
    the given stream (a cudaStream_t as an integer, or None for the default stream)."""
    import torch
    st, _ = H.load_atm("solar")
    rhox = np.asarray(st["rhox"], np.float64)
    nt = len(rhox)
    x = np.array([1.0, 0.7, 0.4, 0.15])
    rng = np.random.default_rng(seed)
    nprof = 257
    xki = 10 ** rng.uniform(-3, 2, (nprof, nt)) * np.linspace(1, 40, nt)
    src = 1e14 * (1 + rng.uniform(0, 1, (nprof, nt))) * np.linspace(1, 3, nt)
    C = fsg.Context(device=dev.index)
    ref = C.locprf_pp(x, xki, src, rhox)
    C.close()
    d = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in
         (("xmu", x), ("xki", xki), ("src", src), ("rhox", rhox))}
    out = torch.full((nprof, len(x)), np.nan, dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    rc = lib.fsg_locprf_pp_noalloc(nprof, len(x), d["xmu"].data_ptr(), nt, d["xki"].data_ptr(),
                                   d["src"].data_ptr(), d["rhox"].data_ptr(), out.data_ptr(), stream)
    assert rc == 0
    torch.cuda.synchronize(dev)
    got = out.cpu().numpy()
    np.testing.assert_allclose(got, ref, rtol=1e-10, atol=0)
    assert np.array_equal(got, ref)


def test_noalloc_on_a_caller_stream(fsg):
    """The caller's own (non-default) stream, twice in a row."""
    import torch
    dev = torch.device("cuda", 0)
    s = torch.cuda.Stream(device=dev)
    for k in range(2):
        _noalloc_vs_allocating(fsg, fsg.lib(), dev, s.cuda_stream, 91 + k)


def test_noalloc_on_a_second_device(fsg):
    """With a second GPU current, the array's address is looked up for that device (its own copy)."""
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("one GPU visible")
    for idx in (1, 0, 1):
        dev = torch.device("cuda", idx)
        with torch.cuda.device(dev):
            _noalloc_vs_allocating(fsg, fsg.lib(), dev, None, 101 + idx)
