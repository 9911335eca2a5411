"""The C-ABI library: it loads, exports every symbol include/fastspec_gpu.h declares, and its
host set-up routines (grid, quadrature, Zeeman patterns) match the oracle.  No device calls."""
import ctypes
import os
import re

import numpy as np

import helpers as H


def declared_symbols():
    src = open(os.path.join(H.REPO, "include", "fastspec_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(fsg_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_header(fsg):
    lib = ctypes.CDLL(fsg.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 25
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    assert set(fsg.EXPORTS) <= set(syms)


def test_make_grid_matches_oracle(fsg, oracle_mod):
    for grid in (dict(wmode=0, wstart=5000.0, wend=5200.0, dstep=0.005),
                 dict(wmode=1, wstart=5000.0, wend=5100.0, dstep=0.3),
                 dict(wmode=0, wstart=6000.0, wend=6000.004, dstep=0.002)):
        w = fsg.make_grid(grid["wmode"], grid["wstart"], grid["wend"], grid["dstep"])
        st, _ = H.load_atm("solar")
        ref = oracle_mod.State(grid, st).wave
        assert np.array_equal(w, ref)


def test_make_grid_rejects_bad(fsg):
    import pytest
    with pytest.raises(fsg.FsgError):
        fsg.make_grid(0, 5000.0, 5000.001, 0.005)
    with pytest.raises(fsg.FsgError):
        fsg.make_grid(3, 5000.0, 5100.0, 0.1)


def test_quadrature_matches_oracle(fsg, oracle_mod):
    for q in (0, 1, 2):
        for n in (1, 2, 5, 7, 9):
            a = fsg.mu_quadrature(q, n)
            b = oracle_mod.mu_quadrature(q, n)
            for x, y in zip(a, b):
                assert np.array_equal(x, y)


def test_zeeman_pattern_matches_oracle(fsg, oracle_mod):
    rng = np.random.default_rng(3)
    for _ in range(200):
        jlo = float(rng.integers(0, 5)); jup = float(np.clip(jlo + rng.integers(-1, 2), 0, 4))
        if jlo == 0 and jup == 0:
            continue
        glo, gup = (np.float32(x) for x in rng.uniform(0, 2.5, 2))
        a = fsg.zeeman_pattern(jlo, jup, glo, gup)
        b = oracle_mod.zeeman_pattern(jlo, jup, glo, gup)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


def test_mu_quad_type(fsg):
    """MuQuadType (utils.f90:1337-1354): which rule the angles of an intensity file follow."""
    for q in (1, 2):
        for n in (2, 5, 9):
            x, _, _ = fsg.mu_quadrature(q, n)
            assert fsg.mu_quad_type(x) == q
            assert fsg.mu_quad_type(x + 2e-6) == 0
    assert fsg.mu_quad_type([1.0]) == 0
    assert fsg.mu_quad_type([0.9, 0.5, 0.1]) == 0

