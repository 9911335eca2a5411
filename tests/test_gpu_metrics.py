"""Tracing and metrics of the driver calls: with FSG_METRICS_JSONL naming a file, every driver call
appends one JSON line with its status, its wall time and the stage figures it returned -- what the
reference prints per stage (lines read and used, time of the line opacity and of the radiative
transfer, fastspec.f90:393-425).  Without the variable nothing is written."""
import json
import os

import pytest

import helpers as H

pytestmark = pytest.mark.gpu


def small_context(fsg, cont=True):
    st, meta = H.load_atm("solar")
    w0, w1, step = 5000.0, 5005.0, 0.005
    C = fsg.Context(precision=fsg.PREC_MIXED, vmicro=1.0)
    C.set_grid(0, w0, w1, step)
    C.set_atmosphere(st)
    if cont:
        C.set_contopac(H.contopac_on(meta, fsg.make_grid(0, w0, w1, step) + w0))
    x, w, _ = fsg.mu_quadrature(1, 7)
    C.set_mu(x, w)
    return C


def test_metrics_lines_follow_the_calls(fsg, tmp_path, monkeypatch):
    from fastspec_b200 import workloads as W
    path = tmp_path / "metrics.jsonl"
    monkeypatch.setenv("FSG_METRICS_JSONL", str(path))
    arr = W.atomic_lines(500, 5000.0, 5005.0, W.SEED0 + 80).arrays()
    C = small_context(fsg)
    r = C.lineop_calc(fsg.LineList.from_arrays(arr), want_lineopac=False, want_lines=False)
    C.radtran()
    nwl, ntau, nmu = C.nwl, C.ntau, C.nmu
    C.close()
    B = small_context(fsg, cont=False)                 # a refused call still leaves its line
    with pytest.raises(fsg.FsgError):
        B.lineop_calc(fsg.LineList.from_arrays(arr))
    B.close()
    rec = [json.loads(line) for line in open(path)]
    assert [x["call"] for x in rec] == ["fsg_lineop_calc", "fsg_radtran", "fsg_lineop_calc"]
    lo, rt, bad = rec
    s = r["stats"]
    assert lo["rc"] == 0 and lo["wall_ms"] > 0
    for k in ("nlines_in", "nlines_used", "nwide", "nweak", "line_evals", "core_evals"):
        assert lo[k] == s[k], k
    assert abs(lo["ms_total"] - s["ms_total"]) < 1e-3
    assert rt["rc"] == 0 and (rt["nwl"], rt["ntau"], rt["nmu"]) == (nwl, ntau, nmu)
    assert bad["rc"] != 0 and "nlines_in" not in bad


def test_no_metrics_without_the_variable(fsg, tmp_path, monkeypatch):
    from fastspec_b200 import workloads as W
    monkeypatch.delenv("FSG_METRICS_JSONL", raising=False)
    monkeypatch.chdir(tmp_path)
    C = small_context(fsg)
    C.lineop_calc(fsg.LineList.from_arrays(W.atomic_lines(100, 5000.0, 5005.0, W.SEED0 + 81).arrays()))
    C.radtran()
    C.close()
    assert os.listdir(tmp_path) == []
