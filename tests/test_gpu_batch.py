"""Batched synthesis on the GPU (fsg_batch_*): each atmosphere's flux against the oracle run on the
whole shared list as the reference would read it for that atmosphere's deck (the lines with centres
in [Wstart, Wend], ioutils.f90:752-753, 1496-1497; mixed-path flux tolerance 1e-5) and against the
single-context path; with a margin, against the oracle on the lines the margin adds; graph replays
are deterministic; a given tuning is applied."""
import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu


def small_batch(fsg, natm=4, span=3.0, nlines=120_000, seed=5):
    from fastspec_b200 import workloads as W
    import fastspec_b200 as F
    members = W.batch_grid(natm, seed=W.SEED0 + 50 + seed)
    lines = W.atomic_lines(nlines, 3000.0, 9000.0, W.SEED0 + 60 + seed)
    order = np.argsort(lines.arrays()["wl"], kind="stable")
    arr = {k: np.ascontiguousarray(v[order]) for k, v in lines.arrays().items()}
    ctxs, cases = [], []
    x, w, _ = fsg.mu_quadrature(1, 7)
    for m in members:
        g = dict(m["grid"])
        g["wend"] = g["wstart"] + span
        wave = F.make_grid(1, g["wstart"], g["wend"], g["dstep"]) + g["wstart"]
        co = H.contopac_on(m["cont"], wave)
        C = fsg.Context(vmicro=1.0)
        C.set_grid(1, g["wstart"], g["wend"], g["dstep"])
        C.set_atmosphere(m["state"])
        C.set_contopac(co)
        C.set_mu(x, w)
        ctxs.append(C)
        cases.append((g, m["state"], co))
    return ctxs, cases, arr


def candidates(arr, g, margin=0.0):
    sel = (arr["wl"] >= g["wstart"] - margin) & (arr["wl"] <= g["wend"] + margin)
    return {k: np.ascontiguousarray(v[sel]) for k, v in arr.items()}


@pytest.mark.parametrize("margin", [0.0, 2.0])
def test_batch_flux_vs_oracle_and_single_context(fsg, oracle_mod, margin):
    ctxs, cases, arr = small_batch(fsg)
    B = fsg.Batch(ctxs, fsg.LineList.from_arrays(arr), margin=margin)
    st = B.run()
    assert st["natm"] == len(ctxs) and st["line_evals"] > 0 and st["ms_total"] > 0
    assert st["tuning"]["tile_pix"] in (64, 128)
    x, w, _ = oracle_mod.mu_quadrature(1, 7)
    ncand = 0
    for i, (g, state, co) in enumerate(cases):
        sfl, sfc = B.flux(i)
        # margin 0: the oracle reads the whole shared list with the reference's WAVE= selection
        cand = (oracle_mod.reader_select(arr, g["wstart"], g["wend"]) if margin == 0.0
                else candidates(arr, g, margin))
        ncand += len(cand["wl"])
        S = oracle_mod.State(g, state, contopac=co, vmicro=1.0)
        r = oracle_mod.lineop_calc(S, oracle_mod.Lines(**cand, kind=2), list_type=2)
        osfl, osfc = oracle_mod.disk_integ(w, *oracle_mod.radtran(S, x, r["lineopac"]))
        assert np.max(np.abs(sfl / osfl - 1)) < 1e-5
        assert np.max(np.abs(sfc / osfc - 1)) < 1e-9
        # the single-context mixed path on the same candidate list
        C = ctxs[i]
        C.lineop_reset()
        C.lineop_calc(fsg.LineList.from_arrays(cand), want_lineopac=False, want_lines=False)
        _, _, csfl, _ = C.radtran()
        assert np.max(np.abs(sfl / csfl - 1)) < 1e-6
    assert st["nlines_candidate"] == ncand
    B.close()


def test_batch_replay_and_given_tuning(fsg):
    ctxs, cases, arr = small_batch(fsg, natm=3, seed=6)
    B = fsg.Batch(ctxs, fsg.LineList.from_arrays(arr))
    B.run()
    f1 = [B.flux(i)[0] for i in range(3)]
    B.run()
    f2 = [B.flux(i)[0] for i in range(3)]
    for a, b in zip(f1, f2):
        assert np.array_equal(a, b)
    B.set_tuning({"tile_pix": 64, "wing_ctas": 148, "core_ctas": 296})
    st = B.run()
    assert st["tuning"]["tile_pix"] == 64 and st["tuning"]["core_ctas"] == 296
    f3 = [B.flux(i)[0] for i in range(3)]
    for a, b in zip(f1, f3):
        assert np.max(np.abs(a / b - 1)) < 1e-6
    B.close()


def test_batch_spherical_member(fsg):
    """An atmosphere given a spherical geometry inside a batch is solved along its rays (LocPrfSph,
    solver.f90:182-261) in the batch's graph: its flux equals the single-context spherical synthesis of
    the same lines, and the plane-parallel members are unchanged."""
    ctxs, cases, arr = small_batch(fsg, natm=3, seed=9)
    g1, st1, _ = cases[1]
    rhox, rho = np.asarray(st1["rhox"], float), np.asarray(st1["rho"], float)
    h = np.zeros(len(rhox))                                  # hydrostatic heights, decreasing inward
    for k in range(1, len(rhox)):
        h[k] = h[k - 1] - (rhox[k] - rhox[k - 1]) / (0.5 * (rho[k] + rho[k - 1]))
    h -= h[-1]
    ctxs[1].set_geometry(3.0e11, h)
    B = fsg.Batch(ctxs, fsg.LineList.from_arrays(arr))
    B.run()
    for i, (g, state, co) in enumerate(cases):
        sfl, sfc = B.flux(i)
        C = ctxs[i]
        C.lineop_reset()
        C.lineop_calc(fsg.LineList.from_arrays(candidates(arr, g)), want_lineopac=False, want_lines=False)
        _, _, csfl, csfc = C.radtran()
        assert np.max(np.abs(sfl / csfl - 1)) < 1e-6, i
        assert np.max(np.abs(sfc / csfc - 1)) < 1e-12, i
    B.close()


def test_batch_rejects_bad_inputs(fsg):
    ctxs, cases, arr = small_batch(fsg, natm=2, seed=7, nlines=2000)
    bad = {k: v[::-1].copy() for k, v in arr.items()}                  # not sorted
    with pytest.raises(fsg.FsgError):
        fsg.Batch(ctxs, fsg.LineList.from_arrays(bad))
    C = fsg.Context(precision=fsg.PREC_FP64)
    with pytest.raises(fsg.FsgError):
        fsg.Batch([C], fsg.LineList.from_arrays(arr))


def test_batch_axis_shares(fsg):
    """Batch-axis sharding (fastspec_b200.shard) with the batched CUDA path as backend: the two shares
    of a 2-rank cost partition, each run as its own batched graph, give every atmosphere's flux of the
    whole batch (1e-6: the tuner may tile a different batch differently; continuum 1e-12); run_batch in
    a process group of one (gloo, fluxes gathered on the host) returns them in the grid's order."""
    import socket
    import torch.distributed as dist
    from fastspec_b200 import shard
    ctxs, cases, arr = small_batch(fsg, natm=5, seed=8)
    lines = fsg.LineList.from_arrays(arr)
    B = fsg.Batch(ctxs, lines)
    B.run()
    whole = [np.stack(B.flux(i)) for i in range(len(ctxs))]
    B.close()
    sizes = [c.nwl for c in ctxs]
    costs = [shard.batch_cost(c.nwl, c.ntau, len(candidates(arr, g)["wl"])) for c, (g, _, _) in zip(ctxs, cases)]
    x, w, _ = fsg.mu_quadrature(1, 7)

    def make_context(i):
        g, state, co = cases[i]
        C = fsg.Context(vmicro=1.0)
        C.set_grid(1, g["wstart"], g["wend"], g["dstep"])
        C.set_atmosphere(state)
        C.set_contopac(co)
        C.set_mu(x, w)
        return C

    def check(i, f):
        f = f.cpu().numpy()
        assert f.shape == whole[i].shape
        assert np.max(np.abs(f[0] / whole[i][0] - 1)) < 1e-6
        assert np.max(np.abs(f[1] / whole[i][1] - 1)) < 1e-12

    parts = shard.batch_partition(costs, 2)
    assert all(parts) and sorted(sum(parts, [])) == list(range(len(ctxs)))
    for p in parts:
        be = shard.BatchGpuBackend(fsg, make_context, lines, "cuda")
        for i, f in zip(p, be.synthesize(p)):
            check(i, f)
        be.batch.close()
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=0, world_size=1)
    try:
        be = shard.BatchGpuBackend(fsg, make_context, lines, "cpu")
        res, mine = shard.run_batch(be, costs, sizes)
        be.batch.close()
    finally:
        dist.destroy_process_group()
    assert mine == list(range(len(ctxs)))
    for i, f in enumerate(res):
        check(i, f)
