#!/usr/bin/env python3
"""Benchmark of the line-opacity -> formal-solver path on the cool-dwarf molecular synthesis.

Workload (one step = one full synthesis): Teff 3500 K, log g 5.0, 72 depths; 1e8 synthetic
molecular lines (TiO/H2O/CO/OH-like, lambda0 uniform in wavenumber over 0.5-2.5 um, log gf ~
N(-5, 1.5), E_low ~ Exp(1 eV) capped at 5 eV, log G6/NH ~ U(-8, -7)); R = 3e5 sampling
(ln-lambda grid, 482,832 points); vmic 1 km/s; 7 Gauss-Legendre angles; flux quadrature.
A step is LineopCalc (central pass over all lines, windows, accumulation) + RadTranCalc +
disk integration.  Inputs (3.6 GB of line records, 278 MB of continuum opacity) exceed the
126 MB L2, so no flush is needed between steps.

Metric: Voigt line-evals/s (evaluations inside the reference's windows: Ntau x window length
summed over retained lines), plus spectra/s.  `value` times the mixed-precision path with the
line list resident in HBM; `e2e` times the public C-ABI call with host (pinned) buffers, the
host->device copy of the line list and the device->host read of the flux inside each step.

--impl reference: the reference's CPU implementation of the path timed on this host: its own
OpenMP executable (copied unmodified to baseline/_ref by the build; there is no Fortran compiler to
build it) on all host threads, on a bounded wavelength sample of the same workload, or, without the
executable, the FP64 C restatement (oracle/) with OpenMP.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(HERE, "tests"))

METRIC = "Voigt line-evals/s (cool-dwarf 1e8-line synthesis)"
UNIT = "line-evals/s"
FLOPS_PER_EVAL = 12          # nominal FP32 work of one wing evaluation (v^2, rational, scale, sum)
W0, W1, DSTEP, NMU = 5000.0, 25000.0, 1.0, 7


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="fastspec_b200", choices=["fastspec_b200", "reference"])
    p.add_argument("--lines", type=float, default=1e8)
    p.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--no-plain", action="store_true", help="skip the plain FP64 path comparison")
    p.add_argument("--shard", action="store_true",
                   help="run the wavelength-sharded synthesis even on one GPU (a process group of one)")
    p.add_argument("--plain-lines", type=float, default=1e6)
    p.add_argument("--no-batched", action="store_true", help="skip the batched-grid measurement")
    p.add_argument("--batch-atm", type=int, default=256)
    p.add_argument("--batch-lines", type=float, default=2e6)
    p.add_argument("--no-fit", action="store_true", help="skip the differentiable-fit measurement")
    p.add_argument("--no-stokes", action="store_true", help="skip the polarised (Stokes) synthesis measurement")
    return p.parse_args()


def load_atmosphere():
    import helpers as H
    return H.load_atm("cooldwarf")


def contopac_for(meta, wave_abs):
    import helpers as H
    return H.contopac_on(meta, wave_abs)


# ---- clocks sampled during the timed region ------------------------------------------------------
class ClockSampler:
    def __init__(self, gpu_index=0):
        self.samples = []
        self._stop = threading.Event()
        self._idx = gpu_index

    def _run(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self._idx), "--query-gpu=" + q,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for k, nm in enumerate(names):
                if len(s) > 5 + k and s[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


# ---- GPU arm -------------------------------------------------------------------------------------
def device_lines(F, torch, arr, dev):
    """Device copies of a line list and the fsg_lines view of them (kind 2, molecular SoA)."""
    dt = {k: torch.from_numpy(np.ascontiguousarray(v)).to(f"cuda:{dev}") for k, v in arr.items()}
    dl = F.CLines()
    dl.n = int(dt["wl"].numel())
    dl.kind = 2
    dl.wl = F.C.cast(dt["wl"].data_ptr(), F._dp)
    for k in ("elo", "gf", "grad", "gqst", "gvdw"):
        setattr(dl, k, F.C.cast(dt[k].data_ptr(), F._fp))
    dl.spc = F.C.cast(dt["spc"].data_ptr(), F._ip)
    dl.ismol = F.C.cast(dt["ismol"].data_ptr(), F._ip)
    return dt, dl


def plain_vs_mixed(F, torch, st, meta, co, dev, nlines):
    """The same synthesis through the plain FP64 path and the mixed path on a smaller list with the
    same distributions over the full grid: line-evals/s of each, and the flux difference."""
    from fastspec_b200 import workloads as W
    arr = W.molecular_lines(nlines, W0, W1, W.SEED0 + 7, exact=False).arrays()
    x, w, _ = F.mu_quadrature(1, NMU)
    out = {}
    flux = {}
    for name, prec in (("fp64", F.PREC_FP64), ("mixed", F.PREC_MIXED)):
        C = F.Context(device=dev, precision=prec, vmicro=meta["vmicro"], molbrd=meta["molbrd"], limitram_gb=24.0)
        C.set_grid(1, W0, W1, DSTEP)
        C.set_atmosphere(st)
        C.set_contopac(co)
        C.set_mu(x, w)
        dt, dl = device_lines(F, torch, arr, dev)
        sfl = torch.empty(C.nwl, dtype=torch.float64, device=f"cuda:{dev}")
        sfc = torch.empty_like(sfl)
        stream = torch.cuda.ExternalStream(C.stream_ptr(), device=dev)

        def step():
            C.lineop_reset()
            s_ = C.lineop_calc_dev(dl)
            C.radtran_dev(None, None, sfl.data_ptr(), sfc.data_ptr())
            return s_

        step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s_ = step()
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        ev = s_["line_evals"] if prec == F.PREC_MIXED else None
        out[name] = {"ms": ms, "ms_accum": s_["ms_accum"], "stats_evals": s_["line_evals"]}
        flux[name] = sfl.cpu().numpy() / sfc.cpu().numpy()
        if ev is not None:
            out["evals"] = ev
        C.close()
    ev = out["evals"]
    return {"sample": "%d lines, same distributions, full grid" % nlines,
            "fp64_value": ev / (out["fp64"]["ms"] / 1e3), "mixed_value": ev / (out["mixed"]["ms"] / 1e3),
            "unit": UNIT, "speedup": out["fp64"]["ms"] / out["mixed"]["ms"],
            "fp64_ms": out["fp64"]["ms"], "mixed_ms": out["mixed"]["ms"],
            "flux_max_rel_diff": float(np.max(np.abs(flux["mixed"] / flux["fp64"] - 1.0)))}


def batched_grid(F, torch, dev, natm, nlines, steps, warmup):
    """The batched configuration: natm atmospheres (depths 48-80, Teff 3800-7500 K, spans 20-200 A at
    R = 5e5) sharing one atomic list of nlines over 3000-9000 A, synthesised by one CUDA-graph
    replay of fsg_batch_run (persistent work-queue kernels, tiles from the autotuner); compared with
    the same atmospheres synthesised one context at a time through fsg_lineop_calc_dev, and with the
    plain FP64 path on a sample of eight of them."""
    from fastspec_b200 import workloads as W
    members = W.batch_grid(natm)
    lines = W.atomic_lines(int(nlines), 3000.0, 9000.0, W.SEED0 + 3, exact=False)
    arr = lines.arrays()
    order = np.argsort(arr["wl"], kind="stable")
    arr = {k: np.ascontiguousarray(v[order]) for k, v in arr.items()}
    LL = F.LineList.from_arrays(arr)
    x, w, _ = F.mu_quadrature(1, NMU)
    ctxs, conts = [], []
    for m in members:
        g = m["grid"]
        wave = F.make_grid(1, g["wstart"], g["wend"], g["dstep"]) + g["wstart"]
        lk = np.log(m["cont"]["cont_opac"])
        co = np.exp(np.stack([np.interp(wave, m["cont"]["cont_wave"], lk[:, t]) for t in range(m["ntau"])], axis=1))
        conts.append(co)
        C = F.Context(device=dev, vmicro=1.0)
        C.set_grid(1, g["wstart"], g["wend"], g["dstep"])
        C.set_atmosphere(m["state"])
        C.set_contopac(co)
        C.set_mu(x, w)
        ctxs.append(C)
    B = F.Batch(ctxs, LL)                          # each atmosphere reads the lines of its span
    t0 = time.perf_counter()
    tuning = B.tune()
    tune_s = time.perf_counter() - t0
    st = B.run()                                   # captures the graph
    for _ in range(max(0, warmup - 1)):
        B.run()
    bs = torch.cuda.ExternalStream(B.stream_ptr(), device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(bs)
    for _ in range(steps):
        st = B.run()
    e1.record(bs)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    # the same atmospheres one context at a time (device line list per atmosphere's candidates)
    wl = arr["wl"]
    t_seq = 0.0
    for C, m in zip(ctxs, members):
        g = m["grid"]
        a0, a1 = np.searchsorted(wl, g["wstart"]), np.searchsorted(wl, g["wend"], side="right")
        sub = F.LineList.from_arrays({k: np.ascontiguousarray(v[a0:a1]) for k, v in arr.items()})
        C.lineop_reset()
        r = C.lineop_calc(sub, want_lineopac=False, want_lines=False)
        t_seq += r["stats"]["ms_total"]
    # the plain FP64 path on every natm/8-th atmosphere, one context at a time (line opacity only: the
    # solver is left out of its time, which favours the FP64 side of the ratio)
    samp = list(range(0, natm, max(1, natm // 8)))
    t64 = 0.0
    for k in samp:
        m, g = members[k], members[k]["grid"]
        C64 = F.Context(device=dev, precision=F.PREC_FP64, vmicro=1.0)
        C64.set_grid(1, g["wstart"], g["wend"], g["dstep"])
        C64.set_atmosphere(m["state"])
        C64.set_contopac(conts[k])
        C64.set_mu(x, w)
        a0, a1 = np.searchsorted(wl, g["wstart"]), np.searchsorted(wl, g["wend"], side="right")
        sub = F.LineList.from_arrays({kk: np.ascontiguousarray(v[a0:a1]) for kk, v in arr.items()})
        r = C64.lineop_calc(sub, want_lineopac=False, want_lines=False)
        t64 += r["stats"]["ms_total"]
        C64.close()
    fp64_sps = len(samp) / (t64 / 1e3)
    nwl_tot = sum(c.nwl for c in ctxs)
    out = {"config": "%d atmospheres (48-80 depths, Teff 3800-7500 K, spans 20-200 A at R=5e5, %d wavelengths in all), "
                     "%d shared atomic lines 3000-9000 A, 7 mu" % (natm, nwl_tot, int(nlines)),
           "spectra_per_s": natm / (ms / 1e3), "line_evals_per_s": st["line_evals"] / (ms / 1e3),
           "ms_per_batch": ms, "line_evals": st["line_evals"], "candidate_lines": st["nlines_candidate"],
           "tuning": tuning, "tuning_s": tune_s, "graph": True,
           "sequential_line_ms": t_seq,
           "plain_fp64_sample": {"atmospheres": len(samp), "spectra_per_s": fp64_sps,
                                 "ms_line_per_atmosphere": t64 / len(samp)},
           "batched_over_plain_fp64": (natm / (ms / 1e3)) / fp64_sps,
           "note": "sequential_line_ms: the same line opacities one context at a time (fsg_lineop_calc, "
                   "device time of central pass + accumulation, no solver)"}
    B.close()
    for C in ctxs:
        C.close()
    return out


def differentiable_fit(F, torch, dev, steps, warmup):
    """The differentiable fit: the solar-like atmosphere with 1e5 atomic lines over 4800-5300 A
    (0.005 A), a target synthesised at perturbed abundances (N(0, 0.1) dex on the elements with
    lines) and log gf (N(0, 0.05)) plus noise at S/N 300; one step = forward synthesis + chi-square +
    adjoint gradients with respect to 30 abundances, 1e5 log gf and vmicro."""
    from fastspec_b200 import workloads as W
    from fastspec_b200 import adjoint as AD
    d = np.load(os.path.join(HERE, "fastspec_b200", "data", "atm_solar.npz"))
    st = {k: d[k] for k in ("rhox", "T", "xne", "xna", "rho", "fractionpf", "xamass", "potion", "ion", "frac_h1",
                            "frac_he1")}
    species = [str(x) for x in d["species"]]
    w0, w1, step = 4800.0, 5300.0, 0.005
    grid = dict(wmode=0, wstart=w0, wend=w1, dstep=step)
    wave = F.make_grid(0, w0, w1, step) + w0
    lk = np.log(d["cont_opac"])
    co = np.exp(np.stack([np.interp(wave, d["cont_wave"], lk[:, t]) for t in range(lk.shape[1])], axis=1))
    arr = W.atomic_lines(100_000, w0 - 0.5, w1 + 0.5, W.SEED0 + 4, exact=False).arrays()
    M = AD.FluxModel(F, grid, st, co, arr, species, vmicro=float(d["vmicro"]), device=dev)
    loggf0 = np.log10(arr["gf"].astype(np.float64))
    rng = np.random.default_rng(W.SEED0 + 4)
    ne = len(AD.ELEMENTS)
    dab = np.zeros(ne)
    for e in sorted(set(s.split()[0] for s in species)):
        dab[AD.ELEMENTS.index(e)] = rng.normal(0.0, 0.1)
    with torch.no_grad():
        f_t = AD.synth_flux(M, torch.tensor(loggf0 + rng.normal(0, 0.05, len(loggf0))), torch.tensor(dab),
                            torch.tensor(float(d["vmicro"])))
        fobs = f_t + torch.tensor(rng.normal(0, 1.0 / 300.0, f_t.numel()), device=f_t.device)

    def step_fn():
        lg = torch.tensor(loggf0, requires_grad=True)
        da = torch.zeros(ne, dtype=torch.float64, requires_grad=True)
        vm = torch.tensor(float(d["vmicro"]), dtype=torch.float64, requires_grad=True)
        f = AD.synth_flux(M, lg, da, vm)
        c = (((f - fobs) * 300.0) ** 2).sum()
        c.backward()
        return float(c.detach()), lg.grad, da.grad, vm.grad

    def forward_only():
        with torch.no_grad():
            f = AD.synth_flux(M, torch.tensor(loggf0), torch.zeros(ne, dtype=torch.float64),
                              torch.tensor(float(d["vmicro"])))
            return float((((f - fobs) * 300.0) ** 2).sum())

    for _ in range(warmup):
        step_fn()
        forward_only()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        forward_only()
    torch.cuda.synchronize()
    ms_fwd = (time.perf_counter() - t0) * 1e3 / steps
    t0 = time.perf_counter()
    for _ in range(steps):
        c, gl, ga, gv = step_fn()
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t0) * 1e3 / steps
    out = {"config": "solar-like 56-depth atmosphere, 1e5 atomic lines 4800-5300 A at 0.005 A (%d wavelengths), "
                     "7 mu; chi-square gradients w.r.t. 30 abundances, 1e5 log gf, vmicro" % M.C.nwl,
           "steps_per_s": 1e3 / ms, "ms_per_step": ms, "ms_forward": ms_fwd, "gradient_cost_over_forward": ms / ms_fwd,
           "chi2": c, "n_params": int(len(loggf0) + ne + 1),
           "grad_norm_loggf": float(torch.linalg.norm(gl)), "grad_vmicro": float(gv),
           "timing": "wall clock of forward + adjoint per step with device synchronisation"}
    M.close()
    return out


def stokes_synthesis(F, torch, dev, steps, warmup):
    """The polarised configuration: 5000 Zeeman lines over 6000-6100 A at 0.002 A (50,001
    wavelengths), the Teff = 5000 K, log g = 4.5 atmosphere (56 depths), BFRAME 1 with |B| = 2 kG at
    inclination 60 deg and azimuth 30 deg, 9 angles: MagLineopCalc (FP64) + MagRadTranCalc (4x4
    DELO-Bezier) + Stokes-I flux, host arrays in and out."""
    from fastspec_b200 import workloads as W
    d = np.load(os.path.join(HERE, "fastspec_b200", "data", "atm_magnetic.npz"))
    st = {k: d[k] for k in ("rhox", "T", "xne", "xna", "rho", "fractionpf", "xamass", "potion", "ion", "frac_h1",
                            "frac_he1")}
    w0, w1, step = 6000.0, 6100.0, 0.002
    wave = F.make_grid(0, w0, w1, step) + w0
    lk = np.log(d["cont_opac"])
    co = np.exp(np.stack([np.interp(wave, d["cont_wave"], lk[:, t]) for t in range(lk.shape[1])], axis=1))
    L = W.zeeman_lines(5000, w0, w1, W.SEED0 + 2)
    z = W.zeeman_components(L, F.zeeman_pattern)
    LL = F.LineList.from_arrays(L.arrays(), zeeman=z)
    x, w, _ = F.mu_quadrature(1, 9)
    bf = [2000.0, 60.0, 30.0]
    out = {"config": "5000 Zeeman lines 6000-6100 A at 0.002 A, 56 depths, BFRAME 1 2 kG 60/30 deg, 9 mu, "
                     "4x4 DELO-Bezier; host arrays in and out",
           "timing": "wall clock per Stokes IQUV synthesis (MagLineopCalc + MagRadTranCalc + Stokes-I flux)"}
    spz = {}
    for name, prec in (("fp64", F.PREC_FP64), ("mixed", F.PREC_MIXED)):
        C = F.Context(device=dev, precision=prec, vmicro=float(d["vmicro"]))
        C.set_grid(0, w0, w1, step)
        C.set_atmosphere(st)
        C.set_contopac(co)
        C.set_mu(x, w)

        def one():
            C._ck(C._lib.fsg_mag_lineop_reset(C.h), "reset")
            r = C.mag_lineop_calc(LL, 1, bf, want=False)
            sp = C.mag_radtran(1, bf)
            return r["stats"], sp

        for _ in range(warmup):
            one()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(steps):
            stt, sp = one()
        ms = (time.perf_counter() - t0) * 1e3 / steps
        spz[name] = sp
        out[name] = {"spectra_per_s": 1e3 / ms, "ms_per_spectrum": ms, "ms_lineop": stt["ms_total"],
                     "ms_center": stt["ms_center"], "ms_accum": stt["ms_accum"],
                     "line_evals": stt["line_evals"], "line_evals_per_s": stt["line_evals"] / (stt["ms_total"] / 1e3)}
        out["nwl"] = C.nwl
        C.close()
    a, b = spz["mixed"], spz["fp64"]
    out["mixed_vs_fp64"] = {"stokes_I_max_rel": float(np.max(np.abs(a[0][:, 0] / b[0][:, 0] - 1))),
                            "stokes_QUV_max_over_Ic": float(max(np.max(np.abs(a[0][:, q] - b[0][:, q]) / b[1])
                                                                for q in (1, 2, 3))),
                            "flux_max_rel": float(np.max(np.abs(a[2] / b[2] - 1)))}
    return out


def run_gpu(args, rank, world):
    import torch
    import fastspec_b200 as F
    from fastspec_b200 import workloads as W

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    st, meta = load_atmosphere()
    wave = F.make_grid(1, W0, W1, DSTEP)
    co = contopac_for(meta, wave + W0)
    nlines = int(args.lines)
    L = W.molecular_lines(nlines, W0, W1, W.SEED0 + 1, exact=False)
    arr = L.arrays()
    x, w, _ = F.mu_quadrature(1, NMU)
    prec = F.PREC_MIXED if args.precision == "mixed" else F.PREC_FP64
    C = F.Context(device=dev, precision=prec, vmicro=meta["vmicro"], molbrd=meta["molbrd"], limitram_gb=24.0)
    C.set_grid(1, W0, W1, DSTEP)
    C.set_atmosphere(st)
    C.set_contopac(co)
    C.set_mu(x, w)
    nwl, ntau = C.nwl, C.ntau
    stream = torch.cuda.ExternalStream(C.stream_ptr(), device=dev)

    # resident device copies of the line list (value arm)
    dt, dl = device_lines(F, torch, arr, dev)
    spl = torch.empty((nwl, NMU), dtype=torch.float64, device=f"cuda:{dev}")
    spc = torch.empty_like(spl)
    sfl = torch.empty(nwl, dtype=torch.float64, device=f"cuda:{dev}")
    sfc = torch.empty_like(sfl)

    sharded = {}
    use_shard = world > 1 or args.shard
    if use_shard:
        # one synthesis split along the wavelength axis over the ranks (fastspec_b200.shard)
        from fastspec_b200 import shard
        backend = shard.GpuBackend(F, C, dt)
        zero = F.Stats().asdict()

        def step_resident():
            res = shard.run(backend)
            sharded["res"] = res
            return res["stats"] or zero
    else:
        def step_resident():
            C.lineop_reset()
            s = C.lineop_calc_dev(dl)
            C.radtran_dev(spl.data_ptr(), spc.data_ptr(), sfl.data_ptr(), sfc.data_ptr())
            return s

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    def timed(fn, steps):
        # one GPU: everything runs on the library's stream.  Sharded: library calls return after
        # their stream is done, the collectives run on torch's stream; events go on torch's
        # stream after a device synchronise so they bracket both
        ev_stream = stream if not use_shard else torch.cuda.current_stream(dev)
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(ev_stream)
        stats = [fn() for _ in range(steps)]
        if use_shard:
            torch.cuda.synchronize()
        e1.record(ev_stream)
        e1.synchronize()
        barrier()
        ms = e0.elapsed_time(e1)
        if world > 1:
            import torch.distributed as dist
            t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{dev}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms, stats

    for _ in range(args.warmup):
        step_resident()
    l0 = C.launches()
    with ClockSampler(dev) as clk:
        ms, stats = timed(step_resident, args.steps)
    launches = C.launches() - l0
    evals = stats[-1]["line_evals"]
    if use_shard:
        from fastspec_b200 import shard
        res = sharded["res"]
        evals = float(shard.pixel_cost(res["windows"], nwl).sum().item()) * ntau     # the whole synthesis

    out = dict(ms=ms, evals=evals, stats=stats[-1], launches=launches, clocks=clk.summary(), nwl=nwl,
               ntau=ntau, nlines=nlines)

    # e2e arm: host pinned line list through fsg_lineop_calc + fsg_radtran (flux read back)
    if not args.no_e2e:
        pin = {k: torch.from_numpy(np.ascontiguousarray(v)).pin_memory() for k, v in arr.items()}
        hl = F.CLines()
        hl.n = nlines
        hl.kind = 2
        hl.wl = F.C.cast(pin["wl"].data_ptr(), F._dp)
        for k in ("elo", "gf", "grad", "gqst", "gvdw"):
            setattr(hl, k, F.C.cast(pin[k].data_ptr(), F._fp))
        hl.spc = F.C.cast(pin["spc"].data_ptr(), F._ip)
        hl.ismol = F.C.cast(pin["ismol"].data_ptr(), F._ip)
        hsfl = torch.empty(nwl, dtype=torch.float64).pin_memory()
        hsfc = torch.empty(nwl, dtype=torch.float64).pin_memory()
        st_ = F.Stats()

        if use_shard:
            def step_e2e():
                for k in dt:
                    dt[k].copy_(pin[k], non_blocking=True)
                res = shard.run(backend)
                if rank == 0:
                    hsfl.copy_(res["flux"][0])
                    hsfc.copy_(res["flux"][1])
                return res["stats"] or zero
        else:
            def step_e2e():
                C.lineop_reset()
                C._ck(C._lib.fsg_lineop_calc(C.h, F.C.byref(hl), None, None, None, None, None, F.C.byref(st_)),
                      "fsg_lineop_calc")
                C._ck(C._lib.fsg_radtran(C.h, None, None, F.C.cast(hsfl.data_ptr(), F._dp),
                                         F.C.cast(hsfc.data_ptr(), F._dp)), "fsg_radtran")
                return st_.asdict()

        for _ in range(max(1, args.warmup // 2)):
            step_e2e()
        ms_e2e, _ = timed(step_e2e, args.steps)
        h2d = sum(int(v.numel() * v.element_size()) for v in pin.values())
        out.update(ms_e2e=ms_e2e, h2d=h2d, d2h=2 * nwl * 8, flux_check=float(hsfl[nwl // 2].item()))
    C.close()
    del dt
    if not args.no_plain and rank == 0:
        out["plain"] = plain_vs_mixed(F, torch, st, meta, co, dev, int(args.plain_lines))
    if not args.no_stokes and rank == 0:
        out["stokes"] = stokes_synthesis(F, torch, dev, args.steps, args.warmup)
    if not args.no_fit and rank == 0:
        out["fit"] = differentiable_fit(F, torch, dev, args.steps, args.warmup)
    if not args.no_batched and rank == 0:
        out["batched"] = batched_grid(F, torch, dev, args.batch_atm, args.batch_lines, args.steps, args.warmup)
    return out


# ---- CPU: the oracle (FP64 restatement of the reference) on a bounded sample -----------------------
def cpu_sample(seconds, w0=10000.0, threads=None):
    import oracle
    from fastspec_b200 import workloads as W
    import fastspec_b200 as F
    oracle.build()
    st, meta = load_atmosphere()
    density = 1e8 / (1.0 / W0 - 1.0 / W1)          # lines per unit wavenumber-in-1/A
    span = 0.5
    while True:
        margin = 4.0
        a, b = w0 - margin, w0 + span + margin
        n = int(density * (1.0 / a - 1.0 / b))
        L = W.molecular_lines(n, a, b, 99, exact=False)
        grid = dict(wmode=1, wstart=w0, wend=w0 + span, dstep=DSTEP)
        wave = F.make_grid(1, w0, w0 + span, DSTEP) + w0
        co = contopac_for(meta, wave)
        S = oracle.State(grid, st, contopac=co, vmicro=meta["vmicro"], molbrd=meta["molbrd"])
        ar = L.arrays()
        OL = oracle.Lines(wl=ar["wl"], elo=ar["elo"], gf=ar["gf"], grad=ar["grad"], gqst=ar["gqst"],
                          gvdw=ar["gvdw"], spc=ar["spc"], ismol=ar["ismol"], kind=2)
        x, w, _ = oracle.mu_quadrature(1, NMU)
        t = time.perf_counter()
        r = oracle.lineop_calc(S, OL, list_type=2)
        spl, spcc = oracle.radtran(S, x, r["lineopac"])
        oracle.disk_integ(w, spl, spcc)
        dt = time.perf_counter() - t
        ev = r["stats"]["line_evals"] + r["stats"]["wide_evals"]
        if dt >= seconds or span >= 64:
            return dict(evals=ev, seconds=dt, span=span, nlines=n, nwl=S.nwl)
        span *= max(2.0, min(8.0, seconds / max(dt, 1e-3)))


REF_BIN = os.path.join(HERE, "baseline", "_ref", "fastspec_Linux_x86_64")


def _stage_seconds(text, key):
    """'Time spent: HH:MM:SS.s' of the reference's stage line that contains key."""
    import re
    for line in text.splitlines():
        if key in line:
            m = re.search(r"Time spent: (\d+):(\d+):([\d.]+)", line)
            if m:
                return int(m.group(1)) * 3600 + int(m.group(2)) * 60 + float(m.group(3))
    return None


def ref_binary_sample(seconds, threads, w0=10000.0):
    """The reference executable on the cool-dwarf workload: a span of the R = 3e5 grid at w0 with the
    molecular lines of the 1e8-line list that fall inside it (the executable reads the lines of its
    wavelength range), OMP_NUM_THREADS = threads.  The span grows until the line-opacity stage takes
    `seconds`.  Its line-evals (windows inside the grid, wide lines included) are counted by the oracle
    on the same list, whose windows equal the executable's."""
    import tempfile
    import oracle
    from fastspec_b200 import workloads as W
    import fastspec_b200 as F
    oracle.build()
    st, meta = load_atmosphere()
    d = np.load(os.path.join(HERE, "fastspec_b200", "data", "atm_cooldwarf.npz"))
    model = W.eddington_model(float(d["teff"]), float(d["logg"]), 72)
    density = 1e8 / (1.0 / W0 - 1.0 / W1)
    span = 2.0
    while True:
        n = int(density * (1.0 / w0 - 1.0 / (w0 + span)))
        L = W.molecular_lines(n, w0, w0 + span, 99, exact=True)
        with tempfile.TemporaryDirectory() as wd:
            W.write_krz(os.path.join(wd, "model.krz"), model)
            L.write_z(os.path.join(wd, "lines.z"), w0, w0 + span)
            deck = ("wave=%.4f, %.4f, %.6f, 1\nsave=0, 0, 0, 0, 1\nvmic=%.3f\nmolbrd=%d\nlines=\n-1  lines.z\n\n"
                    "model=model.krz\nmus=%d\n" % (w0, w0 + span, DSTEP, meta["vmicro"], meta["molbrd"], NMU))
            with open(os.path.join(wd, "in.dat"), "w") as f:
                f.write(deck)
            t0 = time.perf_counter()
            r = subprocess.run([REF_BIN, "in.dat"], cwd=wd, capture_output=True, text=True,
                               env=dict(os.environ, OMP_NUM_THREADS=str(threads)))
            wall = time.perf_counter() - t0
        if r.returncode != 0 or "Total time" not in r.stdout:
            raise RuntimeError("reference executable failed: " + (r.stdout + r.stderr)[-500:])
        tl = _stage_seconds(r.stdout, "Total lines read")
        if (tl is not None and tl >= seconds) or span >= 64:
            break
        span *= max(2.0, min(8.0, seconds / max(tl or 0.05, 0.05)))
    grid = dict(wmode=1, wstart=w0, wend=w0 + span, dstep=DSTEP)
    wave = F.make_grid(1, w0, w0 + span, DSTEP) + w0
    S = oracle.State(grid, st, contopac=contopac_for(meta, wave), vmicro=meta["vmicro"], molbrd=meta["molbrd"])
    ar = L.arrays()
    rr = oracle.lineop_calc(S, oracle.Lines(**ar, kind=2), list_type=2)
    ev = rr["stats"]["line_evals"] + rr["stats"]["wide_evals"]
    return dict(evals=ev, seconds=tl, wall=wall, span=span, nlines=n, nwl=S.nwl, threads=threads,
                stdout_tail=" | ".join(x.strip() for x in r.stdout.splitlines()[-6:]))


def run_reference(args):
    cores = os.cpu_count()
    cfg = {"workload": "cool-dwarf molecular synthesis, 1e8 lines, 72 depths, R=3e5 (5000-25000 A), 7 mu"}
    if os.path.exists(REF_BIN):
        # the reference's own OpenMP executable, its line-opacity stage timed by itself
        seconds = max(3.0, args.cpu_seconds / max(1, args.steps))
        for _ in range(args.warmup):
            ref_binary_sample(1.0, cores)
        rates, ms, samp = [], 0.0, None
        for _ in range(args.steps):
            samp = ref_binary_sample(seconds, cores)
            rates.append(samp["evals"] / samp["seconds"])
            ms += samp["seconds"] * 1e3
        value = float(np.mean(rates))
        sample = ("reference executable (OpenMP, %d threads): line-opacity stage of %.2f A at 10000 A "
                  "(%d lines, %d wavelengths), its own stage time (includes reading the .z list); "
                  "line-evals counted by the oracle on the same list" % (cores, samp["span"], samp["nlines"], samp["nwl"]))
        kind = "reference"
        cfg["sample"] = sample
        cfg["reference_output"] = samp["stdout_tail"]
    else:
        for _ in range(args.warmup):
            cpu_sample(1.0)
        rates, ms, samp = [], 0.0, None
        for _ in range(args.steps):
            samp = cpu_sample(args.cpu_seconds / max(1, args.steps))
            rates.append(samp["evals"] / samp["seconds"])
            ms += samp["seconds"] * 1e3
        value = float(np.mean(rates))
        sample = "oracle FP64 C restatement (OpenMP) on %.2f A at 10000 A (%d lines, %d pixels)" % (
            samp["span"], samp["nlines"], samp["nwl"])
        kind = "port"
        cfg["sample"] = sample
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return
    if world > 1 or args.shard:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        if world == 1:
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            os.environ.setdefault("MASTER_PORT", "29533")
            os.environ.setdefault("RANK", "0")
            os.environ.setdefault("WORLD_SIZE", "1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    r = run_gpu(args, rank, world)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        if os.path.exists(REF_BIN):
            s = ref_binary_sample(args.cpu_seconds, os.cpu_count())
            cpu = {"value": s["evals"] / s["seconds"], "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                   "sample": "reference executable (OpenMP, %d threads), line-opacity stage of %.2f A at 10000 A "
                             "(%d lines, %d wavelengths): %.1f s by its own timer" % (s["threads"], s["span"],
                                                                                    s["nlines"], s["nwl"],
                                                                                    s["seconds"])}
        else:
            s = cpu_sample(args.cpu_seconds)
            cpu = {"value": s["evals"] / s["seconds"], "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                   "sample": "oracle FP64 C restatement (OpenMP) on %.2f A at 10000 A (%d lines, %d pixels), %.1f s"
                             % (s["span"], s["nlines"], s["nwl"], s["seconds"])}
    if world > 1 or args.shard:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    K = args.steps
    ms_step = r["ms"] / K
    value = r["evals"] * K / (r["ms"] / 1e3)
    st = r["stats"]
    nl = max(1, st["accum_launches"])
    wing_evals = r["evals"] - st["core_evals"]
    ms_launch = st["ms_wing_kernels"] / nl
    achieved = (wing_evals / nl) * FLOPS_PER_EVAL / (ms_launch / 1e3) / 1e12
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(HERE, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    smmax = float(peaks.get("sm_max_mhz", 1965.0))
    fp32_peak = 148 * 128 * 2 * smmax * 1e6 / 1e12
    # one reciprocal (MUFU) per wing evaluation; 16 MUFU results per SM and clock
    xu_peak = 148 * 16 * smmax * 1e6
    xu_achieved = wing_evals / (st["ms_wing_kernels"] / 1e3)
    # DRAM bytes of one wing launch: the LineOpac read-modify-write and one read of the records
    traffic = 2.0 * r["nwl"] * r["ntau"] * 8 + st["nlines_used"] * (r["ntau"] * 16 + 32) / nl
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": args.warmup,
        "ms_per_step": ms_step, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32+f64" if args.precision == "mixed" else "f64", "data": "synthetic",
        "config": {"workload": "cool-dwarf molecular synthesis, 1e8 lines, 72 depths, R=3e5 (5000-25000 A), 7 mu",
                   "nlines": r["nlines"], "nwl": r["nwl"], "ntau": r["ntau"], "precision": args.precision,
                   "l2": "inputs (3.6 GB lines, 278 MB ContOpac) exceed the 126 MB L2; no flush",
                   "parallelism": ("wavelength shards over %d GPUs (windows all-gathered over NCCL)" % world)
                                  if world > 1 else "single GPU"},
        "spectra_per_s": K / (r["ms"] / 1e3),
        "line_evals_per_step": r["evals"],
        "lines_retained": st["nlines_used"],
        "stage_ms": {"center": st["ms_center"], "accumulate": st["ms_accum"],
                     "accum_kernels": st["ms_accum_kernels"], "wing_kernels": st["ms_wing_kernels"],
                     "core_kernels": st["ms_core_kernels"], "accum_launches": st["accum_launches"]},
        "roofline": {"kernel": "k_accum_fast (wing pass)", "bound": "fp32", "achieved": achieved,
                     "peak": fp32_peak, "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                     "traffic": traffic,
                     "traffic_source": "per launch: LineOpac read + write (2 x nwl x ntau x 8 B) + the records of the "
                                       "launch's lines (ntau x 16 + 32 B each); ncu dram__bytes_read.sum + "
                                       "dram__bytes_write.sum of the 12 wing launches of the 1e6-line case = 0.92 x "
                                       "this model",
                     "peak_source": "derived: 148 SMs x 128 FP32 lanes x 2 x %.0f MHz (no FP32 peak is measured)" % smmax,
                     "flops_per_eval": FLOPS_PER_EVAL, "evals_per_launch": wing_evals / nl,
                     "ms_per_launch": ms_launch,
                     "xu": {"achieved": xu_achieved, "peak": xu_peak, "unit": "reciprocals/s",
                            "frac": xu_achieved / xu_peak},
                     # the same launch against the measured copy bandwidth: far from HBM-bound
                     "hbm": {"achieved": traffic / (ms_launch / 1e3) / 1e9,
                             "peak": float(peaks.get("hbm_gbs", 6650.0)), "unit": "GB/s",
                             "frac": traffic / (ms_launch / 1e3) / 1e9 / float(peaks.get("hbm_gbs", 6650.0))}},
        "core_pass": {"kernel": "k_core_fast", "evals": st["core_evals"], "ms": st["ms_core_kernels"],
                      "evals_per_s": st["core_evals"] / max(st["ms_core_kernels"], 1e-9) * 1e3},
        "gpu_launches": r["launches"],
        "clocks": r["clocks"],
    }
    if "ms_e2e" in r:
        line["e2e"] = {"value": r["evals"] * K / (r["ms_e2e"] / 1e3), "unit": UNIT,
                       "h2d_bytes_per_step": r["h2d"], "d2h_bytes_per_step": r["d2h"]}
    if cpu:
        line["cpu_baseline"] = cpu
    if "plain" in r:
        line["plain_fp64"] = r["plain"]
    if "batched" in r:
        line["batched"] = r["batched"]
    if "fit" in r:
        line["differentiable_fit"] = r["fit"]
    if "stokes" in r:
        line["stokes"] = r["stokes"]
    print(json.dumps(line))


if __name__ == "__main__":
    main()
