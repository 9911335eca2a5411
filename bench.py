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

Line blocks are capped at 2 GB (the configuration's "lines streamed in 2 GB blocks", LIMITRAM);
`limitram_24gb` repeats one step with 24 GB blocks.  `plain_fp64` runs the plain FP64-faithful GPU
path once on the whole list.

--impl reference: the reference's CPU implementation of the path timed on this host: its own
OpenMP executable (copied unmodified to baseline/_ref by the build; there is no Fortran compiler to
build it) on all host threads, on the configuration's whole grid with a uniform random subsample of
the line list per step (RefSampler), or, without the executable, the FP64 C restatement (oracle/)
with OpenMP.  That arm loads nothing of the CUDA library.
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
W0, W1, DSTEP, NMU = 5000.0, 25000.0, 2.99792458e5 / 3e5, 7      # R = 3e5 on the ln-lambda grid
LIMITRAM_GB = 2.0            # the configuration's 2 GB line blocks
WORKLOAD = ("cool-dwarf molecular synthesis, 1e8 lines, 72 depths (71 after the model's temperature check), "
            "R = 3e5 (5000-25000 A), 7 mu, 2 GB line blocks")


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
    p.add_argument("--limitram", type=float, default=LIMITRAM_GB, help="line-block memory cap [GB]")
    p.add_argument("--no-plain", action="store_true", help="skip the plain FP64 path comparison")
    p.add_argument("--shard", action="store_true",
                   help="run the wavelength-sharded synthesis even on one GPU (a process group of one)")
    p.add_argument("--plain-lines", type=float, default=-1,
                   help="lines of the plain FP64 comparison; default: the whole headline list")
    p.add_argument("--no-extra", action="store_true", help="skip the 24 GB block-size step")
    p.add_argument("--no-batched", action="store_true", help="skip the batched-grid measurement")
    p.add_argument("--batch-atm", type=int, default=256)
    p.add_argument("--batch-lines", type=float, default=2e6)
    p.add_argument("--no-fit", action="store_true", help="skip the differentiable-fit measurement")
    p.add_argument("--no-stokes", action="store_true", help="skip the polarised (Stokes) synthesis measurement")
    p.add_argument("--no-c0", action="store_true", help="skip the plain scalar synthesis (20,000 lines) measurement")
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
def device_list(F, torch, nlines, dev, seed):
    """The headline list drawn on the device (seeded torch generator with the distributions of
    workloads.molecular_lines, sorted by wavelength; 1e8 lines in about a second instead of minutes on
    the host) and its fsg_lines view."""
    import helpers as H
    dt = H.device_molecular_lines(int(nlines), W0, W1, seed, torch.device("cuda", dev))
    return dt, H.device_view(F, dt)


def plain_fp64(F, torch, st, meta, co, dev, dt, nlines, mixed):
    """The plain FP64-faithful GPU path (LineOpacity1's per-wavelength order and FP64 table lerp, the
    reference's PACK / wide lines / segments) on the headline list, or on a uniform subsample of
    nlines of it, one synthesis timed with CUDA events; against the mixed path on the same lines.
    mixed: (ms per step, flux) of the headline's mixed path on the whole list.  Its blocks hold 24 GB of
    FP64 records: with 2 GB blocks the lines that reach one wavelength exceed one block and the
    segmentation stops as the reference's does (synth.f90:1035-1040)."""
    import helpers as H
    n_all = int(dt["wl"].numel())
    if nlines <= 0 or nlines >= n_all:
        sub, nlines = dt, n_all
    else:
        step = n_all // int(nlines)
        sub = {k: v[::step].contiguous() for k, v in dt.items()}
        nlines = int(sub["wl"].numel())
    dl = H.device_view(F, sub)
    x, w, _ = F.mu_quadrature(1, NMU)
    out, flux = {}, {}
    for name, prec in (("fp64", F.PREC_FP64), ("mixed", F.PREC_MIXED)):
        if name == "mixed" and sub is dt:
            out["mixed"] = {"ms": mixed[0]}
            flux["mixed"] = mixed[1]
            continue
        C = F.Context(device=dev, precision=prec, vmicro=meta["vmicro"], molbrd=meta["molbrd"],
                      limitram_gb=24.0 if prec == F.PREC_FP64 else LIMITRAM_GB)
        C.set_grid(1, W0, W1, DSTEP)
        C.set_atmosphere(st)
        C.set_contopac(co)
        C.set_mu(x, w)
        sfl = torch.empty(C.nwl, dtype=torch.float64, device=f"cuda:{dev}")
        sfc = torch.empty_like(sfl)
        stream = torch.cuda.ExternalStream(C.stream_ptr(), device=dev)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        C.lineop_reset()
        s_ = C.lineop_calc_dev(dl)
        C.radtran_dev(None, None, sfl.data_ptr(), sfc.data_ptr())
        e1.record(stream)
        e1.synchronize()
        out[name] = {"ms": e0.elapsed_time(e1), "ms_center": s_["ms_center"], "ms_accum": s_["ms_accum"],
                     "line_evals": s_["line_evals"], "segments_or_blocks": s_["nblocks"], "wide": s_["nwide"]}
        flux[name] = (sfl / sfc).cpu().numpy()
        C.close()
        del sfl, sfc
    ev = out["fp64"]["line_evals"]
    return {"lines": nlines, "sample": "the whole headline list" if sub is dt else
            "every %d-th line of the headline list" % (n_all // nlines),
            "fp64": out["fp64"], "mixed_ms": out["mixed"]["ms"],
            "fp64_value": ev / (out["fp64"]["ms"] / 1e3), "unit": UNIT,
            "mixed_over_fp64": out["fp64"]["ms"] / out["mixed"]["ms"],
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
           "replay_stages_ms": {k: st[k] for k in ("ms_prepare", "ms_wing", "ms_core", "ms_solve")},
           "core_evals": st["core_evals"],
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
    arr = W.atomic_lines(100_000, w0, w1, W.SEED0 + 4, exact=False).arrays()
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


def scalar_c0(F, torch, dev, steps, warmup):
    """The plain scalar configuration: 20,000 atomic lines over 5000-5200 A at 0.005 A (40,001
    wavelengths), the solar-like atmosphere (56 depths), 7 angles: LineopCalc + RadTranCalc + flux
    through the C-ABI with the list and the spectra in host memory, FP64 and mixed; and the reference
    executable on the same deck with all host threads."""
    from fastspec_b200 import workloads as W
    d = np.load(os.path.join(HERE, "fastspec_b200", "data", "atm_solar.npz"))
    st = {k: d[k] for k in ("rhox", "T", "xne", "xna", "rho", "fractionpf", "xamass", "potion", "ion", "frac_h1",
                            "frac_he1")}
    w0, w1, step = 5000.0, 5200.0, 0.005
    wave = F.make_grid(0, w0, w1, step) + w0
    lk = np.log(d["cont_opac"])
    co = np.exp(np.stack([np.interp(wave, d["cont_wave"], lk[:, t]) for t in range(lk.shape[1])], axis=1))
    L = W.atomic_lines(20000, w0, w1, W.SEED0 + 0, exact=True)
    LL = F.LineList.from_arrays(L.arrays())
    x, w, _ = F.mu_quadrature(1, NMU)
    out = {"config": "20,000 atomic lines 5000-5200 A at 0.005 A (40,001 wavelengths), solar-like 56 depths, 7 mu",
           "timing": "wall clock per synthesis (LineopCalc + RadTranCalc + flux, host list in, host spectra out)"}
    flux = {}
    for name, prec in (("fp64", F.PREC_FP64), ("mixed", F.PREC_MIXED)):
        C = F.Context(device=dev, precision=prec, vmicro=float(d["vmicro"]), molbrd=int(d["molbrd"]))
        C.set_grid(0, w0, w1, step)
        C.set_atmosphere(st)
        C.set_contopac(co)
        C.set_mu(x, w)

        def one():
            C.lineop_reset()
            r = C.lineop_calc(LL, want_lineopac=False, want_lines=False)
            return r["stats"], C.radtran()

        for _ in range(warmup):
            one()
        torch.cuda.synchronize()
        n = max(steps, 10)
        t0 = time.perf_counter()
        for _ in range(n):
            stt, sp = one()
        ms = (time.perf_counter() - t0) * 1e3 / n
        flux[name] = sp[2] / sp[3]
        out[name] = {"spectra_per_s": 1e3 / ms, "ms_per_spectrum": ms, "ms_lineop": stt["ms_total"],
                     "line_evals": stt["line_evals"], "line_evals_per_s": stt["line_evals"] / (stt["ms_total"] / 1e3)}
        out["nwl"] = C.nwl
        C.close()
    out["mixed_vs_fp64_flux_max_rel"] = float(np.max(np.abs(flux["mixed"] / flux["fp64"] - 1)))
    if os.path.exists(REF_BIN):
        ref = ref_c0(L, d, os.cpu_count())
        out["reference"] = ref
        if "spectra_per_s" in ref:
            out["mixed_over_reference"] = out["mixed"]["spectra_per_s"] / ref["spectra_per_s"]
            out["fp64_over_reference"] = out["fp64"]["spectra_per_s"] / ref["spectra_per_s"]
    return out


def ref_c0(L, d, threads):
    """The reference executable on the plain scalar deck (the same 20,000 lines as a .z list, the
    solar-like Eddington-grey model it derives the atmosphere state from): its own stage times of the
    line opacity (list reading included) and of the formal solver, and the wall clock of the whole run."""
    import tempfile
    from fastspec_b200 import workloads as W
    with tempfile.TemporaryDirectory() as wd:
        W.write_krz(os.path.join(wd, "model.krz"), W.eddington_model(float(d["teff"]), float(d["logg"]), len(d["T"])))
        L.write_z(os.path.join(wd, "lines.z"), 5000.0, 5200.0)
        deck = ("wave=5000.0, 5200.0, 0.005, 0\nsave=0, 0, 0, 0, 1\nvmic=%.3f\nmolbrd=%d\nlines=\n-1  lines.z\n\n"
                "model=model.krz\nmus=%d\n" % (float(d["vmicro"]), int(d["molbrd"]), NMU))
        with open(os.path.join(wd, "in.dat"), "w") as f:
            f.write(deck)
        t0 = time.perf_counter()
        r = subprocess.run([REF_BIN, "in.dat"], cwd=wd, capture_output=True, text=True,
                           env=dict(os.environ, OMP_NUM_THREADS=str(threads)))
        wall = time.perf_counter() - t0
    if r.returncode != 0 or "Total time" not in r.stdout:
        return {"threads": threads, "error": (r.stdout + r.stderr)[-300:]}
    lines_s = _stage_seconds(r.stdout, "Total lines read")
    rt_s = _stage_seconds(r.stdout, "radiative transfer")
    return {"threads": threads, "opacity_s": lines_s, "solver_s": rt_s, "wall_s": wall,
            "spectra_per_s": 1.0 / max((lines_s or 0.0) + (rt_s or 0.0), 0.1),
            "timing": "the executable's own stage timers (0.1 s resolution, a floor of 0.1 s on their sum): line "
                      "opacity (list reading included) + formal solver, per spectrum; wall_s: the whole program"}


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
    if os.path.exists(REF_BIN):
        ref = ref_stokes(L, os.cpu_count())
        out["reference"] = ref
        out["mixed_over_reference"] = out["mixed"]["spectra_per_s"] / ref["spectra_per_s"]
    return out


def ref_stokes(L, threads):
    """The reference executable on the same polarised deck (the 5000 Zeeman lines with their explicit
    splitting patterns, 6000-6100 A at 0.002 A, BFRAME 1, 2 kG at 60/30 deg, 9 angles), all host
    threads: its own stage times of the magnetic line opacity (list reading included) and of the
    polarised formal solver."""
    import tempfile
    import oracle
    from fastspec_b200 import workloads as W
    d = np.load(os.path.join(HERE, "fastspec_b200", "data", "atm_magnetic.npz"))
    jlo, jup, glo, gup = L.zeeman
    pats = [oracle.zeeman_pattern(jlo[i], jup[i], glo[i], gup[i]) for i in range(L.n)]
    with tempfile.TemporaryDirectory() as wd:
        W.write_krz(os.path.join(wd, "model.krz"), W.eddington_model(float(d["teff"]), float(d["logg"]),
                                                                     len(d["T"])))
        L.write_z(os.path.join(wd, "lines.z"), 6000.0, 6100.0, patterns=pats)
        deck = ("wave=6000.0, 6100.0, 0.002, 0\nsave=0, 0, 0, 0, 1\nvmic=%.3f\nmolbrd=%d\nlines=\n-1  lines.z\n\n"
                "model=model.krz\nmus=9\nbframe=1\nbfield=2000, 60, 30\n" % (float(d["vmicro"]), int(d["molbrd"])))
        with open(os.path.join(wd, "in.dat"), "w") as f:
            f.write(deck)
        t0 = time.perf_counter()
        r = subprocess.run([REF_BIN, "in.dat"], cwd=wd, capture_output=True, text=True,
                           env=dict(os.environ, OMP_NUM_THREADS=str(threads)))
        wall = time.perf_counter() - t0
    if r.returncode != 0 or "Total time" not in r.stdout:
        return {"error": (r.stdout + r.stderr)[-300:]}
    lines_s = _stage_seconds(r.stdout, "Total lines read")
    rt_s = _stage_seconds(r.stdout, "radiative transfer")
    return {"threads": threads, "opacity_s": lines_s, "solver_s": rt_s, "wall_s": wall,
            "spectra_per_s": 1.0 / max((lines_s or 0.0) + (rt_s or 0.0), 0.1),
            "timing": "the executable's own stage timers (0.1 s resolution): line opacity (list reading included) "
                      "+ polarised radiative transfer, per spectrum"}


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
    x, w, _ = F.mu_quadrature(1, NMU)
    prec = F.PREC_MIXED if args.precision == "mixed" else F.PREC_FP64

    def make_context(limitram):
        c = F.Context(device=dev, precision=prec, vmicro=meta["vmicro"], molbrd=meta["molbrd"], limitram_gb=limitram)
        c.set_grid(1, W0, W1, DSTEP)
        c.set_atmosphere(st)
        c.set_contopac(co)
        c.set_mu(x, w)
        return c

    C = make_context(args.limitram)
    nwl, ntau = C.nwl, C.ntau
    stream = torch.cuda.ExternalStream(C.stream_ptr(), device=dev)

    # the line list, resident in HBM (value arm)
    dt, dl = device_list(F, torch, nlines, dev, W.SEED0 + 1)
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
    if use_shard:
        mixed_flux = (sharded["res"]["flux"][0] / sharded["res"]["flux"][1]).cpu().numpy()
    else:
        mixed_flux = (sfl / sfc).cpu().numpy()

    # the same step with 24 GB line blocks
    if not args.no_extra and not use_shard:
        C24 = make_context(24.0)
        stream24 = torch.cuda.ExternalStream(C24.stream_ptr(), device=dev)
        for _ in range(2):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream24)
            C24.lineop_reset()
            s24 = C24.lineop_calc_dev(dl)
            C24.radtran_dev(spl.data_ptr(), spc.data_ptr(), sfl.data_ptr(), sfc.data_ptr())
            e1.record(stream24)
            e1.synchronize()
        out["limitram_24gb"] = {"ms_per_step": e0.elapsed_time(e1), "wing_ms": s24["ms_wing_kernels"],
                                "core_ms": s24["ms_core_kernels"], "blocks": s24["nblocks"],
                                "line_evals_per_s": s24["line_evals"] / (e0.elapsed_time(e1) / 1e3)}
        C24.close()

    # e2e arm: host pinned line list through fsg_lineop_calc + fsg_radtran (flux read back)
    if not args.no_e2e:
        pin = {k: v.cpu().pin_memory() for k, v in dt.items()}
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
    # the side measurements are single-GPU ones: a multi-GPU run leaves them to its N = 1 line, so
    # that no rank waits at the closing barrier for minutes of rank 0's extra work
    side = world == 1
    if not args.no_plain and side:
        out["plain"] = plain_fp64(F, torch, st, meta, co, dev, dt, int(args.plain_lines), (ms / args.steps, mixed_flux))
    del dt, dl
    torch.cuda.empty_cache()
    if not args.no_c0 and side:
        out["c0"] = scalar_c0(F, torch, dev, args.steps, args.warmup)
    if not args.no_stokes and side:
        out["stokes"] = stokes_synthesis(F, torch, dev, args.steps, args.warmup)
    if not args.no_fit and side:
        out["fit"] = differentiable_fit(F, torch, dev, args.steps, args.warmup)
    if not args.no_batched and side:
        out["batched"] = batched_grid(F, torch, dev, args.batch_atm, args.batch_lines, args.steps, args.warmup)
    return out


# ---- CPU: the reference's own executable (or the oracle port) on a bounded sample -------------------
# The sample keeps the configuration's whole grid (5000-25000 A at R = 3e5, 482,832 wavelengths) and
# takes a uniform random subsample of the 1e8-line list (same distributions, its own seed per step).
# Windows are a property of each line and the atmosphere, so the work per line, the share of lines
# whose windows span more than 5000 km/s (wide lines, MarkWideLines, synth.f90:709-744) and the
# per-wavelength accumulation match the full synthesis, scaled by the sample fraction.  The sample
# fits one line block, the reference's fastest mode: the full list would run in the 100,000-line
# minimum blocks NlinesMax falls back to (opacity.f90:712-771: the list alone exceeds LIMITRAM),
# where far more lines are accumulated one by one as wide lines.  The rate is therefore an upper
# bound on the reference's speed for the whole configuration.
REF_BIN = os.path.join(HERE, "baseline", "_ref", "fastspec_Linux_x86_64")
REF_LINES = 50_000            # lines per timed reference sample (1/2000 of the list)
REF_WARM_LINES = 5_000        # lines per warm-up run


def _stage_seconds(text, key):
    """'Time spent: HH:MM:SS.s' of the reference's stage line that contains key."""
    import re
    for line in text.splitlines():
        if key in line:
            m = re.search(r"[Tt]ime spent: (\d+):(\d+):([\d.]+)", line)
            if m:
                return int(m.group(1)) * 3600 + int(m.group(2)) * 60 + float(m.group(3))
    return None


class RefSampler:
    """Samples of the cool-dwarf configuration for the CPU baselines.  Loads nothing of the CUDA
    library: the grid, the windows and the line-eval counts come from the oracle (whose windows equal
    the executable's), the line lists and the model from the workload generator (numpy)."""

    def __init__(self):
        import tempfile
        import oracle
        from fastspec_b200 import workloads as W
        oracle.build()
        self.oracle, self.W = oracle, W
        self.st, self.meta = load_atmosphere()
        self.grid = dict(wmode=1, wstart=W0, wend=W1, dstep=DSTEP)
        self.S = None
        self.wd = tempfile.mkdtemp(prefix="fsref_")
        d = np.load(os.path.join(HERE, "fastspec_b200", "data", "atm_cooldwarf.npz"))
        W.write_krz(os.path.join(self.wd, "model.krz"), W.eddington_model(float(d["teff"]), float(d["logg"]), 72))

    def state(self):
        if self.S is None:
            S0 = self.oracle.State(self.grid, self.st)
            co = contopac_for(self.meta, S0.wave + W0)
            self.S = self.oracle.State(self.grid, self.st, contopac=co, vmicro=self.meta["vmicro"],
                                       molbrd=self.meta["molbrd"])
        return self.S

    def lines(self, n, seed, exact):
        return self.W.molecular_lines(int(n), W0, W1, seed, exact=exact)

    def evals(self, L):
        """Line-evals of a list on the whole grid: Ntau x the retained windows (oracle central pass)."""
        S = self.state()
        r = self.oracle.lineop_calc(S, self.oracle.Lines(**L.arrays(), kind=2), list_type=2, wrange=(1, 0))
        keep = (r["flags"] & 1) == 0
        return float(S.ntau) * float(np.sum(r["iright"][keep].astype(np.int64) - r["ileft"][keep] + 1))

    def run_binary(self, L, threads, wend=W1):
        """One run of the reference executable on list L over [W0, wend]; its stage times."""
        L.write_z(os.path.join(self.wd, "lines.z"), W0, W1)
        deck = ("wave=%.4f, %.4f, %.12f, 1\nsave=0, 0, 0, 0, 1\nvmic=%.3f\nmolbrd=%d\nlines=\n-1  lines.z\n\n"
                "model=model.krz\nmus=%d\n" % (W0, wend, DSTEP, self.meta["vmicro"], self.meta["molbrd"], NMU))
        with open(os.path.join(self.wd, "in.dat"), "w") as f:
            f.write(deck)
        t0 = time.perf_counter()
        r = subprocess.run([REF_BIN, "in.dat"], cwd=self.wd, capture_output=True, text=True,
                           env=dict(os.environ, OMP_NUM_THREADS=str(threads)))
        wall = time.perf_counter() - t0
        if r.returncode != 0 or "Total time" not in r.stdout:
            raise RuntimeError("reference executable failed: " + (r.stdout + r.stderr)[-500:])
        return dict(lines_s=_stage_seconds(r.stdout, "Total lines read"),
                    rt_s=_stage_seconds(r.stdout, "radiative transfer"),
                    total_s=_stage_seconds(r.stdout, "Total time spent"), wall_s=wall,
                    stage_line=next((x.strip() for x in r.stdout.splitlines() if "Total lines read" in x), ""))

    def parse_seconds(self, L, threads):
        """The list-reading share of the stage time: the same list on a two-wavelength grid, where the
        reader parses every record and keeps almost none (its WAVE= selection)."""
        return self.run_binary(L, threads, wend=W0 * np.exp(1.5 * DSTEP / 2.99792458e5))["lines_s"]

    def binary_sample(self, n, seed, threads):
        L = self.lines(n, seed, exact=True)
        run = self.run_binary(L, threads)
        return dict(run, evals=self.evals(L), nlines=L.n, L=L)

    def port_sample(self, n, seed):
        """The oracle (FP64 C restatement, OpenMP) on the same kind of sample, timed here."""
        L = self.lines(n, seed, exact=False)
        S = self.state()
        t = time.perf_counter()
        r = self.oracle.lineop_calc(S, self.oracle.Lines(**L.arrays(), kind=2), list_type=2)
        dt = time.perf_counter() - t
        return dict(evals=r["stats"]["line_evals"] + r["stats"]["wide_evals"], lines_s=dt, nlines=L.n)


def reference_rate(threads, steps, warmup, seed0=20261203 + 500):
    """The reference's line-evals/s on `steps` samples (each its own subsample): per-step rates from the
    executable's own line-opacity stage time less the list-reading share, with their spread."""
    R = RefSampler()
    cores = threads
    if os.path.exists(REF_BIN):
        for k in range(warmup):
            R.run_binary(R.lines(REF_WARM_LINES, seed0 + 1000 + k, exact=True), threads)
        rates, rates_incl, samp, ms, parse = [], [], None, 0.0, 0.0
        for k in range(steps):
            samp = R.binary_sample(REF_LINES, seed0 + k, threads)
            if k == 0:
                parse = R.parse_seconds(samp["L"], threads)
            lines_s = max(samp["lines_s"] - parse, 0.05)
            rates.append(samp["evals"] / lines_s)
            rates_incl.append(samp["evals"] / samp["lines_s"])
            ms += samp["lines_s"] * 1e3
        kind = "reference"
        sample = ("reference executable (OpenMP, %d threads) on the configuration's whole grid (%d wavelengths, "
                  "R = 3e5) with %d-line uniform subsamples of the 1e8-line list (1/%d, one per step): line-"
                  "opacity stage time by its own timer (0.1 s resolution, ~%.1f s per sample) less the list-"
                  "reading share (%.2f s, the same list on a two-wavelength grid); line-evals counted by the "
                  "oracle; single-block mode, an upper bound on the reference's speed for the full list"
                  % (threads, R.state().nwl, REF_LINES, int(1e8 // REF_LINES), ms / 1e3 / steps, parse))
        extra = {"rate_including_list_reading": float(np.mean(rates_incl)), "parse_seconds": parse,
                 "stage_line": samp["stage_line"], "rt_seconds": samp["rt_s"], "total_seconds": samp["total_s"]}
    else:
        cores = os.cpu_count()
        for k in range(warmup):
            R.port_sample(REF_WARM_LINES // 5, seed0 + 1000 + k)
        rates, samp, ms = [], None, 0.0
        for k in range(steps):
            samp = R.port_sample(REF_LINES // 10, seed0 + k)
            rates.append(samp["evals"] / samp["lines_s"])
            ms += samp["lines_s"] * 1e3
        kind = "port"
        sample = ("oracle FP64 C restatement (OpenMP) on the configuration's whole grid with %d-line uniform "
                  "subsamples of the 1e8-line list (one per step)" % (REF_LINES // 10))
        extra = {}
    rates = np.asarray(rates)
    extra.update(rate_min=float(rates.min()), rate_max=float(rates.max()),
                 spread=float((rates.max() - rates.min()) / rates.mean()))
    return dict(value=float(rates.mean()), ms=ms, kind=kind, cores=cores, sample=sample, extra=extra)


def run_reference(args):
    cfg = {"workload": WORKLOAD}
    r = reference_rate(os.cpu_count(), args.steps, args.warmup)
    cfg["sample"] = r["sample"]
    line = {"impl": "reference", "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms"] / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": r["kind"],
                             "sample": r["sample"]},
            "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "reference_samples": r["extra"]}
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
        c = reference_rate(os.cpu_count(), 2, 0)
        cpu = {"value": c["value"], "unit": UNIT, "cores": c["cores"], "kind": c["kind"], "sample": c["sample"],
               "spread": c["extra"]["spread"]}
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
        "config": {"workload": WORKLOAD, "limitram_gb": args.limitram,
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
    if "limitram_24gb" in r:
        line["limitram_24gb"] = r["limitram_24gb"]
    if "batched" in r:
        line["batched"] = r["batched"]
    if "fit" in r:
        line["differentiable_fit"] = r["fit"]
    if "stokes" in r:
        line["stokes"] = r["stokes"]
    if "c0" in r:
        line["plain_scalar_c0"] = r["c0"]
    print(json.dumps(line))


if __name__ == "__main__":
    main()
