"""Shared test helpers: atmosphere states, continuum on a grid, seeded line lists."""
import os

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DATA = os.path.join(REPO, "fastspec_b200", "data")
GOLD = os.path.join(REPO, "tests", "golden")
# the reference tree, for the CPU tests that run its executable or read its shipped examples (they skip
# without it): FASTSPEC_REFERENCE, else the mount the install recipe looks at
def _reference_tree():
    from oracle.install_reference import MOUNT
    tree = os.environ.get("FASTSPEC_REFERENCE") or MOUNT
    return tree if os.path.isdir(tree) else ""


REFERENCE = _reference_tree()

STATE_KEYS = ("rhox", "T", "xne", "xna", "rho", "fractionpf", "xamass", "potion", "ion", "frac_h1", "frac_he1")


def load_atm(name):
    d = np.load(os.path.join(DATA, "atm_%s.npz" % name))
    st = {k: d[k] for k in STATE_KEYS}
    st["frac_h2"] = d["frac_h2"] if "frac_h2" in d.files else np.zeros(len(d["T"]), np.float32)
    meta = dict(vmicro=float(d["vmicro"]), molbrd=int(d["molbrd"]), cont_wave=d["cont_wave"],
                cont_opac=d["cont_opac"], species=[str(s) for s in d["species"]])
    return st, meta


def contopac_on(meta, wave_abs):
    """Continuum opacity on absolute wavelengths by log-linear interpolation of the knots."""
    lk = np.log(meta["cont_opac"])
    out = np.empty((len(wave_abs), lk.shape[1]))
    for t in range(lk.shape[1]):
        out[:, t] = np.exp(np.interp(wave_abs, meta["cont_wave"], lk[:, t]))
    return out


def load_pin(name):
    d = np.load(os.path.join(GOLD, name + ".npz"))
    return {k: d[k] for k in d.files}


def pin_lines(d):
    return dict(wl=d["line_wl"], elo=d["line_elo"], gf=d["line_gf"], grad=d["line_grad"], gqst=d["line_gqst"],
                gvdw=d["line_gvdw"], spc=d["line_spc"], ismol=d["line_ismol"])


def pin_setup(d):
    """(grid dict, state, contopac on the full grid) of a pin fixture."""
    g = d["grid"]
    grid = dict(wmode=int(g[3]), wstart=float(g[0]), wend=float(g[1]), dstep=float(g[2]))
    st, meta = load_atm(str(d["atm"]))
    from fastspec_b200 import workloads  # noqa: F401
    import oracle
    nwl = oracle.State(grid, st).nwl
    i0, i1 = int(d["i0"]), int(d["i1"])
    co = np.empty((nwl, len(st["T"])))
    co[i0:i1 + 1] = d["contopac"]
    co[:i0] = d["contopac"][0]
    co[i1 + 1:] = d["contopac"][-1]
    return grid, st, meta, co


def mag_pin_setup(d):
    """(grid, state, contopac full grid, line arrays, zeeman tuple) of the magnetic pin."""
    grid, st, meta, co = pin_setup(d)
    lines = pin_lines(d)
    z = (d["z_npi"], d["z_nsi"], d["z_spl_pi"], d["z_str_pi"], d["z_spl_si"], d["z_str_si"])
    return grid, st, co, lines, z


def sphere_pin(part):
    """One half of pin_sphere.npz as a pin dict: part "s" (scalar, solar atmosphere, the pin_solar
    list) or "m" (polarised, magnetic atmosphere, stellar-frame field, Zeeman lines)."""
    d = load_pin("pin_sphere")
    out = {k[2:]: v for k, v in d.items() if k.startswith(part + "_")}
    out["atm"] = "solar" if part == "s" else "magnetic"
    if part == "s":
        out.update({k: v for k, v in load_pin("pin_solar").items() if k.startswith("line_")})
        out["vmicro"], out["molbrd"] = 1.0, 0
    else:
        out.update({"line_" + k[6:]: v for k, v in d.items() if k.startswith("mline_")})
        out.update({k: v for k, v in d.items() if k.startswith("z_")})
        out["vmicro"], out["molbrd"] = 1.0, 0
    return out


def device_molecular_lines(n, wmin, wmax, seed, device):
    """A cool-dwarf list of n lines drawn on the device with the distributions of
    workloads.molecular_lines (wavenumber uniform over [1e8/wmax, 1e8/wmin], four species at 25 %,
    log gf ~ N(-5, 1.5), E_low ~ Exp(1 eV) capped at 5 eV, log G6/NH ~ U(-8, -7), Grad = Gqst = 0),
    sorted by wavelength: dict of device tensors.  Seeded torch generator on the device; drawing 1e8
    lines takes well under a second there, against minutes on the host."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    sig = torch.empty(n, dtype=torch.float64, device=device).uniform_(1e8 / wmax, 1e8 / wmin, generator=g)
    wl, order = torch.sort(1e8 / sig)
    del sig
    out = {"wl": wl.contiguous()}
    spc = torch.randint(0, 4, (n,), generator=g, device=device, dtype=torch.int32)
    out["spc"] = spc[order].contiguous()
    del spc
    lg = torch.empty(n, dtype=torch.float32, device=device).normal_(-5.0, 1.5, generator=g)
    out["gf"] = torch.pow(10.0, lg[order]).contiguous()
    del lg
    el = torch.empty(n, dtype=torch.float32, device=device).exponential_(1.0, generator=g)
    out["elo"] = torch.clamp(el[order], max=5.0).contiguous()
    del el
    lv = torch.empty(n, dtype=torch.float32, device=device).uniform_(-8.0, -7.0, generator=g)
    out["gvdw"] = torch.pow(10.0, lv[order]).contiguous()
    del lv, order
    out["grad"] = torch.zeros(n, dtype=torch.float32, device=device)
    out["gqst"] = torch.zeros(n, dtype=torch.float32, device=device)
    out["ismol"] = torch.ones(n, dtype=torch.int32, device=device)
    return out


def device_view(F, dt, a=0, b=None, kind=2):
    """fsg_lines view (CLines) of lines [a, b) of a dict of device tensors."""
    import ctypes as C
    b = int(dt["wl"].numel()) if b is None else b
    v = F.CLines()
    v.n = b - a
    v.kind = kind
    ptr = lambda t, ct: C.cast(t.data_ptr() + a * t.element_size(), C.POINTER(ct))
    v.wl = ptr(dt["wl"], C.c_double)
    for k in ("elo", "gf", "grad", "gqst", "gvdw"):
        setattr(v, k, ptr(dt[k], C.c_float))
    v.spc = ptr(dt["spc"], C.c_int32)
    if "ismol" in dt:
        v.ismol = ptr(dt["ismol"], C.c_int32)
    return v
