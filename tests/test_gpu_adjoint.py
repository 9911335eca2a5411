"""Hand-written adjoint of the synthesis behind torch.autograd (fastspec_b200.adjoint): gradients of a
flux chi-square with respect to element abundances, per-line log gf and the microturbulence, checked
against central finite differences of the FP64 forward (h = 1e-4 dex; 0.02 km/s for vmicro, where
steps of 1e-3 km/s resolve single-pixel window changes), against finite differences of the FP64
oracle, and between the mixed-precision and FP64 forwards."""
import numpy as np
import pytest
import torch

import helpers as H

pytestmark = pytest.mark.gpu
SIG = 1.0 / 300.0
ELS = ["Fe", "Ti", "Cr", "Ni", "Ca"]


def case():
    import fastspec_b200 as F
    from fastspec_b200 import workloads as W
    st, meta = H.load_atm("solar")
    w0, span = 4800.0, 3.0
    grid = dict(wmode=0, wstart=w0, wend=w0 + span, dstep=0.005)
    co = H.contopac_on(meta, F.make_grid(0, w0, w0 + span, 0.005) + w0)
    arr = W.atomic_lines(300, w0 - 0.5, w0 + span + 0.5, 123).arrays()
    return grid, st, meta, co, arr


def model(fsg, prec):
    from fastspec_b200 import adjoint as AD
    grid, st, meta, co, arr = case()
    return AD.FluxModel(fsg, grid, st, co, arr, meta["species"], vmicro=1.0, precision=prec), arr


def target(M, loggf0):
    from fastspec_b200 import adjoint as AD
    rng = np.random.default_rng(5)
    ne = len(AD.ELEMENTS)
    da = np.zeros(ne)
    for el in ELS:
        da[AD.ELEMENTS.index(el)] = rng.normal(0.0, 0.1)
    with torch.no_grad():
        return AD.synth_flux(M, torch.tensor(loggf0 + rng.normal(0, 0.05, len(loggf0))), torch.tensor(da),
                             torch.tensor(1.05)).clone()


def grads(M, loggf0, fobs):
    from fastspec_b200 import adjoint as AD
    ne = len(AD.ELEMENTS)
    lg = torch.tensor(loggf0, requires_grad=True)
    da = torch.zeros(ne, dtype=torch.float64, requires_grad=True)
    vm = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    f = AD.synth_flux(M, lg, da, vm)
    c = (((f - fobs) / SIG) ** 2).sum()
    c.backward()
    return lg.grad.numpy(), da.grad.numpy(), float(vm.grad)


def chi2_at(M, fobs, loggf, da, vm):
    from fastspec_b200 import adjoint as AD
    with torch.no_grad():
        f = AD.synth_flux(M, torch.tensor(loggf), torch.tensor(da), torch.tensor(vm))
        return float((((f - fobs) / SIG) ** 2).sum())


def test_gradients_vs_finite_differences(fsg):
    from fastspec_b200 import adjoint as AD
    M, arr = model(fsg, fsg.PREC_FP64)
    loggf0 = np.log10(arr["gf"].astype(np.float64))
    fobs = target(M, loggf0)
    gl, ga, gv = grads(M, loggf0, fobs)
    ne = len(AD.ELEMENTS)
    h = 1e-4
    for el in ELS:
        e = AD.ELEMENTS.index(el)
        d = np.zeros(ne); d[e] = h
        fd = (chi2_at(M, fobs, loggf0, d, 1.0) - chi2_at(M, fobs, loggf0, -d, 1.0)) / (2 * h)
        assert abs(ga[e] - fd) <= 1e-3 * abs(fd) + 1e-3, (el, ga[e], fd)
    # elements without lines in the list have no gradient
    assert np.all(ga[[AD.ELEMENTS.index(x) for x in ("H", "He", "C", "O", "Zn")]] == 0.0)
    for i in np.argsort(-np.abs(gl))[:6]:
        lp = loggf0.copy(); lp[i] += h
        lm = loggf0.copy(); lm[i] -= h
        fd = (chi2_at(M, fobs, lp, np.zeros(ne), 1.0) - chi2_at(M, fobs, lm, np.zeros(ne), 1.0)) / (2 * h)
        assert abs(gl[i] - fd) <= 1e-3 * abs(fd), (i, gl[i], fd)
    hv = 0.02
    fd = (chi2_at(M, fobs, loggf0, np.zeros(ne), 1.0 + hv) - chi2_at(M, fobs, loggf0, np.zeros(ne), 1.0 - hv)) / (2 * hv)
    assert abs(gv - fd) <= 2e-3 * abs(fd), (gv, fd)
    # the abundance gradient is ln 10 x the element's summed line gradient... already ln 10 x d/dln gf
    sp_el = np.array([AD.ELEMENTS.index(str(s).split()[0]) for s in H.load_atm("solar")[1]["species"]])
    line_el = sp_el[arr["spc"]]
    for el in ELS:
        e = AD.ELEMENTS.index(el)
        assert np.isclose(ga[e], gl[line_el == e].sum(), rtol=1e-12, atol=1e-12)
    M.close()


def test_spherical_gradients_vs_finite_differences(fsg):
    """The same atmosphere as a spherical model (the radius and layer heights of the reference's
    spherical pin; the seven quadrature rays of LocPrfSph, solver.f90:182-261): the adjoint runs each
    ray's sweep backwards and returns a ray point's derivative to the layer it samples.  Gradients
    against central finite differences of the FP64 spherical forward, and different from the
    plane-parallel model's."""
    from fastspec_b200 import adjoint as AD
    d = H.sphere_pin("s")
    M, arr = model(fsg, fsg.PREC_FP64)
    loggf0 = np.log10(arr["gf"].astype(np.float64))
    fobs = target(M, loggf0)
    gl_pp, ga_pp, _ = grads(M, loggf0, fobs)
    M.C.set_geometry(float(d["radius"]), d["height"])
    gl, ga, gv = grads(M, loggf0, fobs)
    ne = len(AD.ELEMENTS)
    h = 1e-4
    for el in ELS:
        e = AD.ELEMENTS.index(el)
        dd = np.zeros(ne); dd[e] = h
        fd = (chi2_at(M, fobs, loggf0, dd, 1.0) - chi2_at(M, fobs, loggf0, -dd, 1.0)) / (2 * h)
        assert abs(ga[e] - fd) <= 1e-3 * abs(fd) + 1e-3, (el, ga[e], fd)
    for i in np.argsort(-np.abs(gl))[:4]:
        lp = loggf0.copy(); lp[i] += h
        lm = loggf0.copy(); lm[i] -= h
        fd = (chi2_at(M, fobs, lp, np.zeros(ne), 1.0) - chi2_at(M, fobs, lm, np.zeros(ne), 1.0)) / (2 * h)
        assert abs(gl[i] - fd) <= 1e-3 * abs(fd), (i, gl[i], fd)
    hv = 0.02
    fd = (chi2_at(M, fobs, loggf0, np.zeros(ne), 1.0 + hv) - chi2_at(M, fobs, loggf0, np.zeros(ne), 1.0 - hv)) / (2 * hv)
    assert abs(gv - fd) <= 2e-3 * abs(fd), (gv, fd)
    assert np.max(np.abs(gl - gl_pp)) > 1e-3 * np.max(np.abs(gl_pp))
    M.close()


def test_mixed_forward_gradients_match_fp64(fsg):
    M64, arr = model(fsg, fsg.PREC_FP64)
    loggf0 = np.log10(arr["gf"].astype(np.float64))
    fobs = target(M64, loggf0)
    g64 = grads(M64, loggf0, fobs)
    M64.close()
    M32, _ = model(fsg, fsg.PREC_MIXED)
    g32 = grads(M32, loggf0, fobs)
    M32.close()
    assert np.max(np.abs(g32[0] - g64[0])) <= 1e-4 * np.max(np.abs(g64[0]))
    assert np.max(np.abs(g32[1] - g64[1])) <= 1e-4 * np.max(np.abs(g64[1]))
    assert abs(g32[2] - g64[2]) <= 1e-4 * abs(g64[2])


def test_abundance_gradient_vs_oracle_fd(fsg, oracle_mod):
    """FP64 reference gradient: central differences of the oracle's synthesis (CPU)."""
    from fastspec_b200 import adjoint as AD
    M, arr = model(fsg, fsg.PREC_FP64)
    loggf0 = np.log10(arr["gf"].astype(np.float64))
    fobs = target(M, loggf0)
    _, ga, _ = grads(M, loggf0, fobs)
    M.close()
    grid, st, meta, co, _ = case()
    x, w, _ = oracle_mod.mu_quadrature(1, 7)
    fo = fobs.cpu().numpy()
    sp_el = [str(s).split()[0] for s in meta["species"]]

    def chi2(el, dh):
        s2 = dict(st)
        f = np.asarray(st["fractionpf"], np.float64).copy()
        for k, e in enumerate(sp_el):
            if e == el:
                f[:, k] *= 10.0 ** dh
        s2["fractionpf"] = f.astype(np.float32)
        S = oracle_mod.State(grid, s2, contopac=co, vmicro=1.0)
        r = oracle_mod.lineop_calc(S, oracle_mod.Lines(**arr, kind=2), list_type=2)
        sfl, sfc = oracle_mod.disk_integ(w, *oracle_mod.radtran(S, x, r["lineopac"]))
        return float((((sfl / sfc - fo) / SIG) ** 2).sum())

    for el in ("Fe", "Ni", "Ca"):
        fd = (chi2(el, 1e-4) - chi2(el, -1e-4)) / 2e-4
        e = AD.ELEMENTS.index(el)
        assert abs(ga[e] - fd) <= 1e-3 * abs(fd) + 1e-3, (el, ga[e], fd)
