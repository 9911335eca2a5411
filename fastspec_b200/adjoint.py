"""Differentiable synthesis: the normalised flux SfL / SfC as a torch.autograd.Function of per-line
log gf, element abundance offsets and the microturbulence.

The forward runs the CUDA path (central pass, line opacity, DELO-Bezier solver, flux quadrature).
The backward is the library's hand-written adjoint (fsg_adjoint_dev): one reverse sweep of the
solver per wavelength gives dL/dLineOpac, and every retained line's profile is recomputed over its
window to reduce dL/d ln gf and the line's share of dL/dvmicro (Faddeeva derivative of H).  With
the continuum and the equation of state held fixed, an element's abundance enters LinCop as the
same factor as gf, so dL/d[X/H] = ln 10 x (sum of dL/d ln gf over the element's lines).
"""
import math

import numpy as np
import torch

LN10 = math.log(10.0)
# element symbols, Z = 1..30
ELEMENTS = ["H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne", "Na", "Mg", "Al", "Si", "P", "S", "Cl", "Ar",
            "K", "Ca", "Sc", "Ti", "V", "Cr", "Mn", "Fe", "Co", "Ni", "Cu", "Zn"]


class FluxModel:
    """One atmosphere, grid and line list on one GPU.  species: names like 'Fe 1' per species index
    of the state (the element is the first word); lines: dict of SoA arrays (wl, elo, gf, grad, gqst,
    gvdw, spc[, ismol]); the gf column is replaced by 10**loggf at every forward."""

    def __init__(self, F, grid, state, contopac, lines, species, vmicro=1.0, precision=None, nmu=7, device=0,
                 elements=ELEMENTS, epsopac=1e-4):
        self.F, self.dev = F, torch.device("cuda", device)
        self.C = F.Context(device=device, precision=F.PREC_MIXED if precision is None else precision,
                           vmicro=vmicro, epsopac=epsopac)
        self.C.set_grid(grid["wmode"], grid["wstart"], grid["wend"], grid["dstep"])
        self.state = dict(state)
        self.fpf0 = np.asarray(state["fractionpf"], np.float32).copy()
        self.C.set_atmosphere(self.state)
        self.C.set_contopac(contopac)
        x, w, _ = F.mu_quadrature(1, nmu)
        self.C.set_mu(x, w)
        self.elements = list(elements)
        sp_el = [self.elements.index(str(s).split()[0]) for s in species]
        self.species_element = np.array(sp_el, np.int64)
        self.dt = {k: torch.from_numpy(np.ascontiguousarray(v)).to(self.dev) for k, v in lines.items()}
        self.n = int(self.dt["wl"].numel())
        from fastspec_b200.shard import GpuBackend
        self.dl = GpuBackend(F, self.C, self.dt).full
        self.line_element = torch.from_numpy(self.species_element[np.asarray(lines["spc"])]).to(self.dev)
        self.sfl = torch.empty(self.C.nwl, dtype=torch.float64, device=self.dev)
        self.sfc = torch.empty_like(self.sfl)
        self.glin = torch.empty(self.n, dtype=torch.float64, device=self.dev)
        self.gvm = torch.empty_like(self.glin)
        self.forwards = 0

    def forward(self, loggf, dabund, vmicro):
        """Normalised flux [nwl] (float64, on the model's device) for log gf [n], abundance offsets
        [len(elements)] (dex, relative to the state) and vmicro [km/s]."""
        self.dt["gf"].copy_(torch.pow(10.0, loggf.detach().to(self.dev, torch.float64)).to(torch.float32))
        da = dabund.detach().cpu().numpy().astype(np.float64)
        self.C.set_fractionpf((self.fpf0 * (10.0 ** da[self.species_element])[None, :]).astype(np.float32))
        self.C.set_vmicro(float(vmicro))
        torch.cuda.current_stream(self.dev).synchronize()
        self.C.lineop_reset()
        self.C.lineop_calc_dev(self.dl)
        self.C.radtran_dev(None, None, self.sfl.data_ptr(), self.sfc.data_ptr())
        self.forwards += 1
        self._fwd = self.forwards
        return self.sfl / self.sfc

    def backward(self, gflux):
        """dL/d(normalised flux) [nwl] -> (dL/dloggf [n], dL/ddabund [len(elements)], dL/dvmicro)."""
        if getattr(self, "_fwd", None) != self.forwards:
            raise RuntimeError("FluxModel.backward must follow its own forward")
        gs = (gflux.detach().to(self.dev, torch.float64) / self.sfc).contiguous()
        torch.cuda.current_stream(self.dev).synchronize()
        self.C.adjoint_dev(self.dl, gs.data_ptr(), self.glin.data_ptr(), self.gvm.data_ptr())
        g_loggf = LN10 * self.glin
        g_ab = torch.zeros(len(self.elements), dtype=torch.float64, device=self.dev)
        g_ab.index_add_(0, self.line_element, g_loggf)
        return g_loggf, g_ab, self.gvm.sum()

    def close(self):
        self.C.close()


class _SynthFlux(torch.autograd.Function):
    @staticmethod
    def forward(ctx, loggf, dabund, vmicro, model):
        ctx.model = model
        ctx.devs = (loggf.device, dabund.device, vmicro.device)
        return model.forward(loggf, dabund, vmicro)

    @staticmethod
    def backward(ctx, g):
        gl, ga, gv = ctx.model.backward(g)
        d0, d1, d2 = ctx.devs
        return gl.to(d0), ga.to(d1), gv.to(d2).reshape(()), None


def synth_flux(model, loggf, dabund, vmicro):
    """Normalised flux as a differentiable function of (loggf [n], dabund [30], vmicro [])."""
    return _SynthFlux.apply(loggf, dabund, vmicro, model)
