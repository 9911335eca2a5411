"""Disk integration with rotation, radial-tangential macroturbulence and Gaussian broadening on the
GPU (fsg_disk_integ_conv_dev) applied to the reference's own intensities, against the reference's
broadened flux (tests/golden/pin_convol.npz) and the oracle; and the full host form after a
synthesis against the oracle."""
import numpy as np
import pytest
import torch

import helpers as H

pytestmark = pytest.mark.gpu
CASES = ["solar_0", "solar_1", "solar_2", "solar_3", "cooldwarf_0", "cooldwarf_1"]


@pytest.mark.parametrize("case", CASES)
def test_convol_against_reference(fsg, oracle_mod, case):
    d = H.load_pin("pin_convol")
    g = d[case + "_grid"]
    vs, vm, vg = d[case + "_convol"]
    x, w, r = fsg.mu_quadrature(1, 7)
    C = fsg.Context()
    C.set_grid(int(g[3]), g[0], g[1], g[2])
    C.set_mu(x, w)
    spl = torch.from_numpy(np.ascontiguousarray(d[case + "_spl"])).cuda()
    spc = torch.from_numpy(np.ascontiguousarray(d[case + "_spc"])).cuda()
    sfl = torch.empty(spl.shape[0], dtype=torch.float64, device="cuda")
    sfc = torch.empty_like(sfl)
    torch.cuda.synchronize()
    C.disk_integ_conv_dev(r, vs, vm, vg, spl.data_ptr(), spc.data_ptr(), sfl.data_ptr(), sfc.data_ptr())
    sfl, sfc = sfl.cpu().numpy(), sfc.cpu().numpy()
    assert np.max(np.abs(sfl / d[case + "_sfl"] - 1)) < 1e-12
    assert np.max(np.abs(sfc / d[case + "_sfc"] - 1)) < 1e-12
    grid = dict(wmode=int(g[3]), wstart=g[0], wend=g[1], dstep=g[2])
    wave = d[case + "_wave"]
    ox, ow, orr = oracle_mod.mu_quadrature(1, 7)
    osfl, _ = oracle_mod.disk_integ_conv(ox, ow, orr, d[case + "_spl"], d[case + "_spc"],
                                         oracle_mod.grid_dv(grid, wave), vs, vm,
                                         oracle_mod.gauss_sigma_pix(grid, wave, vg) if vg > 0 else 0.0)
    assert np.max(np.abs(sfl / osfl - 1)) < 1e-14
    C.close()


def test_synthesis_with_broadening_vs_oracle(fsg, oracle_mod):
    grid, st, co, L = None, None, None, None
    from test_gpu_lineop import solar_case, ctx_for
    grid, st, co, L = solar_case(n=300, seed=71)
    C = ctx_for(fsg, grid, st, co, fsg.PREC_FP64)
    C.lineop_calc(fsg.LineList.from_arrays(L.arrays()))
    x, w, r = fsg.mu_quadrature(1, 7)
    sfl, sfc = C.disk_integ_conv(r, 20.0, 3.0, 80000.0)
    S = oracle_mod.State(grid, st, contopac=co, vmicro=1.0)
    a = L.arrays()
    ro = oracle_mod.lineop_calc(S, oracle_mod.Lines(**a, kind=2), list_type=2)
    spl, spc = oracle_mod.radtran(S, x, ro["lineopac"])
    import fastspec_b200 as F
    wave = F.make_grid(0, grid["wstart"], grid["wend"], grid["dstep"]) + grid["wstart"]
    osfl, osfc = oracle_mod.disk_integ_conv(x, w, r, spl, spc, oracle_mod.grid_dv(grid, wave), 20.0, 3.0,
                                            oracle_mod.gauss_sigma_pix(grid, wave, 80000.0))
    assert np.max(np.abs(sfl / osfl - 1)) < 1e-9
    assert np.max(np.abs(sfc / osfc - 1)) < 1e-9


@pytest.mark.parametrize("key", ["conv_a", "conv_b"])
def test_convolve_spec_file_against_reference(fsg, tmp_path, key):
    """fastspec_b200.convolve_spec_file, the post-processing mode on the device, against the reference's
    own run of it on the same intensity file (tests/golden/fs_outputs.npz); writes fs_flux.bin."""
    from fastspec_b200 import fsio
    d = np.load(H.GOLD + "/fs_outputs.npz")
    spec, vs, vm, vg = {"conv_a": ("spec", 15.0, 3.0, 60000.0), "conv_b": ("spec_mag", 5.0, 0.0, 2.5)}[key]
    sp = str(tmp_path / "fs_spec.bin")
    with open(sp, "wb") as f:
        f.write(d[spec].tobytes())
    out = str(tmp_path / "fs_flux.bin")
    wave, sfl, sfc = fsg.convolve_spec_file(sp, vs, vm, vg, flux_path=out)
    ref = fsio.read_flux(_put(tmp_path, d[key].tobytes()))
    assert np.array_equal(wave, ref["wave"])
    assert np.max(np.abs(sfl / ref["sfl"] - 1)) < 1e-12
    assert np.max(np.abs(sfc / ref["sfc"] - 1)) < 1e-12
    back = fsio.read_flux(out)
    assert np.array_equal(back["sfl"], sfl) and np.array_equal(back["wave"], wave)


def _put(tmp_path, data):
    p = str(tmp_path / "ref_flux.bin")
    with open(p, "wb") as f:
        f.write(data)
    return p
