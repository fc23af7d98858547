"""The CPU oracle against the golden fixtures generated from the reference's
own CPU kernels (tests/golden/make_golden.py). These run without the
reference source tree: the fixtures are committed data."""
import numpy as np

from golden_cases import c1_oracle, load, rel_err
from oracle_lib import oracle


def test_c1_chain_fp64():
    g = load("c1_vis.npz")
    got = c1_oracle(g, oracle())
    l2, mx = rel_err(got, g["vis"])
    assert l2 < 1e-14 and mx < 1e-14, (l2, mx)


def test_c1_chain_fp32():
    g = load("f32_vis.npz")
    got = c1_oracle(g, oracle(), np.float32)
    l2, mx = rel_err(got, g["vis"])
    assert l2 < 1e-6 and mx < 1e-6, (l2, mx)


def test_smearing_gaussian_matrix_and_scalar():
    g = load("smear_vis.npz")
    nst, nsrc = g["u"].size, g["l"].size
    nbl = nst * (nst - 1) // 2
    common = [g[k] for k in "l m n a b c u v w x y".split()]
    scal = [0.0, 3e38, float(g["freq"]) / 299792458.0,
            float(g["bw"] / g["freq"]), float(g["tavg"]), float(g["gha0"]),
            float(g["dec0"])]
    vis = np.zeros(8 * nbl)
    oracle().call("xcorr_matrix_d", np.float64, 0, 1, nsrc, nst, 0, g["J"],
                  g["I"], g["Q"], g["U"], g["V"], *common, *scal, vis)
    l2, mx = rel_err(vis, g["vis"])
    assert l2 < 1e-14 and mx < 1e-14, (l2, mx)
    vis_s = np.zeros(2 * nbl)
    oracle().call("xcorr_scalar_d", np.float64, 1, 1, nsrc, nst, 0, g["Js"],
                  g["I"], g["Q"], g["U"], g["V"], *common, *scal, vis_s)
    l2, mx = rel_err(vis_s, g["vis_scalar"])
    assert l2 < 1e-14 and mx < 1e-14, (l2, mx)


def test_dftw():
    g = load("dftw.npz")
    n_in, n_out, n_c = g["xi"].size, g["xo"].size, int(g["n_c"])
    out_m = np.zeros(n_out * 8)
    oracle().call("dftw_d", np.float64, 1, 1, n_in, float(g["k"]), g["w"],
                  g["xi"], g["yi"], g["zi"], 0, n_out, g["xo"], g["yo"],
                  g["zo"], g["idx"], g["data_m"], 1, 1, 0, out_m,
                  1.0 / n_in)
    assert rel_err(out_m, g["out_m"])[0] < 1e-14
    out_c = np.zeros(n_out * 2)
    oracle().call("dftw_d", np.float64, 0, 0, n_c, float(g["k"]), g["w"],
                  g["xi"], g["yi"], None, 0, n_out, g["xo"], g["yo"], None,
                  None, g["data_c"], 1, 1, 0, out_c, 1.0)
    assert rel_err(out_c, g["out_c"])[0] < 1e-14
