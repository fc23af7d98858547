"""The CUDA paths against the golden fixtures generated from the reference's
own CPU kernels (tests/golden/make_golden.py). Every call goes through the C
ABI. Tolerances: FP64 direct paths 1e-12 (L2 and max |err| / max |V|), the
tensor-core path 1e-6, FP32 1e-5."""
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(),
                                 reason="needs a CUDA device")]

import oskar_b200 as ob  # noqa: E402
from golden_cases import C0, c1_identity_e, load, rel_err  # noqa: E402


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def c1_direct(g, real):
    """uvw -> K -> join -> direct correlation on the GPU, per dump."""
    s = "d" if real == np.float64 else "f"
    tdt = torch.float64 if real == np.float64 else torch.float32
    x, y, z = (np.ascontiguousarray(a, dtype=real) for a in g["ecef"])
    nst = x.size
    l, m, n, I, Q, U, V = (dev(np.asarray(g[k], real))
                           for k in "l m n I Q U V".split())
    nsrc = l.numel()
    E = dev(c1_identity_e(nst, nsrc, real))
    freq = float(g["freq"])
    nbl = nst * (nst - 1) // 2
    stream = ob.stream_ptr()
    out = []
    for t, ha in enumerate(g["ha"]):
        if real == np.float64:
            uvw = [torch.zeros(nst, dtype=tdt, device="cuda")
                   for _ in range(3)]
            ob.call("oskb_convert_ecef_to_station_uvw_d", nst, dev(x),
                    dev(y), dev(z), 0.0, float(g["dec0"]), float(ha), 0, 0,
                    *uvw, stream)
        else:
            uvw = [dev(np.asarray(a, real)) for a in g["uvw"][t]]
        K = torch.zeros(2 * nst * nsrc, dtype=tdt, device="cuda")
        ob.call("oskb_evaluate_jones_K_" + s, nsrc, l, m, n, nst, *uvw,
                2 * math.pi * freq / C0, I, 0.0, 3e38, 0, K, stream)
        J = torch.zeros(8 * nst * nsrc, dtype=tdt, device="cuda")
        ob.call("oskb_mem_multiply_" + s, 3, 0, 0, 0, nst * nsrc, K, E, J,
                stream)
        vis = torch.zeros(8 * nbl, dtype=tdt, device="cuda")
        zz = torch.zeros(nst, dtype=tdt, device="cuda")
        ob.call("oskb_cross_correlate_" + s, 0, 0, nsrc, nst, 0, J, I, Q, U,
                V, l, m, n, None, None, None, *uvw, zz, zz, 0.0, 3e38,
                freq / C0, 0.0, 0.0, 0.0, 0.0, vis, stream)
        out.append(vis.cpu().numpy().reshape(nbl, 8))
    torch.cuda.synchronize()
    return np.stack(out)


def test_c1_direct_fp64():
    g = load("c1_vis.npz")
    l2, mx = rel_err(c1_direct(g, np.float64), g["vis"])
    assert l2 <= 1e-12 and mx <= 1e-12, (l2, mx)


def test_c1_direct_fp32():
    g = load("f32_vis.npz")
    l2, mx = rel_err(c1_direct(g, np.float32), g["vis"])
    assert l2 <= 1e-5 and mx <= 1e-5, (l2, mx)


def test_c1_tensor_core_block():
    """All 10 dumps in one fused block call (FP64 phase, identity beam)."""
    g = load("c1_vis.npz")
    nst, nsrc = g["ecef"].shape[1], g["l"].size
    ntime, nbl = len(g["ha"]), nst * (nst - 1) // 2
    E = dev(c1_identity_e(nst, nsrc, np.float32))
    sky = [dev(g[k]) for k in "l m n I Q U V".split()]
    vis = torch.zeros(ntime * nbl * 8, dtype=torch.float64, device="cuda")
    ob.call("oskb_correlate_block_tc", 0, nsrc, nst, ntime, 1, E, *sky,
            dev(g["uvw"]), dev(np.array([float(g["freq"]) / C0])), 0.0, 3e38,
            vis, None, 0, ob.stream_ptr())
    torch.cuda.synchronize()
    got = vis.cpu().numpy().reshape(ntime, nbl, 8)
    for t in range(ntime):
        l2, mx = rel_err(got[t], g["vis"][t])
        assert l2 <= 1e-6 and mx <= 1e-6, (t, l2, mx)


def test_c1_host_block_driver():
    """The same through the host-buffer block driver (copies included)."""
    g = load("c1_vis.npz")
    nst, nsrc = g["ecef"].shape[1], g["l"].size
    ntime, nbl = len(g["ha"]), nst * (nst - 1) // 2
    E = c1_identity_e(nst, nsrc, np.float32)
    vis = np.zeros((ntime, 1, nbl, 8))
    ob.call("oskb_run_block_tc_host", 0, nsrc, nst, ntime, 1, E,
            *[np.ascontiguousarray(g[k]) for k in "l m n I Q U V".split()],
            np.ascontiguousarray(g["uvw"]), np.array([float(g["freq"])]),
            0.0, 3e38, vis, ob.stream_ptr())
    l2, mx = rel_err(vis[:, 0], g["vis"])
    assert l2 <= 1e-6 and mx <= 1e-6, (l2, mx)


def test_c1_pipelined_plan():
    """The pipelined host-buffer plan: three blocks in flight (the c1
    dumps split 4 + 4 + 2 would not share a shape, so each block is the
    first 5 dumps with a different order of dumps), every block equal to
    the golden visibilities of its dumps."""
    import ctypes
    g = load("c1_vis.npz")
    nst, nsrc = g["ecef"].shape[1], g["l"].size
    nbl = nst * (nst - 1) // 2
    nt = 5
    E = c1_identity_e(nst, nsrc, np.float32)
    lib = ob.load()
    st = ctypes.c_int(0)
    freqs = np.array([float(g["freq"])])
    plan = lib.oskb_tc_plan_create(0, nsrc, nst, nt, 1, freqs.ctypes.data,
                                   0.0, 3e38, ctypes.addressof(st))
    assert st.value == 0 and plan
    try:
        ob.call("oskb_tc_plan_set_sky", plan, *[np.ascontiguousarray(g[k])
                                               for k in "l m n I Q U V".split()])
        orders = [list(range(0, 5)), list(range(5, 10)), [9, 0, 4, 2, 7]]
        uvws = [np.ascontiguousarray(g["uvw"][o]) for o in orders]
        outs = [np.zeros((nt, 1, nbl, 8)) for _ in orders]
        for u, o in zip(uvws, outs):
            assert ob.call("oskb_tc_plan_enqueue", plan, E, u, o) == 0
        assert ob.call("oskb_tc_plan_wait", plan) == 0
        for o, order in zip(outs, orders):
            l2, mx = rel_err(o[:, 0], g["vis"][order])
            assert l2 <= 1e-6 and mx <= 1e-6, (order, l2, mx)
    finally:
        lib.oskb_tc_plan_free(plan)


@pytest.mark.parametrize("matrix", [True, False])
def test_smearing_gaussian(matrix):
    g = load("smear_vis.npz")
    nst, nsrc = g["u"].size, g["l"].size
    nbl = nst * (nst - 1) // 2
    d = {k: dev(g[k]) for k in "J Js I Q U V l m n a b c u v w x y".split()}
    scal = (0.0, 3e38, float(g["freq"]) / C0, float(g["bw"] / g["freq"]),
            float(g["tavg"]), float(g["gha0"]), float(g["dec0"]))
    if matrix:
        vis = torch.zeros(8 * nbl, dtype=torch.float64, device="cuda")
        ob.call("oskb_cross_correlate_d", 0, 1, nsrc, nst, 0, d["J"],
                d["I"], d["Q"], d["U"], d["V"], d["l"], d["m"], d["n"],
                d["a"], d["b"], d["c"], d["u"], d["v"], d["w"], d["x"],
                d["y"], *scal, vis, ob.stream_ptr())
        ref = g["vis"]
    else:
        vis = torch.zeros(2 * nbl, dtype=torch.float64, device="cuda")
        ob.call("oskb_cross_correlate_scalar_d", 1, 1, nsrc, nst, 0, d["Js"],
                d["I"], d["l"], d["m"], d["n"], d["a"], d["b"], d["c"],
                d["u"], d["v"], d["w"], d["x"], d["y"], *scal, vis,
                ob.stream_ptr())
        ref = g["vis_scalar"]
    torch.cuda.synchronize()
    l2, mx = rel_err(vis.cpu().numpy(), ref)
    assert l2 <= 1e-12 and mx <= 1e-12, (l2, mx)


def test_dftw():
    g = load("dftw.npz")
    n_in, n_out, n_c = g["xi"].size, g["xo"].size, int(g["n_c"])
    k = float(g["k"])
    out_m = torch.zeros(n_out * 8, dtype=torch.float64, device="cuda")
    ob.call("oskb_dftw_d", 1, n_in, k, dev(g["w"]), dev(g["xi"]),
            dev(g["yi"]), dev(g["zi"]), 0, n_out, dev(g["xo"]), dev(g["yo"]),
            dev(g["zo"]), dev(g["idx"]), dev(g["data_m"]), 1, 1, 0, out_m,
            1.0 / n_in, ob.stream_ptr())
    out_c = torch.zeros(n_out * 2, dtype=torch.float64, device="cuda")
    ob.call("oskb_dftw_d", 0, n_c, k, dev(g["w"]), dev(g["xi"]),
            dev(g["yi"]), None, 0, n_out, dev(g["xo"]), dev(g["yo"]), None,
            None, dev(g["data_c"]), 1, 1, 0, out_c, 1.0, ob.stream_ptr())
    torch.cuda.synchronize()
    assert max(rel_err(out_m.cpu().numpy(), g["out_m"])) <= 1e-12
    assert max(rel_err(out_c.cpu().numpy(), g["out_c"])) <= 1e-12
