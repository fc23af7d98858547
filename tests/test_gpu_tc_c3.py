"""Tensor-core block correlation at the full C3 array, against the oracle.

The headline configuration is 512 stations log-radial to 65 km, 16 channels
(100-115 MHz) and 64 dumps of 10 s, full-Stokes point sources in a 20 deg
field and E = I + complex N(0, 0.1) per station-source. This test keeps
every station, channel and the dump geometry of that configuration and
takes a sub-sky of its first 2,048 sources (64 source blocks, so the FP32
accumulators are drained into FP64 32 times per problem), so that the FP64
oracle (Jones K -> join -> correlate per dump and channel) finishes in
seconds. It asserts, for every (dump, channel) compared,

    L2 relative <= 1e-6  and  max |err| / max |V| <= 1e-6

through oskb_correlate_block_tc (E in FP32, the oracle fed the same FP32
values) and oskb_correlate_block_tc_d (E in FP64 as an FP64 caller holds it,
the oracle fed the unrounded values, so the bound covers the rounding of E
on load too). Dumps 0 and 63 (the longest projected baselines differ by the
Earth's rotation over the observation) and channels 0, 7 and 15 (the phase
range grows with frequency) are covered. The FP64-class form
(oskb_cross_correlate_tc64_d) is held to 1e-12 on the same array.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(),
                                 reason="needs a CUDA device")]

import oskar_b200 as ob  # noqa: E402
from oracle_lib import oracle  # noqa: E402
from oskar_b200 import workloads  # noqa: E402

TOL = 1e-6
C0 = 299792458.0
NSRC = 2048
DUMPS = (0, 63)


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def errors(got, ref):
    l2 = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    mx = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
    return l2, mx


@pytest.fixture(scope="module")
def c3_sub():
    cfg = workloads.c3(num_src=NSRC)
    E = workloads.jones_e_host(cfg)
    uvw = np.stack([cfg.station_uvw(t) for t in DUMPS])
    return cfg, E, uvw


def oracle_problem(cfg, E, uvw_t, freq):
    nst, nsrc = cfg.num_st, cfg.num_src
    u, v, w = uvw_t
    K = np.zeros(2 * nst * nsrc)
    oracle().call("jones_k_d", np.float64, nsrc, cfg.l, cfg.m, cfg.n, nst, u,
                  v, w, 2 * np.pi * freq / C0, cfg.I, 0.0, 1e300, 0, K)
    J = np.zeros(8 * nst * nsrc)
    oracle().call("mem_mul_cm_m_d", np.float64, nst * nsrc, K,
                  np.ascontiguousarray(E.ravel()), J)
    out = np.zeros(8 * cfg.num_baselines)
    z = np.zeros(nst)
    oracle().call("xcorr_matrix_d", np.float64, 0, 0, nsrc, nst, 0, J, cfg.I,
                  cfg.Q, cfg.U, cfg.V, cfg.l, cfg.m, cfg.n, None, None, None,
                  u, v, w, z, z, 0.0, 3e38, freq / C0, 0.0, 0.0, 0.0, 0.0,
                  out)
    return out


def run_block(cfg, E, uvw, fp64_e):
    nch = len(cfg.freqs_hz)
    vis = torch.zeros(len(DUMPS) * nch * cfg.num_baselines * 8,
                      dtype=torch.float64, device="cuda")
    name = "oskb_correlate_block_tc_d" if fp64_e else "oskb_correlate_block_tc"
    Ed = dev(E if fp64_e else E.astype(np.float32))
    ob.call(name, 0, cfg.num_src, cfg.num_st, len(DUMPS), nch, Ed,
            dev(cfg.l), dev(cfg.m), dev(cfg.n), dev(cfg.I), dev(cfg.Q),
            dev(cfg.U), dev(cfg.V), dev(uvw), dev(cfg.freqs_hz / C0), 0.0,
            3e38, vis, None, 0, ob.stream_ptr())
    torch.cuda.synchronize()
    return vis.cpu().numpy().reshape(len(DUMPS), nch, -1)


def test_tc_c3_fp32_e_all_channels(c3_sub):
    """Every channel of dump 0 and channels 0, 7, 15 of dump 63."""
    cfg, E, uvw = c3_sub
    got = run_block(cfg, E, uvw, fp64_e=False)
    E32 = E.astype(np.float32).astype(np.float64)
    worst = (0.0, 0.0)
    for ti, chans in ((0, range(16)), (1, (0, 7, 15))):
        for c in chans:
            ref = oracle_problem(cfg, E32, uvw[ti], cfg.freqs_hz[c])
            l2, mx = errors(got[ti, c], ref)
            worst = (max(worst[0], l2), max(worst[1], mx))
            assert l2 <= TOL and mx <= TOL, (DUMPS[ti], c, l2, mx)
    print("worst L2 %.3g, max/max %.3g" % worst)


def test_tc_c3_fp64_e(c3_sub):
    """FP64 E as an FP64 caller passes it; the oracle uses it unrounded."""
    cfg, E, uvw = c3_sub
    got = run_block(cfg, E, uvw, fp64_e=True)
    for c in (0, 15):
        ref = oracle_problem(cfg, E, uvw[1], cfg.freqs_hz[c])
        l2, mx = errors(got[1, c], ref)
        assert l2 <= TOL and mx <= TOL, (DUMPS[1], c, l2, mx)


def test_tc64_c3_jones(c3_sub):
    """The FP64-class form (oskb_cross_correlate_tc64_d) on the full C3
    array: J = K E from the oracle for dump 63, channels 0 and 15, against
    the oracle's FP64 correlation of the same J to 1e-12."""
    cfg, E, uvw = c3_sub
    nst, nsrc = cfg.num_st, cfg.num_src
    u, v, w = uvw[1]
    z = np.zeros(nst)
    for c in (0, 15):
        freq = cfg.freqs_hz[c]
        K = np.zeros(2 * nst * nsrc)
        oracle().call("jones_k_d", np.float64, nsrc, cfg.l, cfg.m, cfg.n,
                      nst, u, v, w, 2 * np.pi * freq / C0, cfg.I, 0.0, 1e300,
                      0, K)
        J = np.zeros(8 * nst * nsrc)
        oracle().call("mem_mul_cm_m_d", np.float64, nst * nsrc, K,
                      np.ascontiguousarray(E.ravel()), J)
        ref = np.zeros(8 * cfg.num_baselines)
        oracle().call("xcorr_matrix_d", np.float64, 0, 0, nsrc, nst, 0, J,
                      cfg.I, cfg.Q, cfg.U, cfg.V, cfg.l, cfg.m, cfg.n, None,
                      None, None, u, v, w, z, z, 0.0, 3e38, freq / C0, 0.0,
                      0.0, 0.0, 0.0, ref)
        vis = torch.zeros(8 * cfg.num_baselines, dtype=torch.float64,
                          device="cuda")
        ob.call("oskb_cross_correlate_tc64_d", 0, nsrc, nst, 0, dev(J),
                dev(cfg.I), dev(cfg.Q), dev(cfg.U), dev(cfg.V), dev(u),
                dev(v), 0.0, 3e38, freq / C0, vis, None, 0, ob.stream_ptr())
        torch.cuda.synchronize()
        l2, mx = errors(vis.cpu().numpy(), ref)
        assert l2 <= 1e-12 and mx <= 1e-12, (c, l2, mx)


def test_tc64_block_c3(c3_sub):
    """The FP64-class fused block (oskb_correlate_block_tc64_d) on the full
    C3 array, dump 63, channels 0 and 15, E in FP64, against the oracle's
    Jones K -> join -> FP64 correlate to 5e-12: the phases reach ~3e4
    radians on the 65 km baselines, and the two FP64 phase computations
    (the oracle's 2 pi f / c times the path length, here the path length
    times f / c reduced mod 1) differ by their rounding there."""
    cfg, E, uvw = c3_sub
    nst, nsrc, nbl = cfg.num_st, cfg.num_src, cfg.num_baselines
    inv_wl = cfg.freqs_hz / C0
    vis = torch.zeros(len(DUMPS) * len(inv_wl) * nbl * 8,
                      dtype=torch.float64, device="cuda")
    ob.call("oskb_correlate_block_tc64_d", 0, nsrc, nst, len(DUMPS),
            len(inv_wl), dev(E), dev(cfg.l), dev(cfg.m), dev(cfg.n),
            dev(cfg.I), dev(cfg.Q), dev(cfg.U), dev(cfg.V), dev(uvw),
            dev(inv_wl), 0.0, 3e38, vis, None, 0, ob.stream_ptr())
    torch.cuda.synchronize()
    got = vis.cpu().numpy().reshape(len(DUMPS), len(inv_wl), -1)
    for c in (0, 15):
        ref = oracle_problem(cfg, E, uvw[1], cfg.freqs_hz[c])
        l2, mx = errors(got[1, c], ref)
        assert l2 <= 5e-12 and mx <= 5e-12, (c, l2, mx)
