"""GPU parity of the tensor-core compensated cross-correlation.

Both tensor-core forms must agree with the FP64 CPU oracle to
    L2 relative <= 1e-6  and  max |err| <= 1e-6 * max |V|
on every test here (the stated tolerance of the compensated path):
  - the integer form (the default): sources ordered into amplitude buckets,
    each with its own scale; entries as 24-bit fixed point in three signed
    8-bit limbs, six 8-bit MMAs per K step into exact 32-bit integer
    accumulators, FP64 phase;
  - the FP16 form (OSKB_TC_ARITH=fp16 or any OSKB_TC_TILE): FP16 hi/lo
    split, three products, FP32 accumulation drained to FP64, FP64 phase.
Calls go through the C ABI with torch device buffers.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(),
                                 reason="needs a CUDA device")]

import oskar_b200 as ob  # noqa: E402
from oracle_lib import oracle  # noqa: E402

TOL = 1e-6
C0 = 299792458.0


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def errors(got, ref):
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    l2 = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    mx = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
    return l2, mx


def sky(rng, nsrc, radius_deg=5.0, smin=0.01, smax=10.0):
    r = np.sqrt(rng.uniform(0, 1, nsrc)) * np.sin(np.radians(radius_deg))
    th = rng.uniform(0, 2 * np.pi, nsrc)
    l, m = r * np.cos(th), r * np.sin(th)
    n = np.sqrt(1 - l * l - m * m)
    a = -0.5
    u = rng.uniform(0, 1, nsrc)
    I = (smin ** a + u * (smax ** a - smin ** a)) ** (1 / a)
    Q, U, V = (I * rng.uniform(-0.1, 0.1, nsrc) for _ in range(3))
    return l, m, n, I, Q, U, V


def stations(rng, nst, rmax=5e3):
    r = np.exp(rng.uniform(np.log(20.0), np.log(rmax), nst))
    th = rng.uniform(0, 2 * np.pi, nst)
    return (r * np.cos(th), r * np.sin(th), rng.uniform(-30, 30, nst))


def oracle_vis(nst, nsrc, J, I, Q, U, V, l, m, n, u, v, w, inv_wl, casa=0,
               uv_min=0.0, uv_max=3e38, vis0=None, offset_out=0):
    nbl = nst * (nst - 1) // 2
    out = np.zeros(8 * (nbl + offset_out)) if vis0 is None else vis0.copy()
    z = np.zeros(nst)
    oracle().call("xcorr_matrix_d", np.float64, casa, 0, nsrc, nst,
                  offset_out, J, I, Q, U, V, l, m, n, None, None, None, u, v,
                  w, z, z, uv_min, uv_max, inv_wl, 0.0, 0.0, 0.0, 0.0, out)
    return out


@pytest.mark.parametrize("nst,nsrc", [(2, 1), (5, 33), (31, 100), (33, 64),
                                      (64, 1000), (100, 2500), (130, 777)])
@pytest.mark.parametrize("casa", [0, 1])
def test_tc_jones_api(nst, nsrc, casa):
    rng = np.random.default_rng(nst * 1000 + nsrc)
    l, m, n, I, Q, U, V = sky(rng, nsrc)
    u, v, w = stations(rng, nst)
    J = rng.normal(0, 0.3, (nst, nsrc, 8))
    J[..., 0] += 1
    J[..., 6] += 1
    J = J.ravel()
    inv_wl = 110e6 / C0
    ref = oracle_vis(nst, nsrc, J, I, Q, U, V, l, m, n, u, v, w, inv_wl,
                     casa=casa, offset_out=2)
    nbl = nst * (nst - 1) // 2
    vis = torch.zeros(8 * (nbl + 2), dtype=torch.float64, device="cuda")
    ob.call("oskb_cross_correlate_tc_d", casa, nsrc, nst, 2, dev(J), dev(I),
            dev(Q), dev(U), dev(V), dev(u), dev(v), 0.0, 3e38, inv_wl, vis,
            None, 0, ob.stream_ptr())
    torch.cuda.synchronize()
    l2, mx = errors(vis.cpu().numpy()[16:], ref[16:])
    assert l2 <= TOL and mx <= TOL, (l2, mx)
    flags = (ob._lib.ctypes.c_int * 2)()
    ob.call("oskb_tc_status", None, ob._lib.ctypes.addressof(flags),
            ob._lib.ctypes.addressof(flags) + 4)
    assert flags[0] == 0 and flags[1] == 0


def jones_case(rng, nst, nsrc, I, Q, U, V, l, m, n, casa=0):
    """oskb_cross_correlate_tc_d against the oracle on one J block."""
    u, v, w = stations(rng, nst)
    J = rng.normal(0, 0.3, (nst, nsrc, 8))
    J[..., 0] += 1
    J[..., 6] += 1
    J = J.ravel()
    inv_wl = 110e6 / C0
    ref = oracle_vis(nst, nsrc, J, I, Q, U, V, l, m, n, u, v, w, inv_wl,
                     casa=casa)
    nbl = nst * (nst - 1) // 2
    vis = torch.zeros(8 * nbl, dtype=torch.float64, device="cuda")
    ob.call("oskb_cross_correlate_tc_d", casa, nsrc, nst, 0, dev(J), dev(I),
            dev(Q), dev(U), dev(V), dev(u), dev(v), 0.0, 3e38, inv_wl, vis,
            None, 0, ob.stream_ptr())
    torch.cuda.synchronize()
    return vis.cpu().numpy(), ref


@pytest.mark.parametrize("decades", [3, 6, 12])
def test_tc_integer_dynamic_range(decades, monkeypatch):
    """Fluxes log-uniform over 3, 6 and 12 decades (entries of J C scale as
    the square root of the flux: up to 2^20 in amplitude, past the 16
    buckets of the integer image), with some sources of zero flux: the
    integer form's buckets keep every flux at full precision, the last
    bucket takes all fainter sources."""
    monkeypatch.delenv("OSKB_TC_TILE", raising=False)
    monkeypatch.delenv("OSKB_TC_ARITH", raising=False)
    rng = np.random.default_rng(700 + decades)
    nsrc = 3000
    l, m, n, I, Q, U, V = sky(rng, nsrc)
    I = 10.0 ** rng.uniform(-decades, 0, nsrc)
    Q, U, V = (I * rng.uniform(-0.1, 0.1, nsrc) for _ in range(3))
    for a in (I, Q, U, V):
        a[::97] = 0.0
    got, ref = jones_case(rng, 40, nsrc, I, Q, U, V, l, m, n)
    assert ob.load().oskb_tc_arithmetic() == 8
    l2, mx = errors(got, ref)
    assert l2 <= TOL and mx <= TOL, (l2, mx)


def test_tc_integer_long_bucket(monkeypatch):
    """20,000 sources of one flux (one bucket of 625 source blocks, so its
    accumulators drain inside the bucket as well as at its end)."""
    monkeypatch.delenv("OSKB_TC_TILE", raising=False)
    monkeypatch.delenv("OSKB_TC_ARITH", raising=False)
    rng = np.random.default_rng(71)
    nsrc = 20000
    l, m, n, I, Q, U, V = sky(rng, nsrc)
    I = np.ones(nsrc)
    Q = U = V = np.zeros(nsrc)
    got, ref = jones_case(rng, 33, nsrc, I, Q, U, V, l, m, n, casa=1)
    l2, mx = errors(got, ref)
    assert l2 <= TOL and mx <= TOL, (l2, mx)


def test_tc_integer_zero_sky(monkeypatch):
    """All fluxes zero: zero visibilities, exactly."""
    monkeypatch.delenv("OSKB_TC_TILE", raising=False)
    monkeypatch.delenv("OSKB_TC_ARITH", raising=False)
    rng = np.random.default_rng(72)
    nsrc = 100
    l, m, n, I, Q, U, V = sky(rng, nsrc)
    z = np.zeros(nsrc)
    got, _ = jones_case(rng, 9, nsrc, z, z, z, z, l, m, n)
    assert not np.any(got)


FORMS = ["fp16-128", "fp16-256", "fp16-512", "i8-128"]


def set_form(monkeypatch, form):
    """Selects a contraction form; returns the (tile columns, arithmetic)
    that oskb_tc_tile_columns / oskb_tc_arithmetic then report."""
    if form.startswith("fp16"):
        tile = int(form.split("-")[1])
        monkeypatch.setenv("OSKB_TC_TILE", str(tile))
        return tile, 16
    monkeypatch.delenv("OSKB_TC_TILE", raising=False)
    monkeypatch.delenv("OSKB_TC_ARITH", raising=False)
    return 128, 8


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("nst,nsrc,casa", [(17, 300, 0), (64, 1000, 1),
                                           (130, 777, 0), (161, 2050, 1),
                                           (200, 1200, 0)])
def test_tc_tile_widths(form, nst, nsrc, casa, monkeypatch):
    """Square (128 x 128), wide (128 x 256) and pair (256 x 256 on two CTAs)
    contraction tiles, with an even and an odd number of 32-station row
    blocks (17, 64, 130, 161 and 200 stations: one, two, five, six and
    seven blocks), against the oracle; and the integer form on square
    tiles and on 256 x 128 tiles of CTA pairs (an odd number of row blocks
    leaves the last pair's second half empty)."""
    tile, arith = set_form(monkeypatch, form)
    rng = np.random.default_rng(nst * 7 + nsrc)
    l, m, n, I, Q, U, V = sky(rng, nsrc)
    u, v, w = stations(rng, nst)
    J = rng.normal(0, 0.3, (nst, nsrc, 8))
    J[..., 0] += 1
    J[..., 6] += 1
    J = J.ravel()
    inv_wl = 130e6 / C0
    ref = oracle_vis(nst, nsrc, J, I, Q, U, V, l, m, n, u, v, w, inv_wl,
                     casa=casa)
    nbl = nst * (nst - 1) // 2
    vis = torch.zeros(8 * nbl, dtype=torch.float64, device="cuda")
    ob.call("oskb_cross_correlate_tc_d", casa, nsrc, nst, 0, dev(J), dev(I),
            dev(Q), dev(U), dev(V), dev(u), dev(v), 0.0, 3e38, inv_wl, vis,
            None, 0, ob.stream_ptr())
    torch.cuda.synchronize()
    assert ob.load().oskb_tc_tile_columns() == tile
    assert ob.load().oskb_tc_arithmetic() == arith
    l2, mx = errors(vis.cpu().numpy(), ref)
    assert l2 <= TOL and mx <= TOL, (l2, mx)
    flags = (ob._lib.ctypes.c_int * 2)()
    ob.call("oskb_tc_status", None, ob._lib.ctypes.addressof(flags),
            ob._lib.ctypes.addressof(flags) + 4)
    assert flags[0] == 0 and flags[1] == 0


@pytest.mark.parametrize("tile", [256, 512])
def test_tc_block_tile_widths_agree(tile, monkeypatch):
    """A block of 2 dumps x 3 channels at 97 stations (four row blocks)
    through the square tiles and the wide or pair tiles: within the
    compensated tolerance of each other (each is checked against the
    oracle in test_tc_tile_widths)."""
    rng = np.random.default_rng(5)
    nst, nsrc, ntime, nchan = 97, 900, 2, 3
    l, m, n, I, Q, U, V = sky(rng, nsrc)
    E = rng.normal(0, 0.1, (nst, nsrc, 8)).astype(np.float32)
    uvw = np.stack([np.stack(stations(rng, nst)) for _ in range(ntime)])
    inv_wl = (120e6 + 1e6 * np.arange(nchan)) / C0
    nbl = nst * (nst - 1) // 2
    out = {}
    for t in (128, tile):
        monkeypatch.setenv("OSKB_TC_TILE", str(t))
        vis = torch.zeros(ntime * nchan * nbl * 8, dtype=torch.float64,
                          device="cuda")
        ob.call("oskb_correlate_block_tc", 0, nsrc, nst, ntime, nchan,
                dev(E), dev(l), dev(m), dev(n), dev(I), dev(Q), dev(U),
                dev(V), dev(uvw), dev(inv_wl), 0.0, 3e38, vis, None, 0,
                ob.stream_ptr())
        torch.cuda.synchronize()
        assert ob.load().oskb_tc_tile_columns() == t
        out[t] = vis.cpu().numpy()
    l2, mx = errors(out[tile], out[128])
    assert l2 <= TOL and mx <= TOL, (l2, mx)


def test_tc_accumulates_and_filters():
    """vis is accumulated (+=), and baselines outside the uv range are left
    untouched, as in the reference dispatcher."""
    rng = np.random.default_rng(9)
    nst, nsrc = 40, 300
    l, m, n, I, Q, U, V = sky(rng, nsrc)
    u, v, w = stations(rng, nst, rmax=800.0)
    J = rng.normal(0, 0.2, (nst, nsrc, 8)).ravel()
    inv_wl = 100e6 / C0
    nbl = nst * (nst - 1) // 2
    vis0 = rng.normal(0, 1, 8 * nbl)
    ref = oracle_vis(nst, nsrc, J, I, Q, U, V, l, m, n, u, v, w, inv_wl,
                     uv_min=20.0, uv_max=150.0, vis0=vis0)
    vis = dev(vis0)
    ob.call("oskb_cross_correlate_tc_d", 0, nsrc, nst, 0, dev(J), dev(I),
            dev(Q), dev(U), dev(V), dev(u), dev(v), 20.0, 150.0, inv_wl, vis,
            None, 0, ob.stream_ptr())
    torch.cuda.synchronize()
    got = vis.cpu().numpy()
    l2, mx = errors(got - vis0, ref - vis0)
    assert l2 <= TOL and mx <= TOL, (l2, mx)
    unchanged = np.all((got == vis0).reshape(-1, 8), axis=1)
    assert unchanged.any() and not unchanged.all()


def test_tc_caller_workspace_too_small():
    nst, nsrc = 8, 40
    need = ob.call("oskb_cross_correlate_tc_workspace_bytes", nsrc, nst,
                   check=False)
    ws = torch.zeros(need // 2, dtype=torch.uint8, device="cuda")
    z = torch.zeros(8 * nst * nsrc, dtype=torch.float64, device="cuda")
    st = ob.call("oskb_cross_correlate_tc_d", 0, nsrc, nst, 0, z, z, z, z,
                 z, z, z, 0.0, 3e38, 1.0, z, ws, ws.numel(), ob.stream_ptr(),
                 check=False)
    assert st == -6


@pytest.mark.parametrize("nst,nsrc,ntime,nchan", [(17, 50, 1, 3),
                                                  (64, 1500, 2, 2),
                                                  (97, 640, 3, 1)])
def test_tc_fused_block(nst, nsrc, ntime, nchan):
    """K (FP64 phase) x E x brightness for a block of (time, channel)
    problems in one call, against the oracle's Jones K -> join -> correlate
    for each problem."""
    rng = np.random.default_rng(nst + nsrc)
    l, m, n, I, Q, U, V = sky(rng, nsrc)
    E = rng.normal(0, 0.1, (nst, nsrc, 8))
    E[..., 0] += 1
    E[..., 6] += 1
    E32 = E.astype(np.float32)
    uvw = np.stack([np.stack(stations(rng, nst, rmax=20e3))
                    for _ in range(ntime)])
    inv_wl = (100e6 + 7e6 * np.arange(nchan)) / C0
    nbl = nst * (nst - 1) // 2
    vis = torch.zeros(ntime * nchan * nbl * 8, dtype=torch.float64,
                      device="cuda")
    ob.call("oskb_correlate_block_tc", 0, nsrc, nst, ntime, nchan, dev(E32),
            dev(l), dev(m), dev(n), dev(I), dev(Q), dev(U), dev(V), dev(uvw),
            dev(inv_wl), 0.0, 3e38, vis, None, 0, ob.stream_ptr())
    torch.cuda.synchronize()
    got = vis.cpu().numpy().reshape(ntime, nchan, -1)
    Ed = E32.astype(np.float64).ravel()
    for t in range(ntime):
        u, v, w = uvw[t]
        for c in range(nchan):
            K = np.zeros(2 * nst * nsrc)
            oracle().call("jones_k_d", np.float64, nsrc, l, m, n, nst, u, v,
                          w, 2 * np.pi * inv_wl[c], I, 0.0, 1e300, 0, K)
            J = np.zeros(8 * nst * nsrc)
            oracle().call("mem_mul_cm_m_d", np.float64, nst * nsrc, K, Ed, J)
            ref = oracle_vis(nst, nsrc, J, I, Q, U, V, l, m, n, u, v, w,
                             inv_wl[c])
            l2, mx = errors(got[t, c], ref)
            assert l2 <= TOL and mx <= TOL, (t, c, l2, mx)


def test_tc_block_small_workspace_groups():
    """A caller workspace holding one image forces one problem per group;
    the result must equal the single-group run."""
    rng = np.random.default_rng(77)
    nst, nsrc, ntime, nchan = 40, 200, 2, 3
    l, m, n, I, Q, U, V = sky(rng, nsrc)
    E = rng.normal(0, 0.1, (nst, nsrc, 8)).astype(np.float32)
    uvw = np.stack([np.stack(stations(rng, nst)) for _ in range(ntime)])
    inv_wl = (120e6 + 1e6 * np.arange(nchan)) / C0
    nbl = nst * (nst - 1) // 2
    args = [dev(E), dev(l), dev(m), dev(n), dev(I), dev(Q), dev(U), dev(V),
            dev(uvw), dev(inv_wl), 0.0, 3e38]
    out = []
    for nprob in (ntime * nchan, 1):
        need = ob.call("oskb_correlate_block_tc_workspace_bytes", nsrc, nst,
                       nprob, check=False)
        ws = torch.empty(need, dtype=torch.uint8, device="cuda")
        vis = torch.zeros(ntime * nchan * nbl * 8, dtype=torch.float64,
                          device="cuda")
        ob.call("oskb_correlate_block_tc", 0, nsrc, nst, ntime, nchan, *args,
                vis, ws, ws.numel(), ob.stream_ptr())
        torch.cuda.synchronize()
        out.append(vis.cpu().numpy())
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("form", FORMS)
def test_tc_block_auto_correlations_fused(form, monkeypatch):
    """Auto-correlations from the same contraction (the diagonal station
    pairs of the diagonal tiles) against the oracle's auto-correlation of
    J = K E per (dump, channel), to the compensated tolerance; the cross
    visibilities are the same bits as without them."""
    tile, arith = set_form(monkeypatch, form)
    rng = np.random.default_rng(21)
    nst, nsrc, ntime, nchan = 97, 700, 2, 2
    l, m, n, I, Q, U, V = sky(rng, nsrc)
    E = rng.normal(0, 0.1, (nst, nsrc, 8))
    E[..., 0] += 1
    E[..., 6] += 1
    E32 = E.astype(np.float32)
    uvw = np.stack([np.stack(stations(rng, nst, rmax=20e3))
                    for _ in range(ntime)])
    inv_wl = (100e6 + 7e6 * np.arange(nchan)) / C0
    nbl = nst * (nst - 1) // 2
    args = [dev(E32), dev(l), dev(m), dev(n), dev(I), dev(Q), dev(U), dev(V),
            dev(uvw), dev(inv_wl), 0.0, 3e38]
    vis = torch.zeros(ntime * nchan * nbl * 8, dtype=torch.float64,
                      device="cuda")
    autos = torch.zeros(ntime * nchan * nst * 8, dtype=torch.float64,
                        device="cuda")
    ob.call("oskb_correlate_block_tc_auto", 0, nsrc, nst, ntime, nchan,
            *args, vis, autos, None, 0, ob.stream_ptr())
    vis0 = torch.zeros_like(vis)
    ob.call("oskb_correlate_block_tc", 0, nsrc, nst, ntime, nchan, *args,
            vis0, None, 0, ob.stream_ptr())
    torch.cuda.synchronize()
    assert ob.load().oskb_tc_tile_columns() == tile
    assert ob.load().oskb_tc_arithmetic() == arith
    assert torch.equal(vis, vis0)
    got = autos.cpu().numpy().reshape(ntime, nchan, -1)
    Ed = E32.astype(np.float64).ravel()
    for t in range(ntime):
        u, v, w = uvw[t]
        for c in range(nchan):
            K = np.zeros(2 * nst * nsrc)
            oracle().call("jones_k_d", np.float64, nsrc, l, m, n, nst, u, v,
                          w, 2 * np.pi * inv_wl[c], I, 0.0, 1e300, 0, K)
            J = np.zeros(8 * nst * nsrc)
            oracle().call("mem_mul_cm_m_d", np.float64, nst * nsrc, K, Ed, J)
            ref = np.zeros(8 * nst)
            oracle().call("acorr_matrix_d", np.float64, nsrc, nst, 0, J, I,
                          Q, U, V, ref)
            l2, mx = errors(got[t, c], ref)
            assert l2 <= TOL and mx <= TOL, (t, c, l2, mx)


@pytest.mark.parametrize("nst,nsrc,casa", [(2, 1, 0), (33, 64, 1),
                                           (64, 1000, 0), (130, 777, 1)])
def test_tc_fp32_entry(nst, nsrc, casa):
    """oskb_cross_correlate_tc_f: FP32 J, fluxes, u, v and visibilities
    (as oskb_cross_correlate_f takes them), the integer form's sums added
    into the FP32 visibilities; against the oracle run on the same
    FP32-rounded inputs, to 1e-6, over two calls in a row (the second adds
    to the first) with an output offset."""
    rng = np.random.default_rng(5 * nst + nsrc)
    l, m, n, I, Q, U, V = sky(rng, nsrc)
    u, v, w = stations(rng, nst)
    J = rng.normal(0, 0.3, (nst, nsrc, 8))
    J[..., 0] += 1
    J[..., 6] += 1
    f32 = lambda a: np.asarray(a, np.float32)
    J32, I32, Q32, U32, V32, u32, v32 = map(f32, (J.ravel(), I, Q, U, V, u,
                                                  v))
    inv_wl = np.float32(110e6 / C0)
    up = lambda a: a.astype(np.float64)
    ref = oracle_vis(nst, nsrc, up(J32), up(I32), up(Q32), up(U32), up(V32),
                     l, m, n, up(u32), up(v32), w, float(inv_wl), casa=casa,
                     offset_out=1)
    nbl = nst * (nst - 1) // 2
    vis = torch.zeros(8 * (nbl + 1), dtype=torch.float32, device="cuda")
    for _ in range(2):
        ob.call("oskb_cross_correlate_tc_f", casa, nsrc, nst, 1, dev(J32),
                dev(I32), dev(Q32), dev(U32), dev(V32), dev(u32), dev(v32),
                0.0, 3e38, inv_wl, vis, None, 0, ob.stream_ptr())
    torch.cuda.synchronize()
    got = vis.cpu().numpy().astype(np.float64)
    assert not np.any(got[:8])
    l2, mx = errors(got[8:], 2 * ref[8:])
    assert l2 <= TOL and mx <= TOL, (l2, mx)


def test_tc_fp32_entry_not_psd():
    rng = np.random.default_rng(66)
    nst, nsrc = 20, 200
    l, m, n, I, Q, U, V = sky(rng, nsrc)
    Q = Q.copy()
    Q[9] = 2.5 * I[9]
    u, v, w = stations(rng, nst)
    J = rng.normal(0, 0.3, (nst, nsrc, 8)).astype(np.float32)
    f32 = lambda a: dev(np.asarray(a, np.float32))
    nbl = nst * (nst - 1) // 2
    vis = torch.zeros(8 * nbl, dtype=torch.float32, device="cuda")
    ob.call("oskb_cross_correlate_tc_f", 0, nsrc, nst, 0, dev(J), f32(I),
            f32(Q), f32(U), f32(V), f32(u), f32(v), 0.0, 3e38, 1.0, vis,
            None, 0, ob.stream_ptr())
    torch.cuda.synchronize()
    flags = (ob._lib.ctypes.c_int * 2)()
    ob.call("oskb_tc_status", None, ob._lib.ctypes.addressof(flags),
            ob._lib.ctypes.addressof(flags) + 4)
    assert flags[0] & 1 and flags[1] == 0
    assert not np.any(vis.cpu().numpy())
