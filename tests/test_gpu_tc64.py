"""GPU parity of the FP64-class tensor-core cross-correlation
(oskb_cross_correlate_tc64_d): 48-bit fixed-point entries in six signed
8-bit limbs on the integer tensor cores, sources in amplitude buckets.
It must agree with the FP64 CPU oracle to
    L2 relative <= 1e-12  and  max |err| <= 1e-12 * max |V|
(the FP64 paths' bound), including skies whose fluxes span many decades;
a brightness matrix that is not positive semi-definite leaves vis
untouched and sets the status flag. Calls go through the C ABI with torch
device buffers."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(),
                                 reason="needs a CUDA device")]

import oskar_b200 as ob  # noqa: E402
from oracle_lib import oracle  # noqa: E402
from test_gpu_tc import C0, dev, errors, oracle_vis, sky, stations  # noqa: E402

TOL = 1e-12


def run(nst, nsrc, J, I, Q, U, V, u, v, inv_wl, casa=0, offset_out=0,
        uv_min=0.0, uv_max=3e38, ws=None):
    nbl = nst * (nst - 1) // 2
    vis = torch.zeros(8 * (nbl + offset_out), dtype=torch.float64,
                      device="cuda")
    ws_bytes = 0 if ws is None else ws.numel()
    err = ob.call("oskb_cross_correlate_tc64_d", casa, nsrc, nst, offset_out,
                  dev(J), dev(I), dev(Q), dev(U), dev(V), dev(u), dev(v),
                  uv_min, uv_max, inv_wl, vis, ws, ws_bytes, ob.stream_ptr(),
                  check=False)
    torch.cuda.synchronize()
    flags = (ctypes.c_int * 2)()
    ob.call("oskb_tc_status", ws, ctypes.addressof(flags),
            ctypes.addressof(flags) + 4)
    return err, vis.cpu().numpy(), flags[0], flags[1]


def case(rng, nst, nsrc, decades=None):
    l, m, n, I, Q, U, V = sky(rng, nsrc)
    if decades is not None:
        I = 10.0 ** rng.uniform(-decades, 0, nsrc)
        Q, U, V = (I * rng.uniform(-0.1, 0.1, nsrc) for _ in range(3))
    u, v, w = stations(rng, nst)
    J = rng.normal(0, 0.3, (nst, nsrc, 8))
    J[..., 0] += 1
    J[..., 6] += 1
    return l, m, n, I, Q, U, V, u, v, w, J.ravel()


@pytest.mark.parametrize("nst,nsrc", [(2, 1), (5, 33), (31, 100), (33, 64),
                                      (64, 1000), (100, 2500), (130, 777),
                                      (161, 2050)])
@pytest.mark.parametrize("casa", [0, 1])
def test_tc64_against_oracle(nst, nsrc, casa):
    rng = np.random.default_rng(nst * 1000 + nsrc + 7)
    l, m, n, I, Q, U, V, u, v, w, J = case(rng, nst, nsrc)
    inv_wl = 110e6 / C0
    ref = oracle_vis(nst, nsrc, J, I, Q, U, V, l, m, n, u, v, w, inv_wl,
                     casa=casa, offset_out=2)
    err, got, flags, wait = run(nst, nsrc, J, I, Q, U, V, u, v, inv_wl,
                                casa=casa, offset_out=2)
    assert err == 0 and flags == 0 and wait == 0
    l2, mx = errors(got[16:], ref[16:])
    assert l2 <= TOL and mx <= TOL, (l2, mx)
    assert not np.any(got[:16])


@pytest.mark.parametrize("decades", [3, 6, 12])
def test_tc64_dynamic_range(decades):
    """Fluxes log-uniform over up to 12 decades, some zero: every bucket
    and the catch-all last one, at FP64-class accuracy."""
    rng = np.random.default_rng(900 + decades)
    nst, nsrc = 40, 3000
    l, m, n, I, Q, U, V, u, v, w, J = case(rng, nst, nsrc, decades)
    for a in (I, Q, U, V):
        a[::97] = 0.0
    inv_wl = 150e6 / C0
    ref = oracle_vis(nst, nsrc, J, I, Q, U, V, l, m, n, u, v, w, inv_wl)
    err, got, flags, _ = run(nst, nsrc, J, I, Q, U, V, u, v, inv_wl)
    assert err == 0 and flags == 0
    l2, mx = errors(got, ref)
    assert l2 <= TOL and mx <= TOL, (l2, mx)


def test_tc64_long_bucket_and_uv_filter():
    """20,000 sources of one flux (one bucket of 625 source blocks: three
    chunks of at most 256), with a uv filter that drops some baselines."""
    rng = np.random.default_rng(91)
    nst, nsrc = 33, 20000
    l, m, n, I, Q, U, V, u, v, w, J = case(rng, nst, nsrc)
    I = np.ones(nsrc)
    Q = U = V = np.zeros(nsrc)
    inv_wl = 120e6 / C0
    ref = oracle_vis(nst, nsrc, J, I, Q, U, V, l, m, n, u, v, w, inv_wl,
                     casa=1, uv_min=200.0, uv_max=2500.0)
    err, got, flags, _ = run(nst, nsrc, J, I, Q, U, V, u, v, inv_wl, casa=1,
                             uv_min=200.0, uv_max=2500.0)
    assert err == 0 and flags == 0
    assert np.any(ref == 0.0) and np.any(ref != 0.0)
    l2, mx = errors(got, ref)
    assert l2 <= TOL and mx <= TOL, (l2, mx)
    assert np.all(got[ref == 0.0] == 0.0)


def test_tc64_not_psd_adds_nothing():
    rng = np.random.default_rng(92)
    nst, nsrc = 20, 300
    l, m, n, I, Q, U, V, u, v, w, J = case(rng, nst, nsrc)
    Q = Q.copy()
    Q[17] = 2.0 * I[17]        # I < |Q|: not positive semi-definite
    err, got, flags, wait = run(nst, nsrc, J, I, Q, U, V, u, v, 1.0)
    assert err == 0 and flags & 1 and wait == 0
    assert not np.any(got)


def test_tc64_caller_workspace():
    rng = np.random.default_rng(93)
    nst, nsrc = 70, 500
    l, m, n, I, Q, U, V, u, v, w, J = case(rng, nst, nsrc)
    need = ob.call("oskb_cross_correlate_tc64_workspace_bytes", nsrc, nst,
                   check=False)
    small = torch.empty(need - 256, dtype=torch.uint8, device="cuda")
    err, _, _, _ = run(nst, nsrc, J, I, Q, U, V, u, v, 1.3, ws=small)
    assert err != 0
    ws = torch.empty(need, dtype=torch.uint8, device="cuda")
    err, got, flags, _ = run(nst, nsrc, J, I, Q, U, V, u, v, 1.3, ws=ws)
    ref = oracle_vis(nst, nsrc, J, I, Q, U, V, l, m, n, u, v, w, 1.3)
    assert err == 0 and flags == 0
    l2, mx = errors(got, ref)
    assert l2 <= TOL and mx <= TOL, (l2, mx)


def oracle_block(nst, nsrc, E, I, Q, U, V, l, m, n, uvw, inv_wl):
    """The oracle's Jones K -> join -> FP64 correlate per (time, channel)."""
    out = []
    for t in range(uvw.shape[0]):
        u, v, w = uvw[t]
        row = []
        for kw in inv_wl:
            K = np.zeros(2 * nst * nsrc)
            oracle().call("jones_k_d", np.float64, nsrc, l, m, n, nst, u, v,
                          w, 2 * np.pi * kw, I, 0.0, 1e300, 0, K)
            J = np.zeros(8 * nst * nsrc)
            oracle().call("mem_mul_cm_m_d", np.float64, nst * nsrc, K,
                          np.ascontiguousarray(E.ravel()), J)
            row.append(oracle_vis(nst, nsrc, J, I, Q, U, V, l, m, n, u, v, w,
                                  kw))
        out.append(row)
    return np.array(out)


def run_block64(nst, nsrc, E, I, Q, U, V, l, m, n, uvw, inv_wl, ws=None):
    ntime, nchan = uvw.shape[0], len(inv_wl)
    nbl = nst * (nst - 1) // 2
    vis = torch.zeros(ntime * nchan * nbl * 8, dtype=torch.float64,
                      device="cuda")
    err = ob.call("oskb_correlate_block_tc64_d", 0, nsrc, nst, ntime, nchan,
                  dev(E), dev(l), dev(m), dev(n), dev(I), dev(Q), dev(U),
                  dev(V), dev(uvw), dev(inv_wl), 0.0, 3e38, vis, ws,
                  0 if ws is None else ws.numel(), ob.stream_ptr(),
                  check=False)
    torch.cuda.synchronize()
    flags = (ctypes.c_int * 2)()
    ob.call("oskb_tc_status", ws, ctypes.addressof(flags),
            ctypes.addressof(flags) + 4)
    return err, vis.cpu().numpy().reshape(ntime, nchan, -1), flags[0], \
        flags[1]


@pytest.mark.parametrize("nst,nsrc,ntime,nchan", [(17, 50, 1, 3),
                                                  (64, 1500, 2, 2),
                                                  (97, 640, 3, 1)])
def test_tc64_fused_block(nst, nsrc, ntime, nchan):
    """K (FP64 phase) x E x brightness for a block of (time, channel)
    problems in one call, against the oracle's Jones K -> join -> FP64
    correlate per problem, to 1e-12. Stations within 300 m, so that the
    phases (a few hundred radians) leave the two FP64 phase computations
    (the oracle's 2 pi f / c (u l + v m + w (n - 1)), here the same sum in
    turns reduced mod 1) within 1e-13 of each other."""
    rng = np.random.default_rng(31 * nst + nsrc)
    l, m, n, I, Q, U, V = sky(rng, nsrc)
    E = rng.normal(0, 0.1, (nst, nsrc, 8))
    E[..., 0] += 1
    E[..., 6] += 1
    uvw = np.stack([np.stack(stations(rng, nst, rmax=300.0))
                    for _ in range(ntime)])
    inv_wl = (100e6 + 7e6 * np.arange(nchan)) / C0
    err, got, flags, wait = run_block64(nst, nsrc, E, I, Q, U, V, l, m, n,
                                        uvw, inv_wl)
    assert err == 0 and flags == 0 and wait == 0
    ref = oracle_block(nst, nsrc, E, I, Q, U, V, l, m, n, uvw, inv_wl)
    for t in range(ntime):
        for c in range(nchan):
            l2, mx = errors(got[t, c], ref[t, c])
            assert l2 <= TOL and mx <= TOL, (t, c, l2, mx)


def test_tc64_block_groups_and_not_psd():
    """A caller workspace holding one problem's image (one problem per
    group) gives the same sums as the library-kept one; a brightness
    matrix that is not positive semi-definite adds nothing."""
    rng = np.random.default_rng(95)
    nst, nsrc, ntime, nchan = 40, 300, 2, 3
    l, m, n, I, Q, U, V = sky(rng, nsrc)
    E = rng.normal(0, 0.1, (nst, nsrc, 8))
    E[..., 0] += 1
    E[..., 6] += 1
    uvw = np.stack([np.stack(stations(rng, nst, rmax=300.0))
                    for _ in range(ntime)])
    inv_wl = (120e6 + 1e6 * np.arange(nchan)) / C0
    err, whole, flags, _ = run_block64(nst, nsrc, E, I, Q, U, V, l, m, n,
                                       uvw, inv_wl)
    assert err == 0 and flags == 0
    one = ob.call("oskb_correlate_block_tc64_workspace_bytes", nsrc, nst, 1,
                  check=False)
    ws = torch.empty(one, dtype=torch.uint8, device="cuda")
    err, grouped, flags, _ = run_block64(nst, nsrc, E, I, Q, U, V, l, m, n,
                                         uvw, inv_wl, ws=ws)
    assert err == 0 and flags == 0
    assert np.array_equal(whole, grouped)
    Q = Q.copy()
    Q[5] = 2.0 * I[5]
    err, got, flags, _ = run_block64(nst, nsrc, E, I, Q, U, V, l, m, n, uvw,
                                     inv_wl)
    assert err == 0 and flags & 1
    assert not np.any(got)


def test_tc64_block_auto_correlations():
    """Auto-correlations from the FP64-class block contraction against the
    oracle's auto-correlation of J = K E per (dump, channel), to 1e-12 (the
    phase cancels in J_p B J_p^H); the cross visibilities are the same bits
    as without them."""
    rng = np.random.default_rng(97)
    nst, nsrc, ntime, nchan = 70, 500, 2, 2
    l, m, n, I, Q, U, V = sky(rng, nsrc)
    E = rng.normal(0, 0.1, (nst, nsrc, 8))
    E[..., 0] += 1
    E[..., 6] += 1
    uvw = np.stack([np.stack(stations(rng, nst, rmax=300.0))
                    for _ in range(ntime)])
    inv_wl = (100e6 + 7e6 * np.arange(nchan)) / C0
    nbl = nst * (nst - 1) // 2
    args = [dev(E), dev(l), dev(m), dev(n), dev(I), dev(Q), dev(U), dev(V),
            dev(uvw), dev(inv_wl), 0.0, 3e38]
    vis = torch.zeros(ntime * nchan * nbl * 8, dtype=torch.float64,
                      device="cuda")
    autos = torch.zeros(ntime * nchan * nst * 8, dtype=torch.float64,
                        device="cuda")
    ob.call("oskb_correlate_block_tc64_auto_d", 0, nsrc, nst, ntime, nchan,
            *args, vis, autos, None, 0, ob.stream_ptr())
    vis0 = torch.zeros_like(vis)
    ob.call("oskb_correlate_block_tc64_d", 0, nsrc, nst, ntime, nchan, *args,
            vis0, None, 0, ob.stream_ptr())
    torch.cuda.synchronize()
    assert torch.equal(vis, vis0)
    got = autos.cpu().numpy().reshape(ntime, nchan, -1)
    for t in range(ntime):
        u, v, w = uvw[t]
        for c in range(nchan):
            K = np.zeros(2 * nst * nsrc)
            oracle().call("jones_k_d", np.float64, nsrc, l, m, n, nst, u, v,
                          w, 2 * np.pi * inv_wl[c], I, 0.0, 1e300, 0, K)
            J = np.zeros(8 * nst * nsrc)
            oracle().call("mem_mul_cm_m_d", np.float64, nst * nsrc, K,
                          np.ascontiguousarray(E.ravel()), J)
            ref = np.zeros(8 * nst)
            oracle().call("acorr_matrix_d", np.float64, nsrc, nst, 0, J, I,
                          Q, U, V, ref)
            l2, mx = errors(got[t, c], ref)
            assert l2 <= TOL and mx <= TOL, (t, c, l2, mx)
