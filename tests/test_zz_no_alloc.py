"""The allocation-free tensor-core entry point against the workspace one.

oskb_cross_correlate_tc_noalloc_d serves callers that cannot allocate device
memory while correlating (a fixed device-memory budget, or a loop that cannot
take the device-wide synchronisation of cudaMalloc): its scratch is a fixed
64 MiB array in the library's device memory, reused by every call. This test
calls it twice in a row through the C ABI, on different inputs, and compares
each result with oskb_cross_correlate_tc_d (same kernels, caller workspace)
to the tolerance of the tensor-core tests, 1e-6, and reads the array's
status words through oskb_tc_noalloc_status after each call. It also runs
the largest call that fits the array (512 stations x 4,064 sources: 32 bytes
per station-source plus a 256-byte header) and checks that one more block of
32 sources, or a far larger call, is rejected with OSKAR's out-of-range
status. The file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(),
                                 reason="needs a CUDA device")]

import oskar_b200 as ob  # noqa: E402

TOL = 1e-6
C0 = 299792458.0


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def case(seed, nst, nsrc):
    rng = np.random.default_rng(seed)
    I = rng.uniform(0.05, 5.0, nsrc)
    Q, U, V = (I * rng.uniform(-0.1, 0.1, nsrc) for _ in range(3))
    J = rng.normal(0, 0.3, (nst, nsrc, 8))
    J[..., 0] += 1
    J[..., 6] += 1
    u, v = (rng.uniform(-3e3, 3e3, nst) for _ in range(2))
    return [dev(x) for x in (J.ravel(), I, Q, U, V, u, v)]


def noalloc_status():
    flags, wait = ctypes.c_int(-1), ctypes.c_int(-1)
    ob.call("oskb_tc_noalloc_status", ctypes.addressof(flags),
            ctypes.addressof(wait))
    return flags.value, wait.value


def compare(seed, nst, nsrc, stream):
    J, I, Q, U, V, u, v = case(seed, nst, nsrc)
    nbl = nst * (nst - 1) // 2
    kw = 120e6 / C0
    ref = torch.zeros(8 * (nbl + 1), dtype=torch.float64, device="cuda")
    need = ob.call("oskb_cross_correlate_tc_workspace_bytes", nsrc, nst,
                   check=False)
    ws = torch.empty(need, dtype=torch.uint8, device="cuda")
    ob.call("oskb_cross_correlate_tc_d", 0, nsrc, nst, 1, J, I, Q, U, V,
            u, v, 0.0, 3e38, kw, ref, ws, need, stream)
    got = torch.zeros_like(ref)
    ob.call("oskb_cross_correlate_tc_noalloc_d", 0, nsrc, nst, 1, J, I,
            Q, U, V, u, v, 0.0, 3e38, kw, got, stream)
    torch.cuda.synchronize()
    assert noalloc_status() == (0, 0)
    a, b = got.cpu().numpy(), ref.cpu().numpy()
    assert np.all(a[:8] == 0.0)  # offset_out respected
    l2 = np.linalg.norm(a - b) / np.linalg.norm(b)
    mx = np.max(np.abs(a - b)) / np.max(np.abs(b))
    assert l2 <= TOL and mx <= TOL, (seed, l2, mx)


def test_noalloc_matches_workspace_entry_twice():
    stream = ob.stream_ptr()
    # two calls in a row, different sizes and inputs, the second smaller so
    # stale contents of the shared array would show up
    for seed, nst, nsrc in [(1, 300, 4000), (2, 97, 611)]:
        compare(seed, nst, nsrc, stream)


def test_noalloc_largest_call_that_fits():
    # 16 station blocks x 127 source blocks x 32 KB + 256 B <= 64 MiB
    compare(4, 512, 4064, ob.stream_ptr())


@pytest.mark.parametrize("nst,nsrc", [
    (512, 4096),     # one 32-source block past the limit: 64 MiB + 256 B
    (1024, 8192),    # 256 MiB
])
def test_noalloc_rejects_too_large(nst, nsrc):
    # the size check comes before any pointer is read, so small buffers do
    J, I, Q, U, V, u, v = case(3, 64, 64)
    vis = torch.zeros(8 * 2016, dtype=torch.float64, device="cuda")
    st = ob.call("oskb_cross_correlate_tc_noalloc_d", 0, nsrc, nst, 0, J,
                 I, Q, U, V, u, v, 0.0, 3e38, 1.0, vis, ob.stream_ptr(),
                 check=False)
    assert st == -5
    assert b"static scratch" in ob.load().oskb_last_error()
    torch.cuda.synchronize()
    assert float(vis.abs().sum()) == 0.0
