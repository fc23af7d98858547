"""The learned station-beam surrogate on the GPU: the perceptron kernels
against the FP64 numpy oracle (forward, backward), training, the exact
array-factor samples, and the surrogate beam against the exact beam kernel,
its audit and its fallback."""
import ctypes
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(),
                                 reason="needs a CUDA device")]

import oskar_b200 as ob  # noqa: E402
import mlp_oracle as mo  # noqa: E402

C0 = 299792458.0


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


class Net:
    def __init__(self, dims, omega0=30.0, seed=1):
        self.lib = ob.load()
        self.dims, self.omega0 = list(dims), omega0
        st = ctypes.c_int(0)
        d = (ctypes.c_int * len(dims))(*dims)
        self.ptr = self.lib.oskb_mlp_create(len(dims) - 1,
                                            ctypes.addressof(d), omega0,
                                            seed, ctypes.addressof(st))
        assert st.value == 0 and self.ptr
        self.n = self.lib.oskb_mlp_num_params(self.ptr)

    def get(self, which):
        h = np.zeros(self.n, np.float32)
        assert ob.call("oskb_mlp_copy_to_host", self.ptr, which, h) == 0
        return h

    def set(self, params):
        p = np.ascontiguousarray(params, np.float32)
        assert ob.call("oskb_mlp_set_params", self.ptr, p) == 0

    def free(self):
        self.lib.oskb_mlp_free(self.ptr)


@pytest.mark.parametrize("dims", [[2, 16, 9, 2], [2, 128, 128, 128, 128, 2],
                                  [4, 70, 130, 8]])
def test_mlp_forward_backward_vs_oracle(dims):
    """Forward outputs and backpropagated gradients of the CUDA kernels
    against the FP64 oracle on the same parameters and batch (relative to
    the largest value: 1e-5 forward, 1e-4 gradients, FP32 kernels)."""
    net = Net(dims, omega0=30.0, seed=3)
    try:
        rng = np.random.default_rng(4)
        B = 333
        x = rng.uniform(-1, 1, (B, dims[0])).astype(np.float32)
        t = rng.normal(0, 0.1, (B, dims[-1])).astype(np.float32)
        p = net.get(0).astype(np.float64)
        y_ref, cache = mo.forward(p, dims, 30.0, x.astype(np.float64))
        loss_ref, dy_ref = mo.mse(y_ref, t.astype(np.float64))
        g_ref = mo.backward(p, dims, 30.0, cache, dy_ref)
        xd, td = dev(x), dev(t)
        y = torch.zeros((B, dims[-1]), dtype=torch.float32, device="cuda")
        ob.call("oskb_mlp_forward", net.ptr, B, xd, y, ob.stream_ptr())
        loss = torch.zeros(1, dtype=torch.float32, device="cuda")
        dy = torch.zeros_like(y)
        ob.call("oskb_mlp_mse", B * dims[-1], y, td, dy, loss,
                ob.stream_ptr())
        ob.call("oskb_mlp_backward", net.ptr, B, dy, ob.stream_ptr())
        torch.cuda.synchronize()
        yg = y.cpu().numpy().astype(np.float64)
        assert np.max(np.abs(yg - y_ref)) <= 1e-5 * np.max(np.abs(y_ref))
        assert abs(loss.item() - loss_ref) <= 1e-5 * loss_ref
        g = net.get(1).astype(np.float64)
        assert np.max(np.abs(g - g_ref)) <= 1e-4 * np.max(np.abs(g_ref))
    finally:
        net.free()


def test_mlp_training_fits_a_wave():
    """Adam on the GPU fits sin(5x) cos(3y) to a small error."""
    net = Net([2, 64, 64, 1], omega0=10.0, seed=5)
    try:
        rng = np.random.default_rng(6)
        x = rng.uniform(-1, 1, (20000, 2)).astype(np.float32)
        t = (np.sin(5 * x[:, :1]) * np.cos(3 * x[:, 1:])).astype(np.float32)
        hist = np.zeros(2000 // 100 + 2, np.float32)
        ob.call("oskb_mlp_train", net.ptr, 20000, dev(x), dev(t), 1024,
                2000, 1e-3, 7, 100, hist, ob.stream_ptr())
        assert hist[-1] < 1e-3 * hist[0] and hist[-1] < 1e-4
    finally:
        net.free()


def layout(rng, num_el, radius=19.0):
    r = radius * np.sqrt(rng.uniform(0, 1, num_el))
    th = rng.uniform(0, 2 * math.pi, num_el)
    return r * np.cos(th), r * np.sin(th)


def test_array_factor_samples_vs_numpy():
    rng = np.random.default_rng(8)
    ex, ey = layout(rng, 256)
    kx, ky = (rng.uniform(-4, 4, 5000) for _ in range(2))
    af = torch.zeros((5000, 2), dtype=torch.float32, device="cuda")
    ob.call("oskb_array_factor_samples_f", 256, dev(ex.astype(np.float32)),
            dev(ey.astype(np.float32)), 5000, dev(kx.astype(np.float32)),
            dev(ky.astype(np.float32)), af, ob.stream_ptr())
    torch.cuda.synchronize()
    exf, eyf = ex.astype(np.float32).astype(np.float64), \
        ey.astype(np.float32).astype(np.float64)
    kxf, kyf = kx.astype(np.float32).astype(np.float64), \
        ky.astype(np.float32).astype(np.float64)
    ref = np.exp(1j * (np.outer(kxf, exf) + np.outer(kyf, eyf))).mean(1)
    got = af.cpu().numpy()
    assert np.max(np.abs(got[:, 0] + 1j * got[:, 1] - ref)) <= 1e-6


def surrogate_case(num_el=64, num_st=6, num_dir=4000, steps=3000, seed=9):
    from oskar_b200.surrogate import BeamSurrogate
    rng = np.random.default_rng(seed)
    layouts = [layout(rng, num_el) for _ in range(3)]
    freq = 100e6
    sur = BeamSurrogate(layouts, freq, seed=seed)
    sur.train(num_samples=200_000, steps=steps, batch=4096, lr=1e-4,
              report_every=500, seed=seed)
    types = np.arange(num_st) % 3
    rot = rng.uniform(0, 2 * math.pi, num_st)
    az = rng.uniform(0, 2 * math.pi, num_dir)
    el = np.arcsin(rng.uniform(-0.1, 1, num_dir))
    d = np.stack([np.cos(el) * np.sin(az), np.cos(el) * np.cos(az),
                  np.sin(el)])
    # pointing near the zenith per station, directions shared
    b = np.zeros((num_st, 3))
    b[:, 0] = rng.uniform(-0.2, 0.2, num_st)
    b[:, 1] = rng.uniform(-0.2, 0.2, num_st)
    b[:, 2] = np.sqrt(1 - b[:, 0] ** 2 - b[:, 1] ** 2)
    # a few directions inside each main lobe
    d[:, :num_st] = b.T
    dirs = [np.ascontiguousarray(np.tile(d[i], (num_st, 1)), np.float32)
            for i in range(3)]
    return dict(sur=sur, layouts=layouts, freq=freq, types=types, rot=rot,
                b=b, dirs=dirs, num_el=num_el)


def exact_beam(c):
    ns, nd = c["b"].shape[0], c["dirs"][0].shape[1]
    ex = np.zeros((ns, c["num_el"]), np.float32)
    ey = np.zeros_like(ex)
    for s in range(ns):
        lx, ly = c["layouts"][c["types"][s]]
        co, si = math.cos(c["rot"][s]), math.sin(c["rot"][s])
        ex[s] = co * lx - si * ly
        ey[s] = si * lx + co * ly
    out = torch.zeros((ns, nd, 8), dtype=torch.float32, device="cuda")
    ez = dev(np.zeros_like(ex))
    ob.call("oskb_station_beam_aa_f", ns, c["num_el"], dev(ex), dev(ey), ez,
            None, None, None, None, dev(c["rot"]), dev(c["rot"]), 1.5, 0, 1,
            1, 0, 0, c["freq"], dev(c["b"]), dev(c["b"]), nd,
            *[dev(a) for a in c["dirs"]], 1, out, ob.stream_ptr())
    torch.cuda.synchronize()
    return out.cpu().numpy()


def surrogate_beam(c, bound, stride=100):
    out, audit = c["sur"].beam(c["types"], dev(c["rot"]), dev(c["b"]),
                               *[dev(a) for a in c["dirs"]], c["freq"],
                               audit_stride=stride, audit_bound=bound)
    torch.cuda.synchronize()
    return out.cpu().numpy(), audit


def test_surrogate_beam_audit_fallback_and_gain():
    c = surrogate_case()
    try:
        ref = exact_beam(c)
        # the audit passes with a loose bound: network values are used
        got, audit = surrogate_beam(c, bound=1.0)
        assert not audit["fallback"] and audit["audited"] > 0
        assert audit["network_evaluations"] > 0.5 * ref.shape[0] * \
            ref.shape[1]
        err = np.abs(got - ref).reshape(ref.shape[0], -1, 8).max(axis=2)
        # main-lobe directions (the pointings) are exact
        for s in range(ref.shape[0]):
            assert err[s, s] <= 1e-5
        # gain over the method without the network (no sidelobes at all:
        # A = 0 outside the main lobe): the trained network's rms beam
        # error is far smaller
        k = 2 * math.pi * c["freq"] / C0
        dx, dy, dz = c["dirs"]
        kappa = k * np.hypot(dx - c["b"][:, :1], dy - c["b"][:, 1:2])
        sidelobe = (kappa >= c["sur"].kappa_main) & (dz >= 0)
        base = np.sqrt(np.mean(ref[sidelobe] ** 2))
        trained = np.sqrt(np.mean((got - ref)[sidelobe] ** 2))
        assert trained < 0.1 * base, (trained, base)
        # the audit's largest error bounds the block's rms beam error
        assert 0 < audit["rms_err"] <= audit["max_err"]
        assert trained <= 3 * audit["max_err"]
        # a bound the network cannot meet: every value falls back to the
        # exact sum, so the block equals the exact beam
        got2, audit2 = surrogate_beam(c, bound=1e-9)
        assert audit2["fallback"]
        assert np.max(np.abs(got2 - ref)) <= 1e-5
    finally:
        c["sur"].free()
