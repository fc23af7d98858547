"""Host driver of the learned station-beam surrogate.

One sine-activated perceptron per station type learns the normalised array
factor A(kappa) of that type's planar dipole layout, kappa = k (d - b) in
the station frame (rad/m): the array factor of a station phased to b
depends on direction and frequency only through kappa, and stations of one
type differ only by a rotation, so one network serves every station of the
type. Training samples come from the exact sum (oskb_array_factor_samples_f)
and training runs on the GPU through the library's own kernels
(oskb_mlp_train). Evaluation (oskb_station_beam_surrogate_f) takes the exact
sum inside the main lobe, the network elsewhere, audits a sample of the
network values against the exact sum and falls back to the exact sum for
the whole call when the audit exceeds its bound.
"""
import ctypes
import math
import time

import numpy as np

from . import _lib

C0 = 299792458.0


def first_null_kappa(diameter_m):
    """|kappa| of the first null of a filled circular aperture of this
    diameter (1.22 lambda / D in direction cosine, times k = 2 pi / lambda):
    independent of frequency."""
    return 2.0 * math.pi * 1.22 / diameter_m


class BeamSurrogate:
    """Networks for num_types layouts (each an (x, y) pair of arrays in
    metres, all with the same number of elements)."""

    def __init__(self, layouts, max_frequency_hz, hidden=(128, 128, 128, 128),
                 omega0=30.0, diameter_m=38.0, main_lobe_factor=1.2, seed=1):
        import torch
        self.torch = torch
        self.lib = _lib.load()
        self.num_types = len(layouts)
        self.num_el = len(layouts[0][0])
        self.dims = [2] + list(hidden) + [2]
        self.omega0 = omega0
        # |d - b| <= 2 for directions and pointings on the sky
        self.kappa_scale = 2.0 * 2.0 * math.pi * max_frequency_hz / C0
        self.kappa_main = main_lobe_factor * first_null_kappa(diameter_m)
        lx = np.concatenate([np.asarray(l[0], np.float32) for l in layouts])
        ly = np.concatenate([np.asarray(l[1], np.float32) for l in layouts])
        self.layout_x = torch.from_numpy(lx).cuda()
        self.layout_y = torch.from_numpy(ly).cuda()
        self.nets = []
        for t in range(self.num_types):
            st = ctypes.c_int(0)
            d = (ctypes.c_int * len(self.dims))(*self.dims)
            p = self.lib.oskb_mlp_create(len(self.dims) - 1,
                                         ctypes.addressof(d), omega0,
                                         seed + 7919 * t,
                                         ctypes.addressof(st))
            if st.value or not p:
                raise RuntimeError("oskb_mlp_create failed: %d" % st.value)
            self.nets.append(p)
        self.net_array = (ctypes.c_void_p * self.num_types)(*self.nets)

    def samples(self, type_index, count, seed):
        """Training samples for one type: kappa uniform over the disc
        |kappa| <= kappa_scale, outside 0.9 kappa_main; features
        kappa / kappa_scale, targets A(kappa) from the exact sum."""
        torch = self.torch
        rng = np.random.default_rng(seed)
        r = self.kappa_scale * np.sqrt(rng.uniform(
            (0.9 * self.kappa_main / self.kappa_scale) ** 2, 1.0, count))
        th = rng.uniform(0, 2 * math.pi, count)
        kx = torch.from_numpy((r * np.cos(th)).astype(np.float32)).cuda()
        ky = torch.from_numpy((r * np.sin(th)).astype(np.float32)).cuda()
        af = torch.empty((count, 2), dtype=torch.float32, device="cuda")
        o = type_index * self.num_el
        _lib.call("oskb_array_factor_samples_f", self.num_el,
                  self.layout_x[o:], self.layout_y[o:], count, kx, ky, af,
                  _lib.stream_ptr())
        x = torch.stack([kx, ky], 1) / self.kappa_scale
        return x.contiguous(), af

    def train(self, num_samples=1_000_000, steps=20000, batch=4096,
              lr=1e-4, report_every=1000, seed=11):
        """Trains every type's network; returns per type the loss history
        and the seconds taken (samples included)."""
        torch = self.torch
        out = []
        for t, net in enumerate(self.nets):
            t0 = time.perf_counter()
            x, y = self.samples(t, num_samples, seed + t)
            hist = np.zeros((steps - 1) // report_every + 2, np.float32)
            _lib.call("oskb_mlp_train", net, num_samples, x, y, batch,
                      steps, lr, seed + 101 * t, report_every, hist,
                      _lib.stream_ptr())
            torch.cuda.synchronize()
            out.append({"loss": hist, "seconds": time.perf_counter() - t0})
            del x, y
        return out

    def beam(self, station_type, rotation, beam_enu, x, y, z, frequency_hz,
             dipole_length_m=1.5, normalise_element=0, audit_stride=100,
             audit_bound=1e-4, out=None):
        """Beam [station][direction][2x2] (FP32, device) and the audit
        record. station_type: host int array; rotation, beam_enu: device
        FP64; x, y, z: device FP32 [station][direction]."""
        torch = self.torch
        st = np.ascontiguousarray(station_type, np.int32)
        ns, nd = st.size, x.shape[-1]
        if out is None:
            out = torch.empty((ns, nd, 8), dtype=torch.float32, device="cuda")
        audit = np.zeros(5)
        _lib.call("oskb_station_beam_surrogate_f", ns, self.num_types,
                  self.num_el, st, rotation, self.layout_x, self.layout_y,
                  ctypes.addressof(self.net_array), dipole_length_m,
                  normalise_element, frequency_hz, beam_enu, nd, x, y, z,
                  self.kappa_main, self.kappa_scale, audit_stride,
                  audit_bound, out, audit, _lib.stream_ptr())
        return out, {"max_err": audit[0], "rms_err": audit[1],
                     "audited": int(audit[2]), "fallback": bool(audit[3]),
                     "network_evaluations": int(audit[4])}

    def free(self):
        for p in self.nets:
            self.lib.oskb_mlp_free(p)
        self.nets = []

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
