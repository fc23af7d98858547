"""Beam patterns of aperture-array stations on a sky image: the driver of
the reference's beam-pattern application (oskar/beam_pattern/src/
oskar_beam_pattern_run.c, sim_chunks at :276-500 and write_chunks /
write_pixels at :515-890) over this library's fused kernels.

For every (time, channel) of an observation it forms, on the device:
  - the beam-image pixel grid (oskb_evaluate_image_lmn_grid, the
    application's 'B' grid in the equatorial frame) rotated into the
    station frame at the time's local sidereal time
    (oskb_convert_relative_directions_to_enu_directions);
  - the station beams (Jones E) of the active stations in one launch
    (oskb_station_beam_aa_*), pointed at and normalised to the beam
    direction as oskar_station_beam does;
  - the auto power J B J^H of each station and the cross power averaged
    over station pairs (oskb_evaluate_auto_power_* / _cross_power_*), for
    an unpolarised unit source and for the test source's Stokes
    parameters, as the application's two power products.
Results come back as numpy arrays; the application's image products
(amplitude, phase, IXR, Stokes parameters of the power terms, time and
channel averages) are the functions below, and write_fits writes an image
cube with the application's axes (RA---SIN, DEC--SIN, FREQ, UTC).
"""
import math

import numpy as np

from . import _lib


# --- time: the reference's fast GAST (convert/src/oskar_convert_mjd_to_gmst.c
# and oskar_equation_of_equinoxes_fast.c, restated)
def mjd_to_gmst(mjd):
    d = mjd - 51544.5
    t = d / 36525.0
    gmst = math.fmod(mjd, 1.0) * 2.0 * math.pi + (
        24110.54841 + (8640184.812866 + (0.093104 - 6.2e-6 * t) * t) * t) \
        * 7.2722052166430399038487e-5
    x = math.fmod(gmst, 2.0 * math.pi)
    return x if x >= 0.0 else x + 2.0 * math.pi


def equation_of_equinoxes_fast(mjd):
    d = mjd - 51544.5
    deg = 0.0174532925199432957692
    omega = (125.04 - 0.052954 * d) * deg
    L = (280.47 + 0.98565 * d) * deg
    delta_psi = -0.000319 * math.sin(omega) - 0.000024 * math.sin(2.0 * L)
    epsilon = (23.4393 - 0.0000004 * d) * deg
    return delta_psi * math.cos(epsilon) * 0.261799387799149436539


def mjd_to_gast(mjd):
    return mjd_to_gmst(mjd) + equation_of_equinoxes_fast(mjd)


class BeamPattern:
    """Stations: el_x, el_y, el_z [station][element] (ENU metres, equal
    element counts), orientation_x_deg / orientation_y_deg [station] (the
    reference's element Euler angles, 0 by default: X dipoles then lie
    north-south, Y dipoles east-west), one dipole length; the station
    beams point at and the image is centred on (beam_ra_deg,
    beam_dec_deg). The array is three-dimensional when any el_z is
    non-zero (the reference's oskar_station_array_is_3d)."""

    def __init__(self, lon_deg, lat_deg, el_x, el_y, el_z, beam_ra_deg,
                 beam_dec_deg, orientation_x_deg=0.0, orientation_y_deg=0.0,
                 dipole_length_m=1.5, normalise_element=1,
                 normalise_array=1, normalise_final=1, precision="double"):
        import torch
        self.torch = torch
        self.real = np.float64 if precision == "double" else np.float32
        self.tdtype = torch.float64 if precision == "double" else \
            torch.float32
        self.sfx = "d" if precision == "double" else "f"
        el_x = np.atleast_2d(np.asarray(el_x, np.float64))
        el_y = np.atleast_2d(np.asarray(el_y, np.float64))
        el_z = np.atleast_2d(np.asarray(el_z, np.float64))
        self.num_stations, self.num_elements = el_x.shape
        ns = self.num_stations
        self.is_3d = int(bool(np.any(el_z != 0.0)))
        self.lon = math.radians(lon_deg)
        self.lat = math.radians(lat_deg)
        self.ra0 = math.radians(beam_ra_deg)
        self.dec0 = math.radians(beam_dec_deg)
        ox = np.broadcast_to(np.radians(orientation_x_deg), (ns,))
        oy = np.broadcast_to(np.radians(orientation_y_deg), (ns,))
        self._el = [self._dev(a, self.real) for a in (el_x, el_y, el_z)]
        self._orient = [self._dev(a, np.float64) for a in (ox, oy)]
        self.dipole_length_m = float(dipole_length_m)
        self.flags = (int(normalise_element), int(normalise_array),
                      int(normalise_final))
        self.station_ids = list(range(ns))
        self.stokes = (1.0, 0.0, 0.0, 0.0)
        self.set_image(128, 128, 2.0, 2.0)
        self.set_observation(51544.5, 1.0, 1, 100e6, 0.0, 1)

    def _dev(self, a, dtype):
        return self.torch.from_numpy(
            np.ascontiguousarray(a, dtype=dtype)).cuda()

    def set_image(self, width, height, fov_lon_deg, fov_lat_deg):
        self.width, self.height = int(width), int(height)
        self.fov = (float(fov_lon_deg), float(fov_lat_deg))

    def set_observation(self, mjd_start, inc_sec, num_times, freq_start_hz,
                        freq_inc_hz, num_channels):
        self.mjd_start, self.inc_sec = float(mjd_start), float(inc_sec)
        self.num_times = int(num_times)
        self.freq_start_hz = float(freq_start_hz)
        self.freq_inc_hz = float(freq_inc_hz)
        self.num_channels = int(num_channels)

    def set_station_ids(self, ids):
        ids = [int(i) for i in ids]
        if not ids or min(ids) < 0 or max(ids) >= self.num_stations:
            raise ValueError("station ids out of range")
        self.station_ids = ids

    def set_test_source(self, I, Q=0.0, U=0.0, V=0.0):
        self.stokes = (float(I), float(Q), float(U), float(V))

    def pixel_grid(self):
        """(l, m, n) of the image pixels, m slowest (host, FP64; NaN off
        the sphere), the application's centred beam-image grid."""
        n = self.width * self.height
        l, m, nn = (np.empty(n) for _ in range(3))
        st = _lib.call("oskb_evaluate_image_lmn_grid", self.width,
                       self.height, math.radians(self.fov[0]),
                       math.radians(self.fov[1]), 1, l, m, nn, check=False)
        if st:
            raise ValueError("image grid: status %d" % st)
        return l, m, nn

    def time_mjd(self, t):
        """Mid-dump time of dump t, as the application takes it."""
        return self.mjd_start + self.inc_sec / 86400.0 * (t + 0.5)

    def run(self, jones=True, auto_power=True, cross_power=True):
        """Returns a dict of complex arrays: "jones" [time][channel]
        [station][pixel][2][2], "auto_power" [stokes_in][time][channel]
        [station][pixel][2][2] and "cross_power" [stokes_in][time][channel]
        [pixel][2][2], stokes_in 0 an unpolarised unit source and 1 the test
        source; stations in set_station_ids order, pixels m-major."""
        torch, s = self.torch, self.sfx
        stream = _lib.stream_ptr()
        ids = self.station_ids
        na = len(ids)
        idx = torch.as_tensor(ids, device="cuda")
        el = [a.index_select(0, idx).contiguous() for a in self._el]
        orient = [a.index_select(0, idx).contiguous() for a in self._orient]
        l, m, n = self.pixel_grid()
        npix = l.size
        dl, dm, dn = (self._dev(a, self.real) for a in (l, m, n))
        x, y, z = (torch.empty(npix, dtype=self.tdtype, device="cuda")
                   for _ in range(3))
        one = [self._dev(np.array([v]), self.real) for v in (0.0, 0.0, 1.0)]
        bxyz = [torch.empty(1, dtype=self.tdtype, device="cuda")
                for _ in range(3)]
        beam = torch.empty((na, npix, 8), dtype=self.tdtype, device="cuda")
        ap = torch.empty((2, na, npix, 8), dtype=self.tdtype, device="cuda")
        cp = torch.empty((2, npix, 8), dtype=self.tdtype, device="cuda")
        nt, nc = self.num_times, self.num_channels
        cplx = np.complex128 if s == "d" else np.complex64
        out = {}
        if jones:
            out["jones"] = np.empty((nt, nc, na, npix, 2, 2), cplx)
        if auto_power:
            out["auto_power"] = np.empty((2, nt, nc, na, npix, 2, 2), cplx)
        if cross_power:
            out["cross_power"] = np.empty((2, nt, nc, npix, 2, 2), cplx)
        sources = ((1.0, 0.0, 0.0, 0.0), self.stokes)
        for t in range(nt):
            lst = mjd_to_gast(self.time_mjd(t)) + self.lon
            ha0 = lst - self.ra0
            _lib.call("oskb_convert_relative_directions_to_enu_directions_"
                      + s, npix, dl, dm, dn, ha0, self.dec0, self.lat,
                      x, y, z, stream)
            _lib.call("oskb_convert_relative_directions_to_enu_directions_"
                      + s, 1, *one, ha0, self.dec0, self.lat, *bxyz, stream)
            b = torch.cat(bxyz).to(torch.float64).repeat(na, 1).contiguous()
            for c in range(nc):
                f = self.freq_start_hz + c * self.freq_inc_hz
                _lib.call("oskb_station_beam_aa_" + s, na,
                          self.num_elements, *el, None, None, None, None,
                          *orient, self.dipole_length_m, *self.flags, 0,
                          self.is_3d, f, b, b, npix, x, y, z, 0, beam,
                          stream)
                for k, src in enumerate(sources):
                    if auto_power:
                        _lib.call("oskb_evaluate_auto_power_" + s, 1,
                                  na * npix, 0, beam, *src, 0, ap[k],
                                  stream)
                    if cross_power:
                        _lib.call("oskb_evaluate_cross_power_" + s, 1, npix,
                                  na, beam, *src, 0, cp[k], stream)
                if jones:
                    out["jones"][t, c] = _to_complex(beam)
                if auto_power:
                    out["auto_power"][:, t, c] = _to_complex(ap)
                if cross_power:
                    out["cross_power"][:, t, c] = _to_complex(cp)
        return out


def _to_complex(t):
    a = t.cpu().numpy()
    c = a[..., 0::2] + 1j * a[..., 1::2]
    return c.reshape(a.shape[:-1] + (2, 2))


# --- image products (write_pixels of oskar_beam_pattern_run.c:686-890)
def amplitude(z):
    return np.abs(z)


def phase(z):
    return np.angle(z)


def linear_to_stokes(p, index):
    """Stokes I, Q, U or V (index 0..3) of 2x2 power matrices p[..., 2, 2]
    (the application's LINEAR_TO_STOKES: I = (XX + YY)/2,
    Q = (XX - YY)/2, U = (XY + YX)/2, V = -i (XY - YX)/2)."""
    a, b, c, d = p[..., 0, 0], p[..., 0, 1], p[..., 1, 0], p[..., 1, 1]
    if index == 0:
        return 0.5 * (a + d)
    if index == 1:
        return 0.5 * (a - d)
    if index == 2:
        return 0.5 * (b + c)
    if index == 3:
        return -0.5j * (b - c)
    raise ValueError("stokes index 0..3")


def ixr(jones, limit=1e8):
    """Intrinsic cross-polarisation ratio ((cond + 1) / (cond - 1))^2 of
    2x2 Jones matrices, cond their 2-norm condition number, capped at
    limit (1e8 in FP64, as the application; oskar/math/
    private_cond2_2x2.h)."""
    p = np.einsum("...ij,...kj->...ik", jones, np.conj(jones))
    s = p[..., 0, 0].real + p[..., 1, 1].real
    t1 = (p[..., 0, 0].real - p[..., 1, 1].real) ** 2
    t2 = 4.0 * (p[..., 0, 1].real ** 2 + p[..., 0, 1].imag ** 2)
    diff = np.sqrt(t1 + t2)
    a = np.sqrt(0.5 * (s + diff))
    b = np.sqrt(0.5 * (s - diff))
    with np.errstate(divide="ignore", invalid="ignore"):
        cond = np.where(a > b, a / b, b / a)
        r = ((cond + 1.0) / (cond - 1.0)) ** 2
    return np.minimum(r, limit)


def average(data, axis):
    """Mean over an axis (the application's time or channel averages)."""
    return np.mean(data, axis=axis)


# --- FITS output
def _card(key, value=None, comment=None):
    if value is None:
        s = "%-8s" % key
    elif isinstance(value, str):
        s = "%-8s= '%-8s'" % (key, value)
    elif isinstance(value, bool):
        s = "%-8s= %20s" % (key, "T" if value else "F")
    elif isinstance(value, int):
        s = "%-8s= %20d" % (key, value)
    else:
        s = "%-8s= %20s" % (key, ("%.15G" % value).replace("E", "E"))
    if comment:
        s += " / " + comment
    return s[:80].ljust(80)


def write_fits(path, cube, beam_pattern, bitpix=-64):
    """Writes images [time][channel][height][width] (real) as a FITS
    primary image with the application's axes: RA---SIN and DEC--SIN about
    the beam direction (cell size asin(2 sin(fov / 2) / n), RA decreasing
    with the pixel index, reference pixel (n + 1) / 2), FREQ and UTC
    (oskar_beam_pattern_check_init.c:440-489)."""
    bp = beam_pattern
    cube = np.asarray(cube, np.float64)
    nt, nc, h, w = cube.shape
    r2d = 180.0 / math.pi
    dl = math.asin(2.0 * math.sin(0.5 * math.radians(bp.fov[0])) / w) * r2d
    dm = math.asin(2.0 * math.sin(0.5 * math.radians(bp.fov[1])) / h) * r2d
    cards = [
        _card("SIMPLE", True), _card("BITPIX", bitpix), _card("NAXIS", 4),
        _card("NAXIS1", w), _card("NAXIS2", h), _card("NAXIS3", nc),
        _card("NAXIS4", nt), _card("EXTEND", True),
        _card("CTYPE1", "RA---SIN", "Right Ascension"),
        _card("CRVAL1", math.degrees(bp.ra0)), _card("CDELT1", -dl),
        _card("CRPIX1", (w + 1) / 2.0), _card("CROTA1", 0.0),
        _card("CTYPE2", "DEC--SIN", "Declination"),
        _card("CRVAL2", math.degrees(bp.dec0)), _card("CDELT2", dm),
        _card("CRPIX2", (h + 1) / 2.0), _card("CROTA2", 0.0),
        _card("CTYPE3", "FREQ", "Frequency"),
        _card("CRVAL3", bp.freq_start_hz), _card("CDELT3", bp.freq_inc_hz),
        _card("CRPIX3", 1.0), _card("CROTA3", 0.0),
        _card("CTYPE4", "UTC", "Time"),
        _card("CRVAL4", bp.mjd_start * 86400.0), _card("CDELT4", bp.inc_sec),
        _card("CRPIX4", 1.0), _card("CROTA4", 0.0),
        _card("TIMESYS", "UTC"), _card("TIMEUNIT", "s", "Time axis units"),
        _card("MJD-OBS", bp.mjd_start, "Start time"),
        _card("OBSRA", math.degrees(bp.ra0), "RA"),
        _card("OBSDEC", math.degrees(bp.dec0), "DEC"),
        _card("END")]
    header = "".join(cards)
    header += " " * ((-len(header)) % 2880)
    fmt = ">f8" if bitpix == -64 else ">f4"
    data = np.ascontiguousarray(cube).astype(fmt).tobytes()
    data += b"\0" * ((-len(data)) % 2880)
    with open(path, "wb") as f:
        f.write(header.encode("ascii"))
        f.write(data)


def read_fits(path):
    """Reads back a FITS primary image written by write_fits: (header dict,
    data [NAXIS4][NAXIS3][NAXIS2][NAXIS1])."""
    with open(path, "rb") as f:
        raw = f.read()
    hdr, pos = {}, 0
    while True:
        card = raw[pos:pos + 80].decode("ascii")
        pos += 80
        key = card[:8].strip()
        if key == "END":
            break
        if card[8:10] == "= ":
            v = card[10:].split("/")[0].strip()
            if v.startswith("'"):
                v = v.strip("'").strip()
            elif v in ("T", "F"):
                v = v == "T"
            else:
                v = float(v) if any(ch in v for ch in ".EeNn") else int(v)
            hdr[key] = v
    pos += (-pos) % 2880
    shape = tuple(int(hdr["NAXIS%d" % i])
                  for i in range(int(hdr["NAXIS"]), 0, -1))
    fmt = ">f8" if hdr["BITPIX"] == -64 else ">f4"
    n = int(np.prod(shape))
    data = np.frombuffer(raw, fmt, n, pos).reshape(shape)
    return hdr, data.astype(np.float64)
