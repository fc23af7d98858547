"""Sky tables for the flux-scaling tests.

A sky table is column-major (column k of source s at table[k * capacity + s]),
with the columns of one type adjacent and the types in ascending order, and
a [source][20] count of the columns of each type that hold data for the
source: the layout of the reference's sky model (oskar/sky/private_sky.h,
oskar/sky/src/oskar_sky_sort_columns.c, column types from
oskar/sky/oskar_sky_enum.h:14-35). Sources are given as dicts
{type name: list of values}.
"""
import math

import numpy as np

TYPES = {"I": 3, "Q": 4, "U": 5, "V": 6, "REF_HZ": 7, "SPX": 8, "RM": 9,
         "LIN_SI": 13, "POLA": 14, "POLF": 15, "REF_WAVE": 16, "CURV": 17,
         "LINE_WIDTH": 18, "INC_HZ": 19}
NUM_TYPES = 20
# Column-start arguments in the reference kernel's order
# (oskar/sky/define_sky_scale_flux_with_frequency.h:89-113).
KERNEL_ORDER = ["I", "Q", "U", "V", "REF_HZ", "LIN_SI", "SPX", "RM", "POLF",
                "POLA", "REF_WAVE", "CURV", "LINE_WIDTH", "INC_HZ"]


class SkyTable:
    def __init__(self, sources, dtype, columns=None, capacity=None):
        """columns: {type name: number of columns} (default: the most any
        source uses); capacity: rows per column (default: sources
        rounded up to 256, as the reference allocates)."""
        n = len(sources)
        if columns is None:
            columns = {}
            for src in sources:
                for k, v in src.items():
                    columns[k] = max(columns.get(k, 0), len(v))
        self.capacity = capacity or max(256, -(-(n + 1) // 256) * 256)
        names = sorted(columns, key=lambda k: TYPES[k])
        self.first = {}
        col = 0
        for k in names:
            self.first[k] = col
            col += columns[k]
        self.num_columns = col
        self.num_sources = n
        self.table = np.zeros((col, self.capacity), dtype)
        self.num_valid = np.zeros((max(n, 1), NUM_TYPES), np.int32)
        for s, src in enumerate(sources):
            for k, vals in src.items():
                assert len(vals) <= columns[k]
                for j, v in enumerate(vals):
                    self.table[self.first[k] + j, s] = v
                self.num_valid[s, TYPES[k]] = len(vals)
        self.cols = [self.first.get(k, -1) for k in KERNEL_ORDER]

    def args(self):
        """(capacity, num_columns) and the column starts in kernel order."""
        return self.capacity, self.num_columns, self.cols


def call_scale(lib, real, sky, freq_hz):
    """Runs orc_/ref_sky_scale_flux on the table; returns I, Q, U, V."""
    n = sky.num_sources
    out = [np.zeros(max(n, 1), real) for _ in range(4)]
    lib.call("sky_scale_flux_" + ("d" if real == np.float64 else "f"), real,
             n, sky.capacity, sky.num_columns, float(freq_hz),
             np.ascontiguousarray(sky.table),
             np.ascontiguousarray(sky.num_valid), *sky.cols, *out)
    return [o[:n] for o in out]


def random_sky(n, seed, nan_fraction=0.02):
    """n sources drawn across every spectral and polarisation model the
    scaling supports (power laws, polynomials, curvature, lines, tabulated
    channels, rotation measure with either Q/U or angle/fraction, derived
    Q/U), with a few NaN coefficients."""
    rng = np.random.default_rng(seed)
    out = []
    for s in range(n):
        kind = s % 14
        f0 = float(rng.uniform(50e6, 200e6))
        I = float(rng.uniform(0.1, 10.0))
        src = {"I": [I]}
        if rng.uniform() < 0.5:
            src["Q"] = [I * float(rng.uniform(-0.2, 0.2))]
            src["U"] = [I * float(rng.uniform(-0.2, 0.2))]
        if rng.uniform() < 0.5:
            src["V"] = [I * float(rng.uniform(-0.05, 0.05))]
        if kind == 0:
            pass  # flat: no reference frequency
        elif kind == 1:
            src["REF_HZ"] = [f0]
            src["SPX"] = [float(rng.uniform(-1.0, 0.5))]
        elif kind == 2:
            src["REF_HZ"] = [f0]
            src["SPX"] = list(rng.uniform(-0.8, 0.3, int(rng.integers(2, 4))))
        elif kind == 3:
            src["REF_HZ"] = [f0]
            src["LIN_SI"] = [1.0]
            src["SPX"] = list(rng.uniform(-0.3, 0.3, int(rng.integers(1, 4))))
        elif kind == 4:
            src["REF_HZ"] = [f0]
            src["CURV"] = [float(rng.uniform(-0.3, 0.3))]
            if rng.uniform() < 0.7:
                src["SPX"] = [float(rng.uniform(-1.0, 0.5))]
        elif kind == 5:
            src["REF_HZ"] = [f0]
            src["LINE_WIDTH"] = [float(rng.uniform(50e3, 5e6))]
        elif kind == 6:
            k = int(rng.integers(2, 5))
            src["I"] = list(rng.uniform(0.5, 2.0, k))
            src["REF_HZ"] = list(f0 + np.sort(rng.uniform(0, 3e6, k)))
            src["LINE_WIDTH"] = [float(rng.uniform(100e3, 2e6))]
        elif kind == 7:
            k = int(rng.integers(2, 4))
            src["I"] = list(rng.uniform(0.5, 2.0, k))
            src["REF_HZ"] = [f0]
            src["INC_HZ"] = [float(rng.uniform(0.5e6, 2e6))]
            src["LINE_WIDTH"] = list(rng.uniform(100e3, 2e6, k))
        elif kind == 8:
            k = int(rng.integers(2, 5))
            src["I"] = list(rng.uniform(0.5, 2.0, k))
            src["REF_HZ"] = list(f0 + np.sort(rng.uniform(0, 30e6, k)))
        elif kind == 9:
            k = int(rng.integers(2, 5))
            src["I"] = list(rng.uniform(0.5, 2.0, k))
            src["REF_HZ"] = [f0]
            src["INC_HZ"] = [float(rng.uniform(1e6, 5e6))]
        elif kind == 10:
            src["REF_HZ"] = [f0]
            src["Q"] = [I * 0.1]
            src["U"] = [I * float(rng.uniform(-0.1, 0.1))]
            src["RM"] = [float(rng.uniform(-5, 5))]
            if rng.uniform() < 0.5:
                src["SPX"] = [float(rng.uniform(-1.0, 0.5))]
        elif kind == 11:
            src.pop("Q", None)
            src.pop("U", None)
            src["REF_HZ"] = [f0]
            src["RM"] = [float(rng.uniform(-5, 5))]
            src["POLA"] = [float(rng.uniform(0, math.pi))]
            src["POLF"] = [float(rng.uniform(0, 0.5))]
        elif kind == 12:
            src["REF_HZ"] = [f0]
            src["Q"] = [I * 0.05]
            src["U"] = [I * 0.02]
            src["RM"] = [float(rng.uniform(-5, 5))]
            src["REF_WAVE"] = [float(rng.uniform(1.0, 3.0))]
            src["SPX"] = [float(rng.uniform(-1.0, 0.5))]
        else:
            src.pop("Q", None)
            src["REF_HZ"] = [f0]
            src["POLA"] = [float(rng.uniform(0, math.pi))]
            src["POLF"] = [float(rng.uniform(0, 0.5))]
            src["SPX"] = [float(rng.uniform(-1.0, 0.5))]
        if rng.uniform() < nan_fraction:
            key = [k for k in ("SPX", "RM", "CURV", "V") if k in src]
            if key:
                src[key[0]][0] = float("nan")
        out.append({k: [float(x) for x in v] for k, v in src.items()})
    return out


def mixed_types_sky():
    """The ten sources of the reference's mixed-spectral-types test
    (oskar/sky/test/Test_Sky_scale_flux_with_frequency.cpp:213-247), as
    table entries: flat; a power law; a two-term logarithmic polynomial; a
    three-term linear polynomial; a curved power law; one Gaussian line;
    three lines of one width; three lines of three widths; flux at four
    tabulated frequencies; flux at four regularly spaced frequencies."""
    return [
        {"I": [1.0], "REF_HZ": [0.0]},
        {"I": [1.1], "REF_HZ": [101e6], "SPX": [-0.55]},
        {"I": [1.2], "REF_HZ": [102e6], "SPX": [-0.7, 0.05],
         "LIN_SI": [0.0]},
        {"I": [1.3], "REF_HZ": [103e6], "SPX": [0.08, 0.07, 0.02],
         "LIN_SI": [1.0]},
        {"I": [1.4], "REF_HZ": [104e6], "SPX": [-0.6], "CURV": [0.1]},
        {"I": [1.5], "REF_HZ": [105e6], "LINE_WIDTH": [100e3]},
        {"I": [1.6, 1.7, 1.8], "REF_HZ": [101e6, 102e6, 104e6],
         "LINE_WIDTH": [125e3]},
        {"I": [1.6, 1.7, 1.8], "REF_HZ": [101e6, 102e6, 104e6],
         "LINE_WIDTH": [250e3, 350e3, 500e3]},
        {"I": [1.7, 1.8, 1.9, 1.75],
         "REF_HZ": [101e6, 102.4e6, 103.8e6, 104.1e6]},
        {"I": [1.5, 1.6, 1.7, 1.55], "REF_HZ": [101e6], "INC_HZ": [1e6]},
    ]


def mixed_types_expected(freq_hz):
    """Stokes I the reference's test expects for mixed_types_sky() at
    freq_hz (the closed forms of its assertions)."""
    f = freq_hz
    e = [1.0, 1.1 * (f / 101e6) ** -0.55]
    lr = math.log10(f / 102e6)
    e.append(1.2 * (f / 102e6) ** (-0.7 + 0.05 * lr))
    b = f / 103e6 - 1.0
    e.append(1.3 + 0.08 * b + 0.07 * b * b + 0.02 * b ** 3)
    e.append(1.4 * (f / 104e6) ** -0.6 *
             math.exp(0.1 * math.log(f / 104e6) ** 2))
    x = f - 105e6
    e.append(1.5 * math.exp(-x * x / (2 * 100e3 ** 2)))
    refs, amps = (101e6, 102e6, 104e6), (1.6, 1.7, 1.8)
    e.append(sum(a * math.exp(-(f - r) ** 2 / (2 * 125e3 ** 2))
                 for a, r in zip(amps, refs)))
    e.append(sum(a * math.exp(-(f - r) ** 2 / (2 * w ** 2))
                 for a, r, w in zip(amps, refs, (250e3, 350e3, 500e3))))
    fr = (101e6, 102.4e6, 103.8e6, 104.1e6)
    e.append((1.7, 1.8, 1.9, 1.75)[int(np.argmin([abs(f - r) for r in fr]))])
    fr = [101e6 + j * 1e6 for j in range(4)]
    e.append((1.5, 1.6, 1.7, 1.55)[int(np.argmin([abs(f - r) for r in fr]))])
    return np.array(e)


def spectral_index_sky(n):
    """The reference's spectral-index test sky
    (Test_Sky_scale_flux_with_frequency.cpp:29-88): I, Q, U, V =
    (10, 1, 0.5, 0.1) sin(2 pi i / n) at 10 MHz; even sources logarithmic,
    odd linear; the first half with three coefficients."""
    flux, spx = (10.0, 1.0, 0.5, 0.1), (-0.7, -0.2, 0.1)
    out = []
    for i in range(n):
        w = math.sin(2 * math.pi * i / n)
        src = {"I": [flux[0] * w], "Q": [flux[1] * w], "U": [flux[2] * w],
               "V": [flux[3] * w], "REF_HZ": [10e6],
               "LIN_SI": [0.0 if i % 2 == 0 else 1.0]}
        src["SPX"] = ([spx[0] * w, spx[1], spx[2]] if i < n // 2
                      else [spx[0] * w])
        out.append(src)
    return out


def spectral_index_expected(n, freq_hz):
    """[4][n] values the reference's spectral-index test expects."""
    flux, spx = (10.0, 1.0, 0.5, 0.1), (-0.7, -0.2, 0.1)
    out = np.zeros((4, n))
    for i in range(n):
        w = math.sin(2 * math.pi * i / n)
        r = freq_hz / 10e6
        lr, base = math.log10(r), r - 1.0
        if i < n // 2:
            if i % 2 == 0:
                factor = r ** (spx[0] * w + spx[1] * lr + spx[2] * lr * lr)
            else:
                d = spx[0] * w * base + spx[1] * base ** 2 + spx[2] * base ** 3
                factor = (flux[0] * w + d) / (flux[0] * w) if w else 1.0
        else:
            if i % 2 == 0:
                factor = r ** (spx[0] * w)
            else:
                d = spx[0] * w * base
                factor = (flux[0] * w + d) / (flux[0] * w) if w else 1.0
        for c in range(4):
            out[c, i] = flux[c] * w * factor
    return out
