"""Hierarchical aperture-array stations (two levels and deeper) on the GPU
against the oracle composed the way the reference recurses
(oskar_evaluate_station_beam_aperture_array.c:242-287): every child
station's beam by the single-level chain at the leaves, then at each level
above the parent's element weights and weighted DFT over its children with
the child beams as data. Each oracle piece is pinned against the reference's
own kernels (tests/test_oracle_pin.py). Tolerances: FP64 1e-12, FP32 2e-5 of
the largest beam value (max and L2)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(),
                                 reason="needs a CUDA device")]

import oskar_b200 as ob  # noqa: E402
from beam_cases import enu_dirs  # noqa: E402
from oracle_lib import oracle, suffix  # noqa: E402

TOL = {np.float64: 1e-12, np.float32: 2e-5}
C0 = 299792458.0


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def rel(got, ref):
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    return max(np.max(np.abs(got - ref)) / np.max(np.abs(ref)),
               np.linalg.norm(got - ref) / np.linalg.norm(ref))


def station(real, seed, num_types=2, num_el=16, num_tiles=24, is_3d=1,
            num_dir=700):
    """Tile layouts (4 x 4-ish dipole grids, jittered), tile positions in a
    40 m station, tile types, pointing and directions."""
    rng = np.random.default_rng(seed)
    g = np.arange(4) * 1.25 - 1.875
    gx, gy = np.meshgrid(g, g)
    layouts = []
    for t in range(num_types):
        x = gx.ravel()[:num_el] + rng.normal(0, 0.05, num_el)
        y = gy.ravel()[:num_el] + rng.normal(0, 0.05, num_el)
        z = rng.uniform(-0.1, 0.1, num_el) if is_3d else np.zeros(num_el)
        layouts.append((x, y, z))
    r = 20.0 * np.sqrt(rng.uniform(0, 1, num_tiles))
    th = rng.uniform(0, 2 * np.pi, num_tiles)
    tiles = (r * np.cos(th), r * np.sin(th),
             rng.uniform(-0.3, 0.3, num_tiles) if is_3d else
             np.zeros(num_tiles))
    types = rng.integers(0, num_types, num_tiles).astype(np.int32)
    ox = rng.uniform(0, 0.3, num_types)
    oy = ox + np.pi / 2
    b = np.array([0.15, -0.25, 0.0])
    b[2] = np.sqrt(1 - b[0] ** 2 - b[1] ** 2)
    dirs = enu_dirs(rng, num_dir, real)
    cast = lambda a: np.ascontiguousarray(a, dtype=real)
    return dict(layouts=[tuple(map(cast, l)) for l in layouts],
                tiles=tuple(map(cast, tiles)), types=types, ox=ox, oy=oy,
                b=b, dirs=dirs, freq=150e6, L=1.4, is_3d=is_3d)


def oracle_two_level(c, real, flags, identical):
    norm_el, norm_tile, norm_st, swap = flags
    s = suffix(real)
    nd = len(c["dirs"][0])
    ntypes = 1 if identical else len(c["layouts"])
    beams = []
    for i in range(ntypes):
        x, y, z = c["layouts"][i]
        out = np.zeros(8 * nd, real)
        oracle().call("station_beam_aa_" + s, np.float64, len(x), x, y, z,
                      None, None, None, np.zeros(len(x), real),
                      float(c["ox"][i]), float(c["oy"][i]), c["L"], norm_el,
                      norm_tile, 0, swap, c["is_3d"], c["freq"], *c["b"],
                      *c["b"], nd, *c["dirs"], out)
        beams.append(out)
    tx, ty, tz = c["tiles"]
    nt = len(tx)
    k = real(2 * np.pi * c["freq"] / C0)
    w = np.zeros(2 * nt, real)
    b = c["b"]
    oracle().call("element_weights_dft_" + s, real, nt, tx, ty, tz,
                  np.zeros(nt, real), k, real(b[0]), real(b[1]),
                  real(b[2] if c["is_3d"] else 0.0), w)
    if identical:
        # the reference copies the first child's beam to every child and
        # indexes the data by element (data_idx NULL)
        data = np.concatenate([beams[0]] * nt)
        idx = None
    else:
        data = np.concatenate(beams)
        idx = c["types"]
    out = np.zeros(8 * nd, real)
    oracle().call("dftw_" + s, real, 1, c["is_3d"], nt, k, w, tx, ty, tz, 0,
                  nd, *c["dirs"], idx, data, 1, 1, 0, out,
                  real(1.0 / nt) if norm_st else real(1.0))
    return out


def gpu_two_level(c, real, flags, identical):
    norm_el, norm_tile, norm_st, swap = flags
    s = suffix(real)
    ntypes = 1 if identical else len(c["layouts"])
    lay = c["layouts"][:ntypes]
    el = [dev(np.concatenate([l[i] for l in lay])) for i in range(3)]
    nd = len(c["dirs"][0])
    nt = len(c["tiles"][0])
    ws_bytes = ob.call("oskb_station_beam_two_level_workspace_bytes",
                       8 if real == np.float64 else 4, ntypes, nt, nd,
                       check=False)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    beam = torch.zeros(nd * 8, dtype=torch.float64 if real == np.float64
                       else torch.float32, device="cuda")
    ob.call("oskb_station_beam_two_level_" + s, ntypes, len(lay[0][0]), *el,
            dev(c["ox"][:ntypes]), dev(c["oy"][:ntypes]), c["L"], norm_el,
            norm_tile, nt, *[dev(a) for a in c["tiles"]],
            None if identical else dev(c["types"]), norm_st, swap,
            c["is_3d"], c["freq"], *[float(v) for v in c["b"]], nd,
            *[dev(a) for a in c["dirs"]], ws, ws_bytes, beam,
            ob.stream_ptr())
    torch.cuda.synchronize()
    return beam.cpu().numpy()


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("flags", [(1, 1, 1, 0), (0, 1, 0, 1), (1, 0, 1, 0)])
@pytest.mark.parametrize("is_3d", [1, 0])
def test_two_level_station_types(real, flags, is_3d):
    """Tiles of two layouts (data index = tile type)."""
    c = station(real, seed=3 + is_3d, is_3d=is_3d)
    got = gpu_two_level(c, real, flags, identical=False)
    ref = oracle_two_level(c, real, flags, identical=False)
    assert rel(got, ref) <= TOL[real], rel(got, ref)
    below = c["dirs"][2] < 0
    assert not got.reshape(-1, 8)[below].any()


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_two_level_identical_tiles(real):
    """Identical children: one tile beam, no copies (type index 0 for every
    tile), against the reference's copy-to-every-child composition."""
    c = station(real, seed=11, num_tiles=48)
    flags = (1, 1, 1, 0)
    got = gpu_two_level(c, real, flags, identical=True)
    ref = oracle_two_level(c, real, flags, identical=True)
    assert rel(got, ref) <= TOL[real], rel(got, ref)


def test_two_level_workspace_checked():
    c = station(np.float64, seed=2)
    nd, nt = len(c["dirs"][0]), len(c["tiles"][0])
    need = ob.call("oskb_station_beam_two_level_workspace_bytes", 8, 2, nt,
                   nd, check=False)
    assert need > 0
    ws = torch.empty(need - 256, dtype=torch.uint8, device="cuda")
    beam = torch.zeros(nd * 8, dtype=torch.float64, device="cuda")
    el = [dev(np.concatenate([l[i] for l in c["layouts"]])) for i in range(3)]
    st = ob.call("oskb_station_beam_two_level_d", 2, 16, *el, dev(c["ox"]),
                 dev(c["oy"]), 1.4, 1, 1, nt, *[dev(a) for a in c["tiles"]],
                 dev(c["types"]), 1, 0, 1, 150e6, *[float(v) for v in c["b"]],
                 nd, *[dev(a) for a in c["dirs"]], ws, ws.numel(), beam,
                 ob.stream_ptr(), check=False)
    assert st == -6


# ---------------------------------------------------------------------------
# Any depth: a tree of node types, level 0 the dipole layouts, the top level
# the station. The oracle recurses over the tree the reference's way (every
# child's beam evaluated, identical children copied), the GPU evaluates each
# node type once.
# ---------------------------------------------------------------------------

def tree(real, seed, num_types=(2, 2, 1), num_children=(7, 12), is_3d=1,
         num_dir=600, identical=False):
    """num_types per level (the last 1), num_children per node at each level
    above 0 (varied by +-2 from node to node), children spread over a few
    times the size of the level below; pointings differ by level."""
    rng = np.random.default_rng(seed)
    L = len(num_types)
    cast = lambda a: np.ascontiguousarray(a, dtype=real)
    g = np.arange(4) * 1.25 - 1.875
    gx, gy = np.meshgrid(g, g)
    layouts = []
    for t in range(num_types[0]):
        layouts.append(tuple(map(cast, (
            gx.ravel() + rng.normal(0, 0.05, 16),
            gy.ravel() + rng.normal(0, 0.05, 16),
            rng.uniform(-0.1, 0.1, 16) if is_3d else np.zeros(16)))))
    nodes = []       # per level >= 1: list of (x, y, z, types)
    scale = 5.0
    for l in range(1, L):
        level = []
        for j in range(num_types[l]):
            nc = max(1, num_children[l - 1] + (0 if identical else
                                               int(rng.integers(-2, 3))))
            r = scale * np.sqrt(rng.uniform(0, 1, nc))
            th = rng.uniform(0, 2 * np.pi, nc)
            z = rng.uniform(-0.2, 0.2, nc) * scale / 5 if is_3d else \
                np.zeros(nc)
            types = (np.zeros(nc, np.int32) if identical else
                     rng.integers(0, num_types[l - 1], nc).astype(np.int32))
            level.append((cast(r * np.cos(th)), cast(r * np.sin(th)),
                          cast(z), types))
        nodes.append(level)
        scale *= 4.0
    pointing = []
    for l in range(L):
        b = np.array([0.15 + 0.02 * l, -0.25 + 0.01 * l, 0.0])
        b[2] = np.sqrt(1 - b[0] ** 2 - b[1] ** 2)
        pointing.append(b)
    return dict(layouts=layouts, nodes=nodes, pointing=pointing,
                ox=rng.uniform(0, 0.3, num_types[0]),
                oy=rng.uniform(0, 0.3, num_types[0]) + np.pi / 2,
                dirs=enu_dirs(rng, num_dir, real), freq=120e6, L=1.3,
                is_3d=is_3d, num_types=list(num_types), identical=identical)


def oracle_tree(c, real, norms, norm_el=1, swap=0):
    s = suffix(real)
    nd = len(c["dirs"][0])
    k = real(2 * np.pi * c["freq"] / C0)
    beams = []
    b0 = c["pointing"][0]
    for i, (x, y, z) in enumerate(c["layouts"]):
        out = np.zeros(8 * nd, real)
        oracle().call("station_beam_aa_" + s, np.float64, len(x), x, y, z,
                      None, None, None, np.zeros(len(x), real),
                      float(c["ox"][i]), float(c["oy"][i]), c["L"], norm_el,
                      norms[0], 0, swap, c["is_3d"], c["freq"], *b0, *b0,
                      nd, *c["dirs"], out)
        beams.append(out)
    for l, level in enumerate(c["nodes"], start=1):
        b = c["pointing"][l]
        nxt = []
        for (cx, cy, cz, types) in level:
            nc = len(cx)
            w = np.zeros(2 * nc, real)
            oracle().call("element_weights_dft_" + s, real, nc, cx, cy, cz,
                          np.zeros(nc, real), k, real(b[0]), real(b[1]),
                          real(b[2] if c["is_3d"] else 0.0), w)
            if c["identical"]:
                # the reference's identical children: the first child's beam
                # copied to every child, data indexed by child
                data, idx = np.concatenate([beams[0]] * nc), None
            else:
                data, idx = np.concatenate(beams), types
            out = np.zeros(8 * nd, real)
            oracle().call("dftw_" + s, real, 1, c["is_3d"], nc, k, w, cx, cy,
                          cz, 0, nd, *c["dirs"], idx, data, 1, 1, 0, out,
                          real(1.0 / nc) if norms[l] else real(1.0))
            nxt.append(out)
        beams = nxt
    return beams[0]


def gpu_tree_args(c, real):
    lay = c["layouts"]
    el = [dev(np.concatenate([l[i] for l in lay])) for i in range(3)]
    nodes = [n for level in c["nodes"] for n in level]
    start = np.concatenate([[0], np.cumsum([len(n[0]) for n in nodes])])
    child = [dev(np.concatenate([n[i] for n in nodes])) for i in range(3)]
    types = None if c["identical"] else \
        dev(np.concatenate([n[3] for n in nodes]).astype(np.int32))
    return el, start.astype(np.int32), child, types


def gpu_tree(c, real, norms, norm_el=1, swap=0):
    s = suffix(real)
    el, start, child, types = gpu_tree_args(c, real)
    nd = len(c["dirs"][0])
    L = len(c["num_types"])
    nt = np.asarray(c["num_types"], np.int32)
    ws_bytes = ob.call("oskb_station_beam_hierarchical_workspace_bytes",
                       8 if real == np.float64 else 4, L, nt, start, nd,
                       check=False)
    assert ws_bytes > 0
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    beam = torch.zeros(nd * 8, dtype=torch.float64 if real == np.float64
                       else torch.float32, device="cuda")
    ob.call("oskb_station_beam_hierarchical_" + s, L, nt, 16, *el,
            dev(c["ox"]), dev(c["oy"]), c["L"], norm_el,
            np.asarray(norms, np.int32), start, *child, types, swap,
            c["is_3d"], c["freq"], np.concatenate(c["pointing"]), nd,
            *[dev(a) for a in c["dirs"]], ws, ws_bytes, beam,
            ob.stream_ptr())
    torch.cuda.synchronize()
    return beam.cpu().numpy()


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("norms", [(1, 1, 1), (0, 1, 0), (1, 0, 1)])
@pytest.mark.parametrize("is_3d", [1, 0])
def test_three_level_station(real, norms, is_3d):
    """Dipole tiles of two layouts in sub-stations of two kinds, the
    sub-stations in a station: children indexed by type at both levels."""
    c = tree(real, seed=20 + is_3d, is_3d=is_3d)
    got = gpu_tree(c, real, norms)
    ref = oracle_tree(c, real, norms)
    assert rel(got, ref) <= TOL[real], rel(got, ref)
    below = c["dirs"][2] < 0
    assert not got.reshape(-1, 8)[below].any()
    assert np.abs(got).max() > 0


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_four_level_station(real):
    """Four levels of three, three, two and one node types, with swapped
    dipoles and no element normalisation."""
    c = tree(real, seed=31, num_types=(3, 3, 2, 1), num_children=(5, 6, 8))
    norms = (1, 1, 0, 1)
    got = gpu_tree(c, real, norms, norm_el=0, swap=1)
    ref = oracle_tree(c, real, norms, norm_el=0, swap=1)
    assert rel(got, ref) <= TOL[real], rel(got, ref)


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_identical_children_all_levels(real):
    """Identical children at every level (child_type NULL: one beam per
    level, no copies) against the reference's copy-the-first-child
    recursion."""
    c = tree(real, seed=41, num_types=(1, 1, 1, 1), num_children=(6, 5, 7),
             identical=True)
    norms = (1, 1, 1, 1)
    got = gpu_tree(c, real, norms)
    ref = oracle_tree(c, real, norms)
    assert rel(got, ref) <= TOL[real], rel(got, ref)


def test_two_level_is_the_depth_two_hierarchy():
    """oskb_station_beam_two_level gives the depth-2 hierarchy's beam bit
    for bit."""
    real = np.float64
    c = tree(real, seed=5, num_types=(2, 1), num_children=(30,))
    c["pointing"][1] = c["pointing"][0]
    got = gpu_tree(c, real, (1, 1))
    el, start, child, types = gpu_tree_args(c, real)
    nd = len(c["dirs"][0])
    nt = int(start[-1])
    ws_bytes = ob.call("oskb_station_beam_two_level_workspace_bytes", 8, 2,
                       nt, nd, check=False)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    beam = torch.zeros(nd * 8, dtype=torch.float64, device="cuda")
    ob.call("oskb_station_beam_two_level_d", 2, 16, *el, dev(c["ox"]),
            dev(c["oy"]), c["L"], 1, 1, nt, *child, types, 1, 0, c["is_3d"],
            c["freq"], *[float(v) for v in c["pointing"][0]], nd,
            *[dev(a) for a in c["dirs"]], ws, ws_bytes, beam,
            ob.stream_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(beam.cpu().numpy(), got)
