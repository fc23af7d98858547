"""The pipelined tensor-core block plan (oskb_tc_plan_*): the first block
picks the contraction form by timing the candidates, each slot's compute
work is captured into a CUDA graph at its first block and replayed after
that. Every block's downloaded visibilities must equal, bit for bit, the
device-buffer entry point oskb_correlate_block_tc run with the same
contraction form on the same inputs (the forms are parity-tested against
the oracle in tests/test_gpu_tc.py)."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(),
                                 reason="needs a CUDA device")]

import oskar_b200 as ob  # noqa: E402
from test_gpu_tc import sky, stations, C0  # noqa: E402

# environment that makes the library default equal to plan form 1, 3, 4, 5
FORM_ENV = {1: {}, 3: {"OSKB_TC_TILE": "128"}, 4: {"OSKB_TC_TILE": "256"},
            5: {"OSKB_TC_TILE": "512"}}
ENV_KEYS = ("OSKB_TC_TILE", "OSKB_TC_ARITH", "OSKB_TC_PLAN_FORM",
            "OSKB_TC_PLAN_TUNE", "OSKB_TC_PLAN_GRAPH")


def make_case(seed=9, nst=97, nsrc=900, nt=3, nch=2, nblocks=3):
    rng = np.random.default_rng(seed)
    l, m, n, I, Q, U, V = sky(rng, nsrc)
    E = rng.normal(0, 0.1, (nst, nsrc, 8)).astype(np.float32)
    E[..., 0] += 1
    E[..., 6] += 1
    uvws = [np.stack([np.stack(stations(rng, nst)) for _ in range(nt)])
            for _ in range(nblocks)]
    freqs = 110e6 + 3e6 * np.arange(nch)
    return dict(sky=(l, m, n, I, Q, U, V), E=E, uvws=uvws, freqs=freqs,
                nst=nst, nsrc=nsrc, nt=nt, nch=nch)


def run_plan(c):
    lib = ob.load()
    st = ctypes.c_int(0)
    nbl = c["nst"] * (c["nst"] - 1) // 2
    plan = lib.oskb_tc_plan_create(0, c["nsrc"], c["nst"], c["nt"], c["nch"],
                                   c["freqs"].ctypes.data, 0.0, 3e38,
                                   ctypes.addressof(st))
    assert st.value == 0 and plan
    try:
        ob.call("oskb_tc_plan_set_sky", plan,
                *[np.ascontiguousarray(a) for a in c["sky"]])
        outs = [np.zeros((c["nt"], c["nch"], nbl, 8)) for _ in c["uvws"]]
        for u, o in zip(c["uvws"], outs):
            assert ob.call("oskb_tc_plan_enqueue", plan, c["E"],
                           np.ascontiguousarray(u), o) == 0
        assert ob.call("oskb_tc_plan_wait", plan) == 0
        ms = (ctypes.c_double * 3)()
        ob.call("oskb_tc_plan_tuning_ms", plan, ctypes.addressof(ms))
        return (outs, lib.oskb_tc_plan_form(plan),
                lib.oskb_tc_plan_graph_launches(plan), list(ms))
    finally:
        lib.oskb_tc_plan_free(plan)


def run_direct(c, form, monkeypatch):
    """oskb_correlate_block_tc on device buffers with the form fixed by the
    environment."""
    for k in ENV_KEYS:
        monkeypatch.delenv(k, raising=False)
    for k, v in FORM_ENV[form].items():
        monkeypatch.setenv(k, v)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    nbl = c["nst"] * (c["nst"] - 1) // 2
    args = [dev(c["E"])] + [dev(a) for a in c["sky"]]
    outs = []
    for u in c["uvws"]:
        vis = torch.zeros((c["nt"], c["nch"], nbl, 8), dtype=torch.float64,
                          device="cuda")
        ob.call("oskb_correlate_block_tc", 0, c["nsrc"], c["nst"], c["nt"],
                c["nch"], *args, dev(u), dev(c["freqs"] / C0), 0.0, 3e38,
                vis, None, 0, ob.stream_ptr())
        torch.cuda.synchronize()
        outs.append(vis.cpu().numpy())
    assert ob.load().oskb_tc_arithmetic() == (8 if form == 1 else 16)
    return outs


def test_plan_tunes_and_replays_graphs(monkeypatch):
    for k in ENV_KEYS:
        monkeypatch.delenv(k, raising=False)
    c = make_case()
    outs, form, launches, ms = run_plan(c)
    assert form in (1, 3, 4)
    assert all(t > 0 for t in ms), ms
    # slot 0 replays blocks 0 and 2, slot 1 block 1
    assert launches == 3, ob.load().oskb_last_error().decode()
    ref = run_direct(c, form, monkeypatch)
    for o, r in zip(outs, ref):
        assert np.array_equal(o, r)


@pytest.mark.parametrize("form", [1, 3, 4])
@pytest.mark.parametrize("graph", ["1", "0"])
def test_plan_fixed_form(form, graph, monkeypatch):
    """A fixed form (no tuning), with and without graphs."""
    for k in ENV_KEYS:
        monkeypatch.delenv(k, raising=False)
    monkeypatch.setenv("OSKB_TC_PLAN_FORM", str(form))
    monkeypatch.setenv("OSKB_TC_PLAN_GRAPH", graph)
    c = make_case(seed=10 + form, nt=2, nblocks=3)
    outs, got_form, launches, ms = run_plan(c)
    assert got_form == form
    assert ms == [-1.0, -1.0, -1.0]
    assert launches == (3 if graph == "1" else 0), \
        ob.load().oskb_last_error().decode()
    ref = run_direct(c, form, monkeypatch)
    for o, r in zip(outs, ref):
        assert np.array_equal(o, r)
