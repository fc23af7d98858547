"""CPU checks of the end-to-end simulator fixtures and of the drop-in's
binding to the reference library.

- The reference's own simulator (oracle/_ref/liboskar_refcpu.so, its CPU
  library compiled from its sources) run through tests/ref_sim.py
  reproduces the committed fixtures tests/golden/c1_sim*.npz.
- With oskar_b200/liboskar_b200_dropin.so in LD_PRELOAD, the reference's
  oskar_interferometer_run reaches the drop-in run_block: on a machine
  without a GPU it reports OSKAR_ERR_CUDA_NOT_AVAILABLE (-16) instead of
  running its own CPU path, which shows the interposition and the
  drop-in's check of the simulator's layout (done before the device
  check) without a kernel call.
- The shared-model C1 fixture carries no cross-polarisation beyond
  rounding (every station has the same parallactic rotation, and Q = U =
  V = 0), the per-station one carries the ~1e-4 that Jones R adds.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from dropin_cases import c1_case

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "liboskar_refcpu.so")
DROPIN = os.path.join(ROOT, "oskar_b200", "liboskar_b200_dropin.so")


def _run(case, tmp_path, preload=None, attempts=4):
    cj = tmp_path / "case.json"
    out = tmp_path / "out.npz"
    cj.write_text(json.dumps(case))
    env = {k: v for k, v in os.environ.items() if k != "LD_PRELOAD"}
    if preload:
        env["LD_PRELOAD"] = preload
    for _ in range(attempts):
        r = subprocess.run([sys.executable, os.path.join(HERE, "ref_sim.py"),
                            str(cj), str(out)], env=env, capture_output=True,
                           text=True, timeout=300)
        if r.returncode != -11:
            break
    return r, out


@pytest.mark.parametrize("name,kw", [
    ("c1_sim.npz", {}), ("c1_stations_sim.npz", {"station_per_folder": 1})])
def test_reference_reproduces_fixture(name, kw, tmp_path):
    if not os.path.exists(REF_LIB):
        pytest.skip("reference library not built")
    r, out = _run(c1_case("double", horizon_clip=0, **kw), tmp_path)
    assert r.returncode == 0, r.stderr[-2000:]
    got = np.load(out)["cross"]
    ref = np.load(os.path.join(HERE, "golden", name))["cross"]
    assert got.shape == ref.shape
    assert np.max(np.abs(got - ref)) <= 1e-14 * np.max(np.abs(ref))


def test_fixture_cross_polarisation():
    def xy_over_xx(name):
        d = np.load(os.path.join(HERE, "golden", name))["cross"]
        v = d.reshape(d.shape[0], d.shape[1], -1, 4, 2)
        a = np.hypot(v[..., 0], v[..., 1])
        return a[..., 1].mean() / a[..., 0].mean()
    assert xy_over_xx("c1_sim.npz") < 1e-12
    assert 1e-5 < xy_over_xx("c1_stations_sim.npz") < 1e-3


def test_dropin_is_reached_without_gpu(tmp_path):
    if not os.path.exists(REF_LIB) or not os.path.exists(DROPIN):
        pytest.skip("reference library or drop-in not built")
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present: the GPU tests run the drop-in")
    except ImportError:
        pass
    r, _ = _run(c1_case("double", horizon_clip=0), tmp_path,
                preload=DROPIN, attempts=1)
    assert r.returncode != 0
    assert "OSKAR status -16" in r.stderr, r.stderr[-2000:]
