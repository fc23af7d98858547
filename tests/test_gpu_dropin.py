"""The drop-in oskar_interferometer_run_block inside the unmodified
reference simulator, against the reference's own CPU run.

Each case runs tests/ref_sim.py twice in child processes: once as it is
(the reference library's CPU path end to end), once with
oskar_b200/liboskar_b200_dropin.so in LD_PRELOAD, so that the reference's
oskar_interferometer_run (its worker threads, work-unit claiming, block
finalisation and .vis writer) calls the B200 run_block. The visibility
blocks read back from the two .vis files must agree to

    FP64: max |err| <= 1e-12 max |V| and L2 relative <= 1e-12
    FP32: max |err| <= 2e-5 max |V|  and L2 relative <= 2e-5
          (1e-4 with aperture-array station beams)

(the FP32 bounds cover single-precision phases of a few hundred radians
and station-beam sums formed in a different order of operations), cross-
and auto-correlations alike. The committed fixtures
tests/golden/c1_sim*.npz hold the reference's output for the C1 cases
(made by tests/golden/make_golden.py from the same harness), so that
comparison also runs where the reference library is not built.

The reference's CPU path was seen to crash now and then (SIGSEGV in
oskar_sky_scale_flux_with_frequency after its horizon clip): its runs keep
the clip off where every source is above the horizon anyway, and a crashed
reference run is repeated.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(),
                                 reason="needs a CUDA device")]

from dropin_cases import c1_case, c1_extended_case, c2_small_case  # noqa

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "liboskar_refcpu.so")
DROPIN = os.path.join(ROOT, "oskar_b200", "liboskar_b200_dropin.so")
GOLDEN = os.path.join(HERE, "golden")


def run_sim(case, tmp_path, tag, dropin, attempts=4):
    cj = tmp_path / ("%s.json" % tag)
    out = tmp_path / ("%s.npz" % tag)
    cj.write_text(json.dumps(case))
    env = dict(os.environ)
    env.pop("LD_PRELOAD", None)
    if dropin:
        env["LD_PRELOAD"] = DROPIN
    for _ in range(attempts if not dropin else 1):
        r = subprocess.run([sys.executable, os.path.join(HERE, "ref_sim.py"),
                            str(cj), str(out)], env=env, capture_output=True,
                           text=True, timeout=600)
        if r.returncode == 0 or r.returncode != -11:
            break
    assert r.returncode == 0, (tag, r.returncode, r.stdout[-3000:],
                               r.stderr[-3000:])
    d = dict(np.load(out))
    assert bool(d.pop("dropin")[0]) == dropin
    d.pop("run_seconds", None)
    return d


def compare(got, ref, tol):
    assert set(got) == set(ref), (set(got), set(ref))
    for k in ref:
        a = np.asarray(got[k], np.float64)
        b = np.asarray(ref[k], np.float64)
        assert a.shape == b.shape, (k, a.shape, b.shape)
        l2 = np.linalg.norm(a - b) / np.linalg.norm(b)
        mx = np.max(np.abs(a - b)) / np.max(np.abs(b))
        assert l2 <= tol and mx <= tol, (k, l2, mx)


def need_ref():
    if not os.path.exists(REF_LIB):
        pytest.skip("reference library not built (make -C oracle ref_lib)")


CASES = {
    # C1 as stated: one shared isotropic station model, full polarisation
    "c1": lambda p: c1_case(p, horizon_clip=0),
    # one model per station: Jones R from each station's own latitude and
    # longitude (cross-polarisation from R alone)
    "c1_stations": lambda p: c1_case(p, horizon_clip=0,
                                     station_per_folder=1),
    # spectral full-Stokes fluxes, Gaussians, both smearings, autos, uv
    # filter, two sky chunks, blocks of 4 dumps, two device threads
    "c1_extended": lambda p: c1_extended_case(p, horizon_clip=0),
    # Stokes-I only (scalar Jones, complex visibilities)
    "c1_scalar": lambda p: c1_case(p, horizon_clip=0, pol_mode="Scalar"),
    # aperture-array station beams (48 dipoles per station, the weights
    # steered to the phase centre, normalised there), one layout per
    # station or one shared by all, both polarisation modes
    "c2_small": lambda p: c2_small_case(p),
    "c2_small_shared": lambda p: c2_small_case(p, per_station=False),
    "c2_small_scalar": lambda p: c2_small_case(p, pol_mode="Scalar"),
}
# FP32 bound per case: the single-precision station beams (48-element sums
# and the division by the beam at the phase centre, in a different order of
# operations than the reference's) widen it for the aperture arrays
TOL32 = {"c2_small": 1e-4, "c2_small_shared": 1e-4, "c2_small_scalar": 1e-4}


@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_dropin_matches_reference_run(name, precision, tmp_path):
    need_ref()
    case = CASES[name](precision)
    ref = run_sim(case, tmp_path, "ref", dropin=False)
    got = run_sim(case, tmp_path, "b200", dropin=True)
    compare(got, ref, 1e-12 if precision == "double" else
            TOL32.get(name, 2e-5))


@pytest.mark.parametrize("name", ["c1", "c1_stations"])
def test_dropin_matches_golden(name, tmp_path):
    """Against the committed reference output (no reference library
    needed); the drop-in also runs its own horizon clip, which keeps every
    source of this field."""
    case = CASES[name]("double")
    case["horizon_clip"] = 1
    got = run_sim(case, tmp_path, "b200", dropin=True)
    g = dict(np.load(os.path.join(GOLDEN, "%s_sim.npz" % name)))
    g.pop("dropin", None)
    compare(got, g, 1e-12)


def test_dropin_horizon_clip(tmp_path):
    """Sources on both sides of the horizon: with the clip on in both runs
    (the reference's repeated if it crashes), the drop-in's device clip
    keeps the same sources in the same order."""
    need_ref()
    case = c1_case("double")
    rng = np.random.default_rng(3)
    n = len(case["I"])
    # half the sky over the whole celestial sphere: many below the horizon
    ra = np.asarray(case["ra_rad"])
    dec = np.asarray(case["dec_rad"])
    far = rng.uniform(0, 1, n) < 0.5
    ra[far] = rng.uniform(0, 2 * np.pi, far.sum())
    dec[far] = np.arcsin(rng.uniform(-1, 1, far.sum()))
    case.update(ra_rad=ra.tolist(), dec_rad=dec.tolist(), horizon_clip=1,
                max_sources_per_chunk=300)
    ref = run_sim(case, tmp_path, "ref", dropin=False)
    got = run_sim(case, tmp_path, "b200", dropin=True)
    compare(got, ref, 1e-12)
