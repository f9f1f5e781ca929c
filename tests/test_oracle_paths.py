"""CPU tests pinning the oracle's non-MVS paths to the reference's own code.

tests/golden/ref_cuda_paths.npz holds inputs and outputs of the reference's
CUDA backend (mercury_cuda.cu built unchanged for sm_100a, driven through its
C ABI on a B200 by tests/golden/make_ref_cuda_golden.py): the force matrix of
mercury_cuda_force, RADAU/BS/BS2 runs through mercury_cuda_step + _events,
HYBRID runs through hybrid_begin / the encounter subsystem / hybrid_finish,
the output corrector behind export(h, 1), MVS with the oblateness reaction and
with massive Small bodies, and the TEST algorithm. The oracle runs the same
inputs on the host and must agree at the reference's own bars: 2e-12 relative
for forces (reference tests/test_mercury.py:113-133) and 1e-10 AU, AU/day
absolute for integrated states (tests/test_gpu_algorithms.py:32), with event
identities (ids, kinds) equal.
"""
from pathlib import Path

import numpy as np
import pytest

from adaptive_cases import oracle_intervals
from mercuda_b200.system import System

GOLDEN = Path(__file__).resolve().parent / "golden" / "ref_cuda_paths.npz"
STATE_BAR = 1e-10


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def names(prefix):
    with np.load(GOLDEN) as g:
        return sorted({k.split("/")[0] for k in g.files if k.startswith(prefix)})


def system(g, name):
    s = System(m=g[f"{name}/m"], x=g[f"{name}/x0"], v=g[f"{name}/v0"], nbig=int(g[f"{name}/nbig"]),
               ngf=g[f"{name}/ngf"], jcen=g[f"{name}/jcen"].copy(), rce=g[f"{name}/rce"].copy(),
               rphys=g[f"{name}/rphys"].copy(), rcrit=g[f"{name}/rcrit"].copy(), pn=int(g[f"{name}/pn"]))
    return s


def event_keys(ev):
    return sorted((min(int(e["i"]), int(e["j"])), max(int(e["i"]), int(e["j"])), int(e["kind"])) for e in ev)


@pytest.mark.parametrize("name", names("force_"))
def test_force_matrix_matches_reference(oracle, golden, name):
    s = system(golden, name)
    want = golden[f"{name}/a"]
    got = oracle.force(s)
    rel = np.max(np.abs(got[1:] - want[1:]) / np.maximum(np.abs(want[1:]), 1e-20))
    assert rel < 2e-12, rel


@pytest.mark.parametrize("name", names("hvar_"))
def test_adaptive_runs_match_reference(oracle, golden, name):
    """mal_hvar with mdt_ra15 / mdt_bs1 / mdt_bs2 over 32 days in 7.3-day output
    intervals: final states within 1e-10 of the reference's, same events."""
    alg = {"RADAU": 4, "BS": 2, "BS2": 3}[name.split("_")[1]]
    s = system(golden, name)
    direction = -1.0 if name.endswith("d-1") else 1.0
    ev, h, steps, forces, rejected = oracle_intervals(oracle, s, alg, 0.0, 32.0 * direction, 7.3, 0.5, 1e-12)
    dx = np.max(np.abs(s.x - golden[f"{name}/x"]))
    dv = np.max(np.abs(s.v - golden[f"{name}/v"]))
    assert dx < STATE_BAR and dv < STATE_BAR, (dx, dv)
    assert event_keys(ev) == event_keys(golden[f"{name}/events"])


@pytest.mark.parametrize("name", names("hy_"))
def test_hybrid_runs_match_reference(oracle, golden, name):
    """mdt_hy with mdt_hkce's BS2 subsystem: final democratic-heliocentric states
    within 1e-10, the same encounter pairs and records, and the physical
    velocities of export(h, 1)."""
    s = system(golden, name)
    h = float(golden[f"{name}/h"])
    nsteps = int(golden[f"{name}/nsteps"])
    ev, _, forces, pairs = oracle.hy_run(s, 0.0, h, nsteps)
    dx = np.max(np.abs(s.x - golden[f"{name}/x"]))
    dv = np.max(np.abs(s.v - golden[f"{name}/v"]))
    assert dx < STATE_BAR and dv < STATE_BAR, (dx, dv)
    assert pairs == int(golden[f"{name}/pairs"])
    assert event_keys(ev) == event_keys(golden[f"{name}/events"])
    # physical (heliocentric) velocities: v + sum_k m_k v_k / m_0
    vh = s.v.copy()
    vh[1:] = s.v[1:] + (s.m[1:, None] * s.v[1:]).sum(axis=0) / s.m[0]
    assert np.max(np.abs(golden[f"{name}/xe"] - s.x)) < STATE_BAR
    assert np.max(np.abs(golden[f"{name}/ve"][1:] - vh[1:])) < STATE_BAR


@pytest.mark.parametrize("name", names("mvs_"))
def test_mvs_variants_match_reference(oracle, golden, name):
    """MVS with the oblateness reaction, massive Small bodies, Marsden terms,
    backwards, the TEST algorithm: final states within 1e-10, identical event
    lists (ids, kinds, steps), and export(h, 1): the output corrector for MVS,
    the map variables themselves for TEST."""
    s = system(golden, name)
    h = float(golden[f"{name}/h"])
    nsteps = int(golden[f"{name}/nsteps"])
    ev, st = oracle.mvs_run(s, 0.0, h, nsteps, 0.005, central=True, threads=4)
    dx = np.max(np.abs(s.x - golden[f"{name}/x"]))
    dv = np.max(np.abs(s.v - golden[f"{name}/v"]))
    assert dx < STATE_BAR and dv < STATE_BAR, (dx, dv)
    key = lambda e, k: (int(k), min(int(e["i"]), int(e["j"])), max(int(e["i"]), int(e["j"])), int(e["kind"]))
    assert sorted(map(key, ev, st)) == sorted(map(key, golden[f"{name}/events"], golden[f"{name}/event_steps"]))
    if int(golden[f"{name}/algorithm"]) == 1:
        xe, ve = oracle.mvs_corrector(s, h, forward=True)
    else:   # the TEST algorithm exports its map variables unchanged (mercury_cuda.cu:504-516)
        xe, ve = s.x, s.v
    assert np.max(np.abs(xe[1:] - golden[f"{name}/xe"][1:])) < STATE_BAR
    assert np.max(np.abs(ve[1:] - golden[f"{name}/ve"][1:])) < STATE_BAR
