"""This library against the reference's own CUDA backend, through the same
drop-in calls on the same inputs.

tests/golden/ref_cuda_paths.npz holds what the reference backend
(mercury_cuda.cu built unchanged for sm_100a) returned on a B200 when driven
as its Fortran host drives it (tests/golden/make_ref_cuda_golden.py): the
force matrix, RADAU/BS/BS2 runs in output intervals, HYBRID runs with the BS2
encounter subsystem, MVS with the oblateness reaction, massive Small bodies,
Marsden terms, backwards and as the TEST algorithm, and the corrected state
of export(h, 1). The bars are the reference's own CPU-vs-CUDA bars: 2e-12
relative for forces (its tests/test_mercury.py:113-133), 1e-10 absolute for
integrated states (tests/test_gpu_algorithms.py:32), identical event
identities.
"""
from pathlib import Path

import numpy as np
import pytest

from adaptive_cases import run_intervals
from mercuda_b200.backend import Backend
from mercuda_b200.system import System

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "ref_cuda_paths.npz"
STATE_BAR = 1e-10


def names(prefix):
    with np.load(GOLDEN) as g:
        return sorted({k.split("/")[0] for k in g.files if k.startswith(prefix)})


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def system(g, name):
    return System(m=g[f"{name}/m"], x=g[f"{name}/x0"], v=g[f"{name}/v0"], nbig=int(g[f"{name}/nbig"]),
                  ngf=g[f"{name}/ngf"], jcen=g[f"{name}/jcen"].copy(), rce=g[f"{name}/rce"].copy(),
                  rphys=g[f"{name}/rphys"].copy(), rcrit=g[f"{name}/rcrit"].copy(), pn=int(g[f"{name}/pn"]))


def event_keys(ev):
    return sorted((min(int(e["i"]), int(e["j"])), max(int(e["i"]), int(e["j"])), int(e["kind"])) for e in ev)


def assert_states(x, v, g, name, bar=STATE_BAR):
    dx = np.max(np.abs(x - g[f"{name}/x"]))
    dv = np.max(np.abs(v - g[f"{name}/v"]))
    assert dx < bar and dv < bar, (dx, dv)


@pytest.mark.parametrize("name", names("force_"))
def test_force_matrix_matches_reference(cuda_lib, golden, name):
    s = system(golden, name)
    be = Backend("BS", cuda_lib)
    be.configure()
    be.upload(s)
    got = be.force()
    be.free()
    want = golden[f"{name}/a"]
    rel = np.max(np.abs(got[1:] - want[1:]) / np.maximum(np.abs(want[1:]), 1e-20))
    assert rel < 2e-12, rel


@pytest.mark.parametrize("name", names("hvar_"))
def test_adaptive_runs_match_reference(cuda_lib, golden, name):
    alg = name.split("_")[1]
    s = system(golden, name)
    direction = -1.0 if name.endswith("d-1") else 1.0
    be = Backend(alg, cuda_lib)
    be.configure()
    be.upload(s)
    ev, h = run_intervals(be, s, 0.0, 32.0 * direction, 7.3, 0.5, 1e-12)
    x, v = be.download()
    be.free()
    assert_states(x, v, golden, name)
    assert event_keys(ev) == event_keys(golden[f"{name}/events"])


@pytest.mark.parametrize("name", names("hy_"))
def test_hybrid_runs_match_reference(cuda_lib, golden, name):
    s = system(golden, name)
    h = float(golden[f"{name}/h"])
    be = Backend("HYBRID", cuda_lib)
    be.configure()
    be.upload(s)
    state = {"dtflag": 0}
    events, pairs, t = [], 0, 0.0
    for _ in range(int(golden[f"{name}/nsteps"])):
        ev, npair = be.hybrid_step(s, t, h, 1e-12, state, 0.005)
        pairs += npair
        t = t + h
        events.append(ev)
        events.append(be.events(t, h, 0.005))
    x, v = be.download()
    xe, ve = be.export(h, physical=True)
    be.free()
    assert_states(x, v, golden, name)
    assert pairs == int(golden[f"{name}/pairs"])
    assert event_keys(np.concatenate(events)) == event_keys(golden[f"{name}/events"])
    assert np.max(np.abs(xe - golden[f"{name}/xe"])) < STATE_BAR
    assert np.max(np.abs(ve - golden[f"{name}/ve"])) < STATE_BAR


@pytest.mark.parametrize("name", names("mvs_"))
def test_mvs_variants_match_reference(cuda_lib, golden, name):
    s = system(golden, name)
    h = float(golden[f"{name}/h"])
    alg = {1: "MVS", 9: "TEST"}[int(golden[f"{name}/algorithm"])]
    be = Backend(alg, cuda_lib)
    be.configure()
    be.upload(s)
    got, t = [], 0.0
    for k in range(int(golden[f"{name}/nsteps"])):
        be.step(t, h, dtflag=0 if k == 0 else 2)
        got.extend((k, min(int(e["i"]), int(e["j"])), max(int(e["i"]), int(e["j"])), int(e["kind"]))
                   for e in be.events(t + h, h, 0.005))
        t = t + h
    x, v = be.download()
    xe, ve = be.export(h, physical=True)
    be.free()
    assert_states(x, v, golden, name)
    want = [(int(k), min(int(e["i"]), int(e["j"])), max(int(e["i"]), int(e["j"])), int(e["kind"]))
            for e, k in zip(golden[f"{name}/events"], golden[f"{name}/event_steps"])]
    assert sorted(got) == sorted(want)
    assert np.max(np.abs(xe[1:] - golden[f"{name}/xe"][1:])) < STATE_BAR
    assert np.max(np.abs(ve[1:] - golden[f"{name}/ve"][1:])) < STATE_BAR
