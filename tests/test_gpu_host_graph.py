"""Host-buffer calls below the chunked size (GPU).

With page-locked buffers, mtp_compute captures its copies, kernels and
read-backs as one CUDA graph on the second consecutive call with the same
arguments and replays it while they repeat.  The replay must give bitwise the
results of the directly enqueued work, read the buffers' current contents,
and follow coefficient changes.  mtp_execute_potential packs into persistent
page-locked staging and must agree with mtp_compute on every call.
"""

import ctypes

import numpy as np
import pytest

from conftest import golden_case, potential_path
from mtp_b200._lib import EATOM, EFLAG, VATOM, VFLAG, check, lib
from mtp_b200.engine import MTPEngine, pinned_empty, stress_from_virial
from mtp_b200.mtp_file import read_mtp

pytestmark = pytest.mark.gpu

P = lambda a: a.ctypes.data_as(ctypes.c_void_p)


def _inputs(tag):
    g = golden_case(tag)
    arrs = {k: np.ascontiguousarray(g[k], dt) for k, dt in (("itypes", np.int32), ("rijs", np.float64),
                                                              ("js", np.int32), ("jtypes", np.int32),
                                                              ("counts", np.int32))}
    return potential_path(str(g["potential"])), arrs, float(g["volume"])


def _pinned_copy(arrs):
    out = {}
    for k, a in arrs.items():
        out[k] = pinned_empty(a.shape, a.dtype)
        out[k][...] = a
    return out


def _call(eng, a, out):
    """mtp_compute into the caller's output arrays (all flags)."""
    N, n = a["js"].shape
    check(lib().mtp_compute(eng.handle, N, n, P(a["itypes"]), P(a["rijs"]), P(a["js"]), P(a["jtypes"]),
                            P(a["counts"]), EFLAG | VFLAG | EATOM | VATOM, P(out["e"]), P(out["F"]), P(out["vir"]),
                            P(out["eatom"]), P(out["vatom"])), eng.handle)
    return {k: v.copy() for k, v in out.items()}


def _outputs(N, alloc):
    return {"e": alloc((1,)), "F": alloc((N, 3)), "vir": alloc((6,)), "eatom": alloc((N,)), "vatom": alloc((N, 6))}


def _same(x, y):
    for k in x:
        assert np.array_equal(x[k], y[k]), k


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_graph_replay_is_bitwise_the_direct_path(precision):
    path, arrs, _ = _inputs("bcc54_L16")
    N, n = arrs["js"].shape
    pin_in = _pinned_copy(arrs)
    pin_out = _outputs(N, lambda s: pinned_empty(s, np.float64))
    page_out = _outputs(N, np.zeros)
    with MTPEngine(path, N, n, precision=precision) as eng:
        eng.use_own_stream()
        ref = _call(eng, arrs, page_out)                  # pageable: enqueued directly
        runs = [_call(eng, pin_in, pin_out) for _ in range(4)]
        st = eng.stats()
        assert st["graph_captures"] == 1 and st["graph_replays"] == 2, st
        for r in runs:
            _same(r, ref)

        # a replay reads the buffers' current contents
        rng = np.random.default_rng(3)
        arrs2 = dict(arrs)
        arrs2["rijs"] = arrs["rijs"] + rng.normal(0.0, 0.01, arrs["rijs"].shape)
        pin_in["rijs"][...] = arrs2["rijs"]
        moved = _call(eng, pin_in, pin_out)
        assert eng.stats()["graph_replays"] == 3
        _same(moved, _call(eng, arrs2, page_out))
        assert not np.array_equal(moved["F"], ref["F"])

        # new coefficients invalidate the graph; the next calls use them
        pot = read_mtp(path)
        theta = np.asarray(pot.moment_coeffs, np.float64) * 1.5
        eng.set_coeffs(moment=theta)
        after = [_call(eng, pin_in, pin_out) for _ in range(3)]
        want = _call(eng, arrs2, page_out)
        for r in after:
            _same(r, want)
        assert eng.stats()["graph_captures"] == 2
        assert not np.array_equal(want["e"], moved["e"])


def test_execute_potential_staging_agrees_on_every_call():
    path, arrs, vol = _inputs("small_L20")
    N, n = arrs["js"].shape
    rng = np.random.default_rng(4)
    with MTPEngine(path, N, n) as eng:
        for k in range(3):
            a = dict(arrs)
            a["rijs"] = arrs["rijs"] + (rng.normal(0.0, 0.01, arrs["rijs"].shape) if k else 0.0)
            e, F, stress = eng.execute_potential(a["itypes"], a["rijs"], a["js"], a["jtypes"], a["counts"], vol)
            ref = eng.compute(a["itypes"], a["rijs"], a["js"], a["jtypes"], a["counts"])
            assert e == ref["energy"]
            assert np.array_equal(F, ref["forces"])
            np.testing.assert_allclose(stress, stress_from_virial(ref["virial"], vol), rtol=1e-15, atol=0)
