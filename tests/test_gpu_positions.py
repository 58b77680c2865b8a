"""Rows built on the device from positions (GPU): mtp_compute_positions.

A pair style with device-side rows sends positions of local and ghost atoms,
their owners and species, and the raw neighbour list (skin included).  The GPU
must keep exactly the candidates a host loop keeps (pair_jax_mtp.cpp:110-167:
|x_j - x_i| < cutoff, list order, ghost -> owner, unowned ghost -> species -1),
so the results are bitwise those of mtp_compute on host-packed rows.
"""

import ctypes

import numpy as np
import pytest

from conftest import potential_path
from mtp_b200 import synth
from mtp_b200._lib import EATOM, EFLAG, VATOM, VFLAG, MTPError, check, lib
from mtp_b200.engine import MTPEngine, pinned_empty

pytestmark = pytest.mark.gpu

CUTOFF, SKIN = 5.0, 0.3


def _system(kind, a, reps, seed, nspecies):
    s = synth.lattice_structure(kind, a, reps)
    rng = np.random.default_rng(seed)
    s.positions = s.positions + rng.normal(0.0, 0.08, s.positions.shape)
    s.types = rng.integers(0, nspecies, s.natoms).astype(np.int32)
    x, owner, lists = synth.ghosts_and_lists(s, CUTOFF + SKIN)
    species = s.types[owner].astype(np.int32)
    return s.natoms, x, species, owner, lists


def _pack_lists(N, lists, rng=None):
    stride = max(len(c) for c in lists)
    neigh = np.full((N, stride), -1, np.int32)
    num = np.zeros(N, np.int32)
    for i, c in enumerate(lists):
        c = c if rng is None else rng.permutation(c)
        neigh[i, :len(c)] = c
        num[i] = len(c)
    return neigh, num


def _host_rows(N, x, species, owner, neigh, num, max_nbr):
    """The pair style's host loop, operation for operation."""
    cut2 = CUTOFF * CUTOFF
    rij = np.zeros((N, max_nbr, 3))
    js = np.full((N, max_nbr), -1, np.int32)
    jt = np.full((N, max_nbr), -1, np.int32)
    cnt = np.zeros(N, np.int32)
    for i in range(N):
        n = 0
        for j in neigh[i, :num[i]]:
            if j == i or j >= len(x):
                continue
            dx, dy, dz = x[j, 0] - x[i, 0], x[j, 1] - x[i, 1], x[j, 2] - x[i, 2]
            if dx * dx + dy * dy + dz * dz >= cut2:
                continue
            rij[i, n] = (dx, dy, dz)
            js[i, n] = owner[j]
            jt[i, n] = species[j] if owner[j] >= 0 else -1
            n += 1
        cnt[i] = n
    return rij, js, jt, cnt


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("kind,a,reps,pot", [("bcc", 2.87, (3, 3, 3), "cfg1md_L16_S2.mtp"),
                                             ("fcc", 3.6, (3, 3, 3), "cfg2md_L24_S3.mtp")])
def test_device_rows_are_bitwise_the_host_rows(kind, a, reps, pot, precision):
    path = potential_path(pot)
    nspecies = 2 if "S2" in pot else 3
    N, x, species, owner, lists = _system(kind, a, reps, 7, nspecies)
    owner = owner.copy()
    owner[N + 5] = -1                      # one ghost without an owner: species -1 in its rows
    neigh, num = _pack_lists(N, lists, np.random.default_rng(8))
    max_nbr = 64
    rows = _host_rows(N, x, species, owner, neigh, num, max_nbr)
    assert rows[3].max() <= max_nbr and rows[3].min() > 0
    with MTPEngine(path, N, max_nbr, cutoff=CUTOFF, precision=precision) as eng:
        ref = eng.compute(species[:N], *rows, eatom=True, vatom=True)
        for _ in range(2):
            got = eng.compute_positions(N, x, species, owner, neigh, num, eatom=True, vatom=True)
            for k in ("energy", "forces", "virial", "site_energies", "vatom"):
                assert np.array_equal(np.asarray(got[k]), np.asarray(ref[k])), k


def test_overfull_row_is_a_capacity_error_and_the_handle_recovers():
    path = potential_path("cfg1md_L16_S2.mtp")
    N, x, species, owner, lists = _system("bcc", 2.87, (3, 3, 3), 9, 2)
    neigh, num = _pack_lists(N, lists)
    kept = _host_rows(N, x, species, owner, neigh, num, 96)[3]
    small = int(kept.max()) - 4
    with MTPEngine(path, N, small, cutoff=CUTOFF) as eng:
        with pytest.raises(MTPError, match="MTP_E_CAPACITY"):
            eng.compute_positions(N, x, species, owner, neigh, num)
        # the same handle afterwards: lists cut to at most `small` candidates
        cut = np.minimum(num, small).astype(np.int32)
        rows = _host_rows(N, x, species, owner, neigh, cut, small)
        ref = eng.compute(species[:N], *rows)
        got = eng.compute_positions(N, x, species, owner, neigh, cut)
        assert got["energy"] == ref["energy"]
        assert np.array_equal(got["forces"], ref["forces"])


def test_page_locked_calls_replay_a_graph_bitwise():
    """Page-locked inputs and outputs: the second call is captured, later calls
    replay it; every result equals the directly enqueued (pageable) call, and a
    replay reads the positions as they are at the call."""
    path = potential_path("cfg1md_L16_S2.mtp")
    N, x, species, owner, lists = _system("bcc", 2.87, (3, 3, 3), 11, 2)
    neigh, num = _pack_lists(N, lists)
    arrays = {"x": x, "sp": species, "own": owner, "nb": neigh, "num": num}
    pin = {}
    for k, a in arrays.items():
        pin[k] = pinned_empty(a.shape, a.dtype)
        pin[k][...] = a
    out = {"e": pinned_empty((1,)), "F": pinned_empty((N, 3)), "vir": pinned_empty((6,)),
           "ea": pinned_empty((N,)), "va": pinned_empty((N, 6))}
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)

    def call(eng):
        check(lib().mtp_compute_positions(eng.handle, N, len(x), P(pin["x"]), P(pin["sp"]), P(pin["own"]),
                                          neigh.shape[1], P(pin["nb"]), P(pin["num"]),
                                          EFLAG | VFLAG | EATOM | VATOM, P(out["e"]), P(out["F"]), P(out["vir"]),
                                          P(out["ea"]), P(out["va"])), eng.handle)
        return {"energy": float(out["e"][0]), "forces": out["F"].copy(), "virial": out["vir"].copy(),
                "site_energies": out["ea"].copy(), "vatom": out["va"].copy()}

    with MTPEngine(path, N, 64, cutoff=CUTOFF) as eng:
        eng.use_own_stream()
        ref = eng.compute_positions(N, x, species, owner, neigh, num, eatom=True, vatom=True)
        runs = [call(eng) for _ in range(4)]
        st = eng.stats()
        assert st["graph_captures"] == 1 and st["graph_replays"] == 2, st
        for r in runs:
            for k in ref:
                assert np.array_equal(np.asarray(r[k]), np.asarray(ref[k])), k
        x2 = x + np.random.default_rng(12).normal(0.0, 0.01, x.shape)
        pin["x"][...] = x2
        moved = call(eng)
        assert eng.stats()["graph_replays"] == 3
        want = eng.compute_positions(N, x2, species, owner, neigh, num, eatom=True, vatom=True)
        for k in want:
            assert np.array_equal(np.asarray(moved[k]), np.asarray(want[k])), k


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_pointer_variant_matches_host_variant(precision):
    """mtp_compute_positions_device (inputs already on the GPU, as a KOKKOS-style
    pair style holds them) gives bitwise the host-buffer variant's results, on
    two calls in a row; an overfull row is reported by sync_status."""
    import torch
    path = potential_path("cfg2md_L24_S3.mtp")
    N, x, species, owner, lists = _system("fcc", 3.6, (3, 3, 3), 13, 3)
    neigh, num = _pack_lists(N, lists, np.random.default_rng(14))
    dev = torch.device("cuda")
    t = lambda a: torch.as_tensor(a).to(dev).contiguous()
    with MTPEngine(path, N, 64, cutoff=CUTOFF, precision=precision) as eng:
        ref = eng.compute_positions(N, x, species, owner, neigh, num, eatom=True, vatom=True)
        for _ in range(2):
            ea = torch.empty(N, dtype=torch.float64, device=dev)
            va = torch.empty((N, 6), dtype=torch.float64, device=dev)
            e, F, w = eng.compute_positions_device(N, t(x), t(species), t(owner), t(neigh), t(num), eatom=ea,
                                                   vatom=va)
            torch.cuda.synchronize()
            eng.sync_status()
            assert float(e.cpu()[0]) == ref["energy"]
            assert np.array_equal(F.cpu().numpy(), ref["forces"])
            assert np.array_equal(w.cpu().numpy(), ref["virial"])
            assert np.array_equal(ea.cpu().numpy(), ref["site_energies"])
            assert np.array_equal(va.cpu().numpy(), ref["vatom"])
    with MTPEngine(path, N, 30, cutoff=CUTOFF, precision=precision) as eng:
        eng.compute_positions_device(N, t(x), t(species), t(owner), t(neigh), t(num))
        torch.cuda.synchronize()
        with pytest.raises(MTPError, match="MTP_E_CAPACITY"):
            eng.sync_status()
