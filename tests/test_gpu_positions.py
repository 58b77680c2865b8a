"""Rows built on the device from positions (GPU): mtp_compute_positions.

A pair style with device-side rows sends positions of local and ghost atoms,
their owners and species, and the raw neighbour list (skin included).  The GPU
must keep exactly the candidates a host loop keeps (pair_jax_mtp.cpp:110-167:
|x_j - x_i| < cutoff, list order, ghost -> owner, unowned ghost -> species -1),
so the results are bitwise those of mtp_compute on host-packed rows.
"""

import numpy as np
import pytest

from conftest import potential_path
from mtp_b200 import synth
from mtp_b200._lib import MTPError
from mtp_b200.engine import MTPEngine

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
