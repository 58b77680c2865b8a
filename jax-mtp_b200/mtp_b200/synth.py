"""Seeded synthetic atomic structures and padded neighbour data.

The reference ships no benchmark data (its only data is 21 two-atom VASP
configurations), so every workload here is generated from a seed with
``numpy.random.default_rng``:

* lattice sites are enumerated cell by cell with ``iz`` outermost, then
  ``iy``, then ``ix``, and the basis atom innermost;
* thermal displacements are ``N(0, sigma^2)`` per component from their own
  seed; species come from their own seed.

The padded neighbour layout mirrors what the reference's LAMMPS bridge hands
to the evaluator (pair_style_files/pair_jax_mtp.cpp:110-167): per centre atom
a row of ``n_pad`` slots holding ``r_ij = x_j - x_i`` (minimum image or an
explicit periodic image), the owner index of ``j`` and its species; unused
slots carry species ``-1``.
"""

from __future__ import annotations

import dataclasses
import math
from typing import List, Optional, Sequence

import numpy as np

__all__ = [
    "Structure", "NeighborData", "lattice_structure", "build_neighbors", "pack_batch",
    "config0", "config1", "config2_structure", "training_batch", "maxwell_boltzmann",
    "KB_EV", "MVV2E",
]

KB_EV = 8.617333262e-5          # Boltzmann constant, eV/K
MVV2E = 1.0364269e-4            # LAMMPS 'metal': amu*A^2/ps^2 -> eV

_FCC = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
_BCC = np.array([[0, 0, 0], [0.5, 0.5, 0.5]])
_HCP = np.array([[0, 0, 0], [1.0 / 3.0, 2.0 / 3.0, 0.5]])


@dataclasses.dataclass
class Structure:
    positions: np.ndarray   # [N, 3] Cartesian, Angstrom
    cell: np.ndarray        # [3, 3] rows are the lattice vectors
    types: np.ndarray       # [N] int32 species index

    @property
    def natoms(self) -> int:
        return int(self.positions.shape[0])

    @property
    def volume(self) -> float:
        return float(abs(np.linalg.det(self.cell)))


@dataclasses.dataclass
class NeighborData:
    """Padded per-atom neighbour rows (the evaluator's input layout)."""

    itypes: np.ndarray      # [N] int32
    rijs: np.ndarray        # [N, n_pad, 3] float64
    js: np.ndarray          # [N, n_pad] int32 owner index of the neighbour
    jtypes: np.ndarray      # [N, n_pad] int32 species of the neighbour, -1 = empty slot
    counts: np.ndarray      # [N] int32 filled slots per row
    volume: float

    @property
    def natoms(self) -> int:
        return int(self.itypes.shape[0])

    @property
    def n_pad(self) -> int:
        return int(self.js.shape[1])


def _basis(kind: str, a: float):
    if kind == "fcc":
        return _FCC, np.eye(3) * a
    if kind == "bcc":
        return _BCC, np.eye(3) * a
    if kind == "hcp":
        c = a * math.sqrt(8.0 / 3.0)
        cell = np.array([[a, 0, 0], [-0.5 * a, 0.5 * math.sqrt(3.0) * a, 0], [0, 0, c]])
        return _HCP, cell
    raise ValueError(f"unknown lattice {kind!r}")


def lattice_structure(kind: str, a: float, reps: Sequence[int]) -> Structure:
    """Perfect lattice; sites ordered iz, iy, ix (cells) then basis atom."""
    basis, unit = _basis(kind, a)
    nx, ny, nz = (int(r) for r in reps)
    iz, iy, ix = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    cells = np.stack([ix.ravel(), iy.ravel(), iz.ravel()], axis=1).astype(np.float64)
    frac = (cells[:, None, :] + basis[None, :, :]).reshape(-1, 3)
    frac /= np.array([nx, ny, nz], dtype=np.float64)
    cell = unit * np.array([nx, ny, nz], dtype=np.float64)[:, None]
    pos = frac @ cell
    return Structure(pos, cell, np.zeros(len(pos), dtype=np.int32))


def _image_ranges(cell: np.ndarray, cutoff: float) -> np.ndarray:
    vol = abs(np.linalg.det(cell))
    out = []
    for a in range(3):
        b, c = (a + 1) % 3, (a + 2) % 3
        h = vol / np.linalg.norm(np.cross(cell[b], cell[c]))   # plane spacing
        out.append(int(math.ceil(cutoff / h)))
    return np.array(out)


def ghosts_and_lists(s: Structure, rlist: float):
    """Local atoms, periodic ghosts and full neighbour lists as an MD code hands
    them to a pair style (orthorhombic cells whose edges exceed ``rlist``).

    Returns (x [nall, 3] wrapped local positions then ghost images within
    ``rlist`` of the box, owner [nall] int32 local index of each atom's owner,
    lists: for every local atom the indices of all other atoms closer than
    ``rlist``, in index order).
    """
    cell = np.asarray(s.cell, dtype=np.float64)
    if np.count_nonzero(cell - np.diag(np.diag(cell))) or np.any(np.diag(cell) <= rlist):
        raise ValueError("ghosts_and_lists needs an orthorhombic cell with edges longer than rlist")
    L = np.diag(cell).copy()
    N = s.natoms
    pos = np.mod(s.positions, L)
    xs, own = [pos], [np.arange(N)]
    for sx in (-1, 0, 1):
        for sy in (-1, 0, 1):
            for sz in (-1, 0, 1):
                if sx == sy == sz == 0:
                    continue
                img = pos + np.array([sx, sy, sz]) * L
                keep = np.all((img > -rlist) & (img < L + rlist), axis=1)
                xs.append(img[keep])
                own.append(np.arange(N)[keep])
    x = np.concatenate(xs)
    owner = np.concatenate(own).astype(np.int32)
    idx = np.arange(len(x))
    lists = []
    for i in range(N):
        d2 = np.sum((x - x[i]) ** 2, axis=1)
        lists.append(np.nonzero((d2 < rlist * rlist) & (idx != i))[0].astype(np.int32))
    return x, owner, lists


def build_neighbors(s: Structure, cutoff: float, n_pad: Optional[int] = None,
                    pad_multiple: int = 8) -> NeighborData:
    """Full neighbour list with every periodic image inside ``cutoff``.

    Brute force over atom pairs and image shifts (fine for the few-thousand
    atom structures the tests and CPU baselines use).  Rows are sorted by
    (j, image) so the slot order is deterministic.  ``n_pad`` defaults to the
    largest row rounded up to ``pad_multiple``.
    """
    N = s.natoms
    pos = s.positions
    cell = s.cell
    nmax = _image_ranges(cell, cutoff)
    shifts = np.array([[i, j, k] for i in range(-nmax[0], nmax[0] + 1)
                       for j in range(-nmax[1], nmax[1] + 1)
                       for k in range(-nmax[2], nmax[2] + 1)], dtype=np.float64)
    rows_j: List[list] = [[] for _ in range(N)]
    rows_r: List[list] = [[] for _ in range(N)]
    rc2 = cutoff * cutoff
    # wrap to the home cell so shifts are small
    inv = np.linalg.inv(cell)
    frac = pos @ inv
    frac -= np.floor(frac)
    pw = frac @ cell
    chunk = max(1, 4_000_000 // max(1, N * len(shifts)))
    for i0 in range(0, N, chunk):
        i1 = min(N, i0 + chunk)
        # d[i, s, j, :] = pw[j] + shift_s @ cell - pw[i]
        sv = shifts @ cell                                   # [S, 3]
        d = pw[None, None, :, :] + sv[None, :, None, :] - pw[i0:i1, None, None, :]
        r2 = np.einsum("isjk,isjk->isj", d, d)
        ii, ss, jj = np.nonzero(r2 < rc2)
        self_mask = (ii + i0 == jj) & np.all(shifts[ss] == 0, axis=1)
        ii, ss, jj = ii[~self_mask], ss[~self_mask], jj[~self_mask]
        order = np.lexsort((ss, jj, ii))
        ii, ss, jj = ii[order], ss[order], jj[order]
        for a, sh, b in zip(ii, ss, jj):
            rows_j[a + i0].append(b)
            rows_r[a + i0].append(d[a, sh, b])
    counts = np.array([len(r) for r in rows_j], dtype=np.int32)
    maxc = int(counts.max()) if N else 0
    if n_pad is None:
        n_pad = max(pad_multiple, ((maxc + pad_multiple - 1) // pad_multiple) * pad_multiple)
    if maxc > n_pad:
        raise ValueError(f"a row has {maxc} neighbours, more than n_pad={n_pad}")
    rijs = np.zeros((N, n_pad, 3))
    js = np.full((N, n_pad), N, dtype=np.int32)
    jtypes = np.full((N, n_pad), -1, dtype=np.int32)
    for i in range(N):
        c = counts[i]
        if c:
            rijs[i, :c] = np.array(rows_r[i])
            js[i, :c] = rows_j[i]
            jtypes[i, :c] = s.types[np.array(rows_j[i])]
    return NeighborData(s.types.astype(np.int32).copy(), rijs, js, jtypes, counts, s.volume)


def pack_batch(nds: Sequence[NeighborData], n_pad: Optional[int] = None):
    """Concatenate per-configuration neighbour data into one flat atom batch.

    Neighbour indices are offset to global atom indices.  Returns
    ``(NeighborData, config_of_atom [Ntot] int32, atom_offsets [C+1] int64, volumes [C])``.
    """
    if n_pad is None:
        n_pad = max(nd.n_pad for nd in nds)
    tot = sum(nd.natoms for nd in nds)
    rijs = np.zeros((tot, n_pad, 3))
    js = np.full((tot, n_pad), -1, dtype=np.int32)
    jt = np.full((tot, n_pad), -1, dtype=np.int32)
    it = np.zeros(tot, dtype=np.int32)
    cnt = np.zeros(tot, dtype=np.int32)
    cfg = np.zeros(tot, dtype=np.int32)
    offs = np.zeros(len(nds) + 1, dtype=np.int64)
    o = 0
    for c, nd in enumerate(nds):
        n, p = nd.natoms, nd.n_pad
        rijs[o:o + n, :p] = nd.rijs
        jj = nd.js.astype(np.int64).copy()
        valid = nd.jtypes >= 0
        js[o:o + n, :p] = np.where(valid, jj + o, -1)
        jt[o:o + n, :p] = nd.jtypes
        it[o:o + n] = nd.itypes
        cnt[o:o + n] = nd.counts
        cfg[o:o + n] = c
        o += n
        offs[c + 1] = o
    vols = np.array([nd.volume for nd in nds])
    return NeighborData(it, rijs, js, jt, cnt, float("nan")), cfg, offs, vols


# ----------------------------------------------------------------------------
# Workloads (sizes and distributions of the benchmark configurations)
# ----------------------------------------------------------------------------

def config0(seed_pos: int = 1) -> Structure:
    """fcc a=4.05 A, 4x4x4 cells (256 atoms), sigma=0.05 A from ``seed_pos``, 1 species."""
    s = lattice_structure("fcc", 4.05, (4, 4, 4))
    s.positions = s.positions + np.random.default_rng(seed_pos).normal(0.0, 0.05, s.positions.shape)
    return s


def config1(seed_species: int = 3) -> Structure:
    """bcc a=2.87 A, 10x10x10 cells (2000 atoms), species 50/50 from ``seed_species``."""
    s = lattice_structure("bcc", 2.87, (10, 10, 10))
    n = s.natoms
    s.types = np.random.default_rng(seed_species).permutation(
        np.concatenate([np.zeros(n // 2), np.ones(n - n // 2)])).astype(np.int32)
    return s


def config2_structure(reps: int = 64, seed_pos: int = 51, seed_species: int = 52,
                      sigma: float = 0.08) -> Structure:
    """fcc a=3.6 A, reps^3 cells (64^3 -> 1,048,576 atoms), 3 species uniform, sigma=0.08 A."""
    s = lattice_structure("fcc", 3.6, (reps, reps, reps))
    s.positions = s.positions + np.random.default_rng(seed_pos).normal(0.0, sigma, s.positions.shape)
    s.types = np.random.default_rng(seed_species).integers(0, 3, s.natoms).astype(np.int32)
    return s


def maxwell_boltzmann(natoms: int, temperature: float, mass: float, seed: int) -> np.ndarray:
    """Velocities in A/ps (LAMMPS 'metal' units) at ``temperature`` K, zero total momentum."""
    sig = math.sqrt(KB_EV * temperature / (mass * MVV2E))
    v = np.random.default_rng(seed).normal(0.0, sig, (natoms, 3))
    v -= v.mean(axis=0, keepdims=True)
    return v


def _near_cubic(ncells: int):
    n = max(1, int(math.ceil(ncells ** (1.0 / 3.0))))
    nx = ny = nz = n
    while nz > 1 and nx * ny * (nz - 1) >= ncells:
        nz -= 1
    while ny > 1 and nx * (ny - 1) * nz >= ncells:
        ny -= 1
    return nx, ny, nz


def training_batch(nconfigs: int, nmin: int, nmax: int, species_count: int, seed: int,
                   a_range=(2.8, 4.2), strain: float = 0.03, sigma: float = 0.1) -> List[Structure]:
    """Periodic training configurations (fcc/bcc/hcp, random size, strain, vacancies).

    For each configuration, drawn in order from one ``default_rng(seed)``:
    atom count ``N ~ U{nmin..nmax}``, lattice kind, lattice constant
    ``a ~ U(a_range)``, the N occupied sites (random vacancies in the
    smallest near-cubic supercell holding N sites), a symmetric strain with
    entries ``U(-strain, strain)``, displacements ``N(0, sigma^2)`` and
    species ``U{0..species_count-1}``.
    """
    rng = np.random.default_rng(seed)
    out = []
    kinds = ("fcc", "bcc", "hcp")
    for _ in range(nconfigs):
        n = int(rng.integers(nmin, nmax + 1))
        kind = kinds[int(rng.integers(0, 3))]
        a = float(rng.uniform(*a_range))
        nb = {"fcc": 4, "bcc": 2, "hcp": 2}[kind]
        reps = _near_cubic(-(-n // nb))
        s = lattice_structure(kind, a, reps)
        keep = np.sort(rng.choice(s.natoms, size=n, replace=False))
        eps = rng.uniform(-strain, strain, (3, 3))
        eps = 0.5 * (eps + eps.T)
        F = np.eye(3) + eps
        cell = s.cell @ F
        pos = s.positions[keep] @ F + rng.normal(0.0, sigma, (n, 3))
        types = rng.integers(0, species_count, n).astype(np.int32)
        out.append(Structure(pos, cell, types))
    return out
