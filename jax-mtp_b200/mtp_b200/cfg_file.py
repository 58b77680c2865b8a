"""MLIP ``.cfg`` configurations (training data): reader and writer.

The format is the one the reference reads with ``read_cfg``
(motep_original_files/old_io/mlip/cfg.py:15-135) and writes with ``write_cfg``
(same file, :200-290).  A file holds blocks::

    BEGIN_CFG
     Size
        2
     Supercell                       (optional: no cell = not periodic)
        10.0 0.0 0.0
         0.0 10.0 0.0
         0.0 0.0 10.0
     AtomData:  id type cartes_x cartes_y cartes_z fx fy fz
                 1    0  0.0 0.0 0.0   0.0 0.0 -4.8
                 2    0  0.0 0.0 0.65  0.0 0.0  4.8
     Energy
        -6.54
     PlusStress:  xx yy zz yz xz xy
        -0.13 -0.13 3.04 0.0 0.0 0.0
     Feature   EFS_by  VASP
    END_CFG

Positions are Cartesian (``cartes_*``) or fractional (``direct_*``);
``SuperCell`` and ``Atomic_data:`` are accepted spellings.  ``PlusStress`` is
the virial in eV; the stress the training loss compares with the model's is
``-PlusStress / V`` in the order xx, yy, zz, yz, xz, xy (cfg.py:131-134).
Extra per-atom columns are kept in ``Configuration.atom_data``.
"""

from __future__ import annotations

import dataclasses
import os
from typing import Dict, List, Optional, Sequence

import numpy as np

__all__ = ["Configuration", "CfgFormatError", "parse_cfg_text", "read_cfg", "format_cfg", "write_cfg"]

VOIGT = ("xx", "yy", "zz", "yz", "xz", "xy")


class CfgFormatError(ValueError):
    """A malformed ``.cfg`` block (the message names the line)."""


@dataclasses.dataclass
class Configuration:
    types: np.ndarray                       # [N] int32 species index
    positions: np.ndarray                   # [N, 3] Cartesian, Angstrom
    cell: Optional[np.ndarray] = None       # [3, 3] rows are lattice vectors; None = no periodic cell
    energy: Optional[float] = None          # eV
    forces: Optional[np.ndarray] = None     # [N, 3] eV/A
    plus_stress: Optional[np.ndarray] = None  # [6] virial (eV), order xx, yy, zz, yz, xz, xy
    features: Dict[str, object] = dataclasses.field(default_factory=dict)
    atom_data: Dict[str, np.ndarray] = dataclasses.field(default_factory=dict)

    @property
    def natoms(self) -> int:
        return int(self.types.shape[0])

    @property
    def volume(self) -> float:
        if self.cell is None:
            raise CfgFormatError("configuration has no Supercell: no volume")
        return float(abs(np.linalg.det(self.cell)))

    @property
    def stress(self) -> Optional[np.ndarray]:
        """Training stress target -PlusStress / V (xx, yy, zz, yz, xz, xy), eV/A^3."""
        if self.plus_stress is None or self.cell is None:
            return None
        return -np.asarray(self.plus_stress, dtype=np.float64) / self.volume


def _num(tok: str, lineno: int, what: str) -> float:
    try:
        return float(tok)
    except ValueError:
        raise CfgFormatError(f"line {lineno}: {what}: '{tok}' is not a number") from None


def parse_cfg_text(text: str) -> List[Configuration]:
    lines = text.splitlines()
    out: List[Configuration] = []
    i = 0
    n = len(lines)

    def nxt(what: str):
        nonlocal i
        while i < n:
            line = lines[i]
            i += 1
            if line.strip():
                return line, i
        raise CfgFormatError(f"end of file while reading {what}")

    while i < n:
        line = lines[i]
        i += 1
        if not line.startswith("BEGIN_CFG"):
            continue
        begin = i
        size = None
        cell = None
        energy = None
        stress = None
        features: Dict[str, object] = {}
        cols: Optional[List[str]] = None
        rows: List[List[str]] = []
        while True:
            if i >= n:
                raise CfgFormatError(f"line {begin}: BEGIN_CFG without END_CFG")
            line = lines[i]
            i += 1
            toks = line.split()
            if not toks:
                continue
            key = toks[0]
            if line.startswith("END_CFG"):
                break
            if key == "Size":
                l2, ln = nxt("Size")
                size = int(_num(l2.split()[0], ln, "Size"))
                if size < 0:
                    raise CfgFormatError(f"line {ln}: negative Size")
            elif key in ("Supercell", "SuperCell"):
                cell = np.zeros((3, 3))
                for r in range(3):
                    l2, ln = nxt("Supercell")
                    vals = l2.split()
                    if len(vals) != 3:
                        raise CfgFormatError(f"line {ln}: a Supercell row needs 3 numbers")
                    cell[r] = [_num(v, ln, "Supercell") for v in vals]
            elif key in ("AtomData:", "Atomic_data:"):
                if size is None:
                    raise CfgFormatError(f"line {i}: AtomData before Size")
                cols = toks[1:]
                for _ in range(size):
                    l2, ln = nxt("AtomData")
                    vals = l2.split()
                    if len(vals) != len(cols):
                        raise CfgFormatError(f"line {ln}: {len(vals)} values for {len(cols)} AtomData columns")
                    rows.append(vals)
            elif key == "Energy":
                l2, ln = nxt("Energy")
                energy = _num(l2.split()[0], ln, "Energy")
            elif key == "PlusStress:":
                keys = toks[1:]
                l2, ln = nxt("PlusStress")
                vals = [_num(v, ln, "PlusStress") for v in l2.split()]
                if len(vals) != len(keys) or sorted(keys) != sorted(VOIGT):
                    raise CfgFormatError(f"line {ln}: PlusStress needs the six components {VOIGT}")
                d = dict(zip(keys, vals))
                stress = np.array([d[k] for k in VOIGT])
            elif key == "Feature":
                if len(toks) >= 3:
                    try:
                        features[toks[1]] = float(toks[2])
                    except ValueError:
                        features[toks[1]] = " ".join(toks[2:])
                elif len(toks) == 2:
                    features[toks[1]] = ""
        if cols is None or size is None:
            raise CfgFormatError(f"line {begin}: configuration without Size and AtomData")
        data = {c: [r[k] for r in rows] for k, c in enumerate(cols)}
        if "type" not in data:
            raise CfgFormatError(f"line {begin}: AtomData has no 'type' column")
        types = np.array([int(v) for v in data["type"]], dtype=np.int32)
        cart = ("cartes_x", "cartes_y", "cartes_z")
        frac = ("direct_x", "direct_y", "direct_z")
        if all(c in data for c in cart):
            pos = np.array([[float(data[c][a]) for c in cart] for a in range(size)]).reshape(size, 3)
        elif all(c in data for c in frac):
            if cell is None:
                raise CfgFormatError(f"line {begin}: direct coordinates without a Supercell")
            pos = np.array([[float(data[c][a]) for c in frac] for a in range(size)]).reshape(size, 3) @ cell
        else:
            raise CfgFormatError(f"line {begin}: AtomData needs cartes_x/y/z or direct_x/y/z")
        forces = None
        if all(c in data for c in ("fx", "fy", "fz")):
            forces = np.array([[float(data[c][a]) for c in ("fx", "fy", "fz")] for a in range(size)]).reshape(size, 3)
        extra = {c: np.array([float(v) for v in data[c]]) for c in cols
                 if c not in ("id", "type", "fx", "fy", "fz") + cart + frac}
        out.append(Configuration(types, pos, cell, energy, forces, stress, features, extra))
    return out


def read_cfg(path: os.PathLike) -> List[Configuration]:
    with open(path) as fh:
        return parse_cfg_text(fh.read())


def format_cfg(configs: Sequence[Configuration]) -> str:
    parts = []
    for c in configs:
        s = ["BEGIN_CFG", " Size", f"    {c.natoms}"]
        if c.cell is not None:
            s.append(" Supercell")
            for r in np.asarray(c.cell):
                s.append("   " + " ".join(f"{v:17.10f}" for v in r))
        head = " AtomData:  id type       cartes_x      cartes_y      cartes_z"
        if c.forces is not None:
            head += "           fx          fy          fz"
        s.append(head)
        for a in range(c.natoms):
            row = f"    {a + 1:10d} {int(c.types[a]):4d} " + " ".join(f"{v:17.10f}" for v in c.positions[a])
            if c.forces is not None:
                row += " " + " ".join(f"{v:17.10f}" for v in c.forces[a])
            s.append(row)
        if c.energy is not None:
            s += [" Energy", f"    {c.energy:.12f}"]
        if c.plus_stress is not None:
            s.append(" PlusStress:  " + "  ".join(f"{k:>10s}" for k in VOIGT))
            s.append("    " + " ".join(f"{v:17.10f}" for v in c.plus_stress))
        for k, v in c.features.items():
            s.append(f" Feature   {k}\t{v}")
        s.append("END_CFG")
        parts.append("\n".join(s) + "\n")
    return "\n".join(parts)


def write_cfg(path: os.PathLike, configs: Sequence[Configuration]) -> None:
    with open(path, "w") as fh:
        fh.write(format_cfg(configs))
