"""Write the plain data file read by the mini LAMMPS driver (pair_style/mini_lammps.cpp).

Format: "natoms ntypes", "Lx Ly Lz", then one line per atom
"tag type x y z vx vy vz" (LAMMPS types are species + 1; orthorhombic box).
"""

from __future__ import annotations

import numpy as np

from .synth import Structure


def write_data(path: str, s: Structure, velocities: np.ndarray, ntypes: int) -> None:
    cell = np.asarray(s.cell)
    if np.abs(cell - np.diag(np.diag(cell))).max() > 0:
        raise ValueError("the mini driver needs an orthorhombic box")
    with open(path, "w") as fh:
        fh.write(f"{s.natoms} {ntypes}\n")
        fh.write(" ".join(f"{x:.17g}" for x in np.diag(cell)) + "\n")
        for i in range(s.natoms):
            x = s.positions[i]
            v = velocities[i]
            fh.write(f"{i + 1} {int(s.types[i]) + 1} {x[0]:.17g} {x[1]:.17g} {x[2]:.17g} "
                     f"{v[0]:.17g} {v[1]:.17g} {v[2]:.17g}\n")
