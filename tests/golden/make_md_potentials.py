"""Write the MD variants of the benchmark potentials (no reference checkout needed).

    python tests/golden/make_md_potentials.py

The random coefficient distributions of the static workloads (radial
N(0, 0.1^2), moment N(0, 0.01^2)) give forces of 10^3-10^4 eV/A on the
lattices of the MD workloads, and a random MTP has no short-range repulsion,
so atoms meet below min_dist where the Chebyshev expansion diverges.  The MD
variants are still plain MTPs in the same basis:

* radial function mu = 0 of every species pair holds the Chebyshev fit of
  p(d) = A exp(-b (d - min_dist)), and the coefficient of the scalar basis
  function m[0] = sum_j f_0(d_j) is 1, so the energy contains the purely
  repulsive pair term (max_dist - d)^2 p(d), PAIR_ENERGY eV at the lattice's
  nearest-neighbour distance; at fixed volume it holds the crystal together
  (as soft spheres do) and keeps atoms apart;
* every other moment coefficient is theta_a = z_a / s_a * scale, z_a ~ N(0, 1)
  (default_rng(seed + 100)), s_a the RMS of basis function a over a thermal
  sample of the lattice, `scale` giving an RMS many-body force of
  MANYBODY_RMS_FORCE on that sample;
* the other radial functions keep their N(0, 0.1^2) draws.
"""

from __future__ import annotations

import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [REPO, os.path.join(REPO, "jax-mtp_b200")]

from mtp_b200 import synth  # noqa: E402
from mtp_b200.mtp_file import read_mtp, write_mtp  # noqa: E402
from oracle import mtp_oracle as O  # noqa: E402

MANYBODY_RMS_FORCE = 0.1    # eV/A
PAIR_ENERGY = 0.3           # eV at the nearest-neighbour distance
PAIR_DECAY = 2.5            # 1/A

# (source potential, output name, lattice, a, nearest-neighbour distance, species, seed)
VARIANTS = [
    ("cfg1_L16_S2.mtp", "cfg1md_L16_S2.mtp", "bcc", 2.87, 2.87 * np.sqrt(3) / 2, 2, 2),
    ("cfg2_L24_S3.mtp", "cfg2md_L24_S3.mtp", "fcc", 3.6, 3.6 / np.sqrt(2), 3, 5),
]


def pair_coefficients(rmin, rmax, K, d0):
    """Chebyshev coefficients of p(d) = A exp(-b (d - rmin)) with the pair
    energy (rmax - d)^2 p(d) equal to PAIR_ENERGY at d0."""
    b = PAIR_DECAY
    A = PAIR_ENERGY / ((rmax - d0) ** 2 * np.exp(-b * (d0 - rmin)))
    xs = np.cos(np.pi * (np.arange(64) + 0.5) / 64)
    ds = 0.5 * (xs * (rmax - rmin) + (rmax + rmin))
    p = A * np.exp(-b * (ds - rmin))
    T = np.polynomial.chebyshev.chebvander(xs, K - 1)
    coef, *_ = np.linalg.lstsq(T, p, rcond=None)
    return coef


def main():
    for src, dst, kind, a, d0, S, seed in VARIANTS:
        pot = read_mtp(os.path.join(HERE, "potentials", src))
        pc = pair_coefficients(pot.min_dist, pot.max_dist, pot.radial_basis_size, d0)
        pot.radial_coeffs[:, :, 0, :] = pc[None, None, :]
        s = synth.lattice_structure(kind, a, (3, 3, 3))
        rng = np.random.default_rng(seed + 200)
        s.positions = s.positions + rng.normal(0.0, 0.08, s.positions.shape)
        s.types = rng.integers(0, S, s.natoms).astype(np.int32)
        nd = synth.build_neighbors(s, pot.max_dist)
        tab = O.OracleTables.from_potential(pot)
        rij = torch.tensor(nd.rijs)
        d, valid, f, safe = O.radial_values(tab, rij, torch.tensor(nd.itypes, dtype=torch.int64),
                                            torch.tensor(nd.jtypes, dtype=torch.int64))
        m = O.moments_from_tables(tab, safe / d[..., None], f)
        basis = m[:, torch.tensor(tab.mapping)].numpy()
        s_a = np.sqrt((basis ** 2).mean(axis=0))
        s_a[s_a == 0] = 1.0
        z = np.random.default_rng(seed + 100).normal(size=pot.alpha_scalar_moments)
        pair_slot = int(np.nonzero(np.asarray(pot.alpha_moment_mapping) == 0)[0][0])
        pot.moment_coeffs = z / s_a
        pot.moment_coeffs[pair_slot] = 0.0
        r = O.evaluate(pot, nd.itypes, nd.rijs, nd.js, nd.jtypes, nd.volume)
        rms = float(np.sqrt((r["forces"] ** 2).sum(1).mean()))
        pot.moment_coeffs = pot.moment_coeffs * (MANYBODY_RMS_FORCE / rms)
        pot.moment_coeffs[pair_slot] = 1.0
        r = O.evaluate(pot, nd.itypes, nd.rijs, nd.js, nd.jtypes, nd.volume)
        write_mtp(os.path.join(HERE, "potentials", dst), pot)
        print(dst, "rms |F| = %.3f eV/A, max |F| = %.3f, E/atom = %.3f eV" %
              (np.sqrt((r["forces"] ** 2).sum(1).mean()), np.abs(r["forces"]).max(), r["energy"] / s.natoms))


if __name__ == "__main__":
    main()
