"""Pressure and box relaxation through the pair style's virial (GPU).

The reference's own LAMMPS input relaxes the box with `fix box/relax iso 0.0`
and `minimize` (test_lammps.in:27-28), which reads the pair style's virial;
its README lists the pressure for NPT as an open item (README.md:40, 47)
because the reference hands LAMMPS the stress divided by the volume, with the
wrong sign and Voigt order (jax_backend.py:355-360, pair_jax_mtp.cpp:203-205).
Here the virial is checked against the oracle's energy-volume derivative, and
a box relaxation of the mini LAMMPS driver must end where the oracle's energy
is stationary:

* every component of the LAMMPS virial equals -dE/d(strain) of the C++ FP64
  oracle by central finite differences (homogeneous strain of a config-1
  cell), and the pair style's thermo pressure equals -dE/dV;
* box/relax of a B2 (CsCl-ordered) bcc crystal reaches the oracle's energy
  minimum of E(a) to 1e-4 A.

The relaxed crystal uses a random-coefficient potential (the stated
distributions); such a potential has no short-range repulsion, so only a
symmetric crystal, whose atoms feel no force, has a box minimum to relax to:
a displaced random alloy collapses into the region below min_dist.
"""

import json
import os
import subprocess

import numpy as np
import pytest

from conftest import REPO, potential_path
from mtp_b200 import synth
from mtp_b200.engine import MTPEngine
from mtp_b200.lammps_data import write_data
from mtp_b200.mtp_file import read_mtp
from oracle.cpu_ref import CpuMTP

pytestmark = pytest.mark.gpu
DRIVER = os.path.join(REPO, "jax-mtp_b200", "pair_style", "_build", "mini_lammps")
NKTV2P = 1.6021765e6      # eV/A^3 -> bar (LAMMPS metal)
# cfg1_L16_S2.mtp (level 16, 2 species, the stated random coefficients) has a
# local minimum of the B2 crystal's energy near a = 3.2 A; the MD variant is
# purely repulsive in volume, so it has no box to relax to
RELAX_POT = "cfg1_L16_S2.mtp"


@pytest.fixture(scope="module")
def driver():
    subprocess.run(["make", "-C", os.path.join(REPO, "jax-mtp_b200", "pair_style")], check=True,
                   stdout=subprocess.DEVNULL)
    return DRIVER


def _b2(a, reps=4):
    s = synth.lattice_structure("bcc", a, (reps, reps, reps))
    s.types = (np.arange(s.natoms) % 2).astype(np.int32)     # corner 0, body centre 1
    return s


def _energy(cpu, s, cutoff):
    nd = synth.build_neighbors(s, cutoff)
    return cpu.compute(nd.itypes, nd.rijs, nd.js, nd.jtypes, nd.counts)


def _strained(s, eps):
    F = np.eye(3) + eps
    out = synth.Structure(s.positions @ F.T, s.cell @ F.T, s.types.copy())
    return out


def test_virial_matches_strain_derivative_of_oracle_energy(driver, tmp_path):
    """Config-1 cell (bcc a=2.87 A, 10^3 cells, 50/50 species, sigma 0.05 A)."""
    name = "cfg1md_L16_S2.mtp"
    pot = read_mtp(potential_path(name))
    cpu = CpuMTP(pot)
    s = synth.config1()
    s.positions = s.positions + np.random.default_rng(4).normal(0.0, 0.05, s.positions.shape)
    # one neighbour set with a 0.3 A skin, strained as a whole: slots beyond
    # max_dist drop out in the kernel and the oracle alike
    nd = synth.build_neighbors(s, pot.max_dist + 0.3)
    N, n = nd.js.shape
    with MTPEngine(potential_path(name), N, n) as eng:
        W = eng.compute(nd.itypes, nd.rijs, nd.js, nd.jtypes, nd.counts)["virial"]   # xx yy zz xy xz yz
    h = 1e-5
    comps = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
    for k, (a, b) in enumerate(comps):
        eps = np.zeros((3, 3))
        eps[a, b] += 0.5 * h
        eps[b, a] += 0.5 * h
        Ep = cpu.compute(nd.itypes, nd.rijs @ (np.eye(3) + eps).T, nd.js, nd.jtypes, nd.counts)["energy"]
        Em = cpu.compute(nd.itypes, nd.rijs @ (np.eye(3) - eps).T, nd.js, nd.jtypes, nd.counts)["energy"]
        dE = (Ep - Em) / (2 * h)
        assert abs(W[k] + dE) <= 1e-6 * max(1.0, np.abs(W).max()), (k, W[k], -dE)
    # the pair style's pressure at zero velocities: -dE/dV under isotropic strain
    write_data(str(tmp_path / "d.txt"), s, np.zeros((N, 3)), 2)
    out = subprocess.run([driver, str(tmp_path / "d.txt"), potential_path(name), str(N), "64", "5.0", "55.845",
                          "0.001", "0", "10", "0.3"], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    press = float([l.split() for l in out.stdout.splitlines() if l.startswith("step 0")][0][11])
    V = s.volume
    Ep = cpu.compute(nd.itypes, nd.rijs * (1 + h), nd.js, nd.jtypes, nd.counts)["energy"]
    Em = cpu.compute(nd.itypes, nd.rijs * (1 - h), nd.js, nd.jtypes, nd.counts)["energy"]
    dEdV = (Ep - Em) / (V * ((1 + h) ** 3 - (1 - h) ** 3))
    assert abs(press - (-dEdV * NKTV2P)) <= 1e-6 * abs(dEdV * NKTV2P) + 1e-3, (press, -dEdV * NKTV2P)


def _relax(driver, tmp_path, s, ftol, ptol_bar, max_box=60):
    write_data(str(tmp_path / "in.txt"), s, np.zeros((s.natoms, 3)), 2)
    out_txt = tmp_path / "out.txt"
    out = subprocess.run([driver, str(tmp_path / "in.txt"), potential_path(RELAX_POT), str(s.natoms), "96", "5.0",
                          "55.845", "0.001", str(max_box), "10", "0.3", "fp64", "1", "device", "boxrelax",
                          str(ftol), str(ptol_bar), str(out_txt)], capture_output=True, text=True, timeout=900)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr
    summary = json.loads(out.stdout.strip().splitlines()[-1])
    rows = np.loadtxt(out_txt, skiprows=2)
    L = np.loadtxt(out_txt, skiprows=1, max_rows=1)
    pos = rows[:, 2:5]
    types = rows[:, 1].astype(np.int32) - 1
    return summary, synth.Structure(pos, np.diag(L), types)


def test_box_relax_reaches_oracle_lattice_constant(driver, tmp_path):
    from scipy.optimize import minimize_scalar
    pot = read_mtp(potential_path(RELAX_POT))
    cpu = CpuMTP(pot)
    res = minimize_scalar(lambda a: _energy(cpu, _b2(a, 3), pot.max_dist)["energy"], bracket=(3.1, 3.2, 3.3),
                          tol=1e-10)
    a_ref = float(res.x)
    assert 3.1 < a_ref < 3.3
    summary, out = _relax(driver, tmp_path, _b2(3.2), ftol=1e-8, ptol_bar=1e-3)
    assert summary["converged"]
    a_relaxed = summary["box"][0] / 4
    assert abs(a_relaxed - a_ref) <= 1e-4, (a_relaxed, a_ref)

