"""pair_style jax/mtp driven by the mini LAMMPS host driver (GPU).

The whole host call path of the reference's MD configuration: local + ghost
atoms, a full neighbour list with a skin, ghost -> owner mapping by tag,
packing into the flat rows, mtp_compute through the C ABI, force and virial
accumulation, velocity Verlet.  Checks the step-0 energy against the FP64
oracle on the same structure and the NVE energy drift.
"""

import json
import os
import subprocess

import numpy as np
import pytest

from conftest import REPO, potential_path
from mtp_b200 import synth
from mtp_b200.lammps_data import write_data
from mtp_b200.mtp_file import read_mtp
from oracle.cpu_ref import CpuMTP

pytestmark = pytest.mark.gpu
DRIVER = os.path.join(REPO, "jax-mtp_b200", "pair_style", "_build", "mini_lammps")


@pytest.fixture(scope="module")
def driver():
    subprocess.run(["make", "-C", os.path.join(REPO, "jax-mtp_b200", "pair_style")], check=True,
                   stdout=subprocess.DEVNULL)
    return DRIVER


def _run(driver, tmp_path, s, v, pot_name, steps, precision="fp64", thermo=10, rows="device"):
    data = tmp_path / "data.txt"
    write_data(str(data), s, v, 2)
    out = subprocess.run([driver, str(data), potential_path(pot_name), str(s.natoms), "64", "5.0", "55.845",
                          "0.001", str(steps), "10", "0.3", precision, str(thermo), rows],
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    lines = out.stdout.strip().splitlines()
    thermo_lines = [l.split() for l in lines if l.startswith("step")]
    return thermo_lines, json.loads(lines[-1])


def test_pair_style_energy_matches_oracle(driver, tmp_path):
    s = synth.lattice_structure("bcc", 2.87, (6, 6, 6))
    s.positions += np.random.default_rng(2).normal(0, 0.05, s.positions.shape)
    s.types = np.random.default_rng(3).integers(0, 2, s.natoms).astype(np.int32)
    v = np.zeros((s.natoms, 3))
    th, summ = _run(driver, tmp_path, s, v, "cfg1md_L16_S2.mtp", 1)
    pot = read_mtp(potential_path("cfg1md_L16_S2.mtp"))
    nd = synth.build_neighbors(s, 5.0)
    ref = CpuMTP(pot).compute(nd.itypes, nd.rijs, nd.js, nd.jtypes, nd.counts)
    e0 = float(th[0][3])
    assert abs(e0 - ref["energy"]) <= 1e-10 * abs(ref["energy"])


def test_pair_style_nve_config1(driver, tmp_path):
    """Config 1 geometry: bcc a=2.87, 10^3 cells (2000 atoms), 50/50 species, 300 K, dt 1 fs."""
    s = synth.config1()
    v = synth.maxwell_boltzmann(s.natoms, 300.0, 55.845, seed=4)
    th, summ = _run(driver, tmp_path, s, v, "cfg1md_L16_S2.mtp", 200, thermo=50)
    assert summ["pair_calls"] == 201
    assert abs(summ["energy_drift_eV_per_atom"]) < 1e-4
    th2, summ2 = _run(driver, tmp_path, s, v, "cfg1md_L16_S2.mtp", 200, precision="mixed", thermo=50)
    # mixed vs FP64 potential energy at step 0 (meV/atom)
    de = abs(float(th2[0][1]) - float(th[0][1])) / s.natoms * 1e3
    assert de < 0.1, de


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_pair_style_device_rows_match_host_rows(driver, tmp_path, precision):
    """rows device (positions + list to the GPU) and rows host (r_ij packed on
    the host) give the same trajectory, thermo line for thermo line."""
    s = synth.lattice_structure("bcc", 2.87, (5, 5, 5))
    s.positions += np.random.default_rng(5).normal(0, 0.05, s.positions.shape)
    s.types = np.random.default_rng(6).integers(0, 2, s.natoms).astype(np.int32)
    v = np.random.default_rng(7).normal(0, 0.02, (s.natoms, 3))
    dev, _ = _run(driver, tmp_path, s, v, "cfg1md_L16_S2.mtp", 30, precision, 5, "device")
    host, _ = _run(driver, tmp_path, s, v, "cfg1md_L16_S2.mtp", 30, precision, 5, "host")
    assert len(dev) == len(host) == 7
    assert dev == host
