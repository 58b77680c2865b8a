"""The benchmark potentials against the oracle at the stated absolute bars (GPU).

The MD benchmarks run two potentials: cfg1md_L16_S2.mtp (level 16, 2 species,
the 2,000-atom bcc pair-style case) and cfg2md_L24_S3.mtp (level 24, 3
species, the 1,048,576-atom fcc mixed-vs-FP64 case).  Here both are evaluated
on cells of their benchmark's lattice, with thermal displacements, against the
C++ FP64 restatement of the reference algorithm (oracle/mtp_cpu.cpp, which the
CPU suite checks against the reference's own numpy code and finite
differences):

* FP64 kernel: <= 1e-10 relative on the energy, every site energy, every force
  component and the virial (the drop-in bar);
* mixed kernel: the absolute bars, not scaled by the size of the forces:
  every site energy within 0.1 meV, the total energy within 0.1 meV per atom,
  every force component within 1 meV/A.

The mixed kernel is checked at every launch shape the autotuner may pick for
it (256 lanes x 2 atoms, 512 lanes x 4 atoms, 256 lanes x 1 atom).
"""

import numpy as np
import pytest

from conftest import potential_path
from mtp_b200 import synth
from mtp_b200.engine import MTPEngine
from mtp_b200.mtp_file import read_mtp
from oracle.cpu_ref import CpuMTP

pytestmark = pytest.mark.gpu

REL = 1e-10
E_SITE_MEV = 0.1     # meV per site energy
E_TOTAL_MEV = 0.1    # meV per atom, total energy
F_MEV = 1.0          # meV/A per force component


def _cell_l24():
    """Level-24 benchmark lattice: fcc a=3.6 A, 8^3 cells = 2,048 atoms, 3 species, sigma 0.08 A."""
    return synth.config2_structure(8)


def _cell_l16():
    """Level-16 pair-style lattice: bcc a=2.87 A, 10^3 cells = 2,000 atoms, 50/50 species, sigma 0.05 A."""
    s = synth.config1()
    s.positions = s.positions + np.random.default_rng(4).normal(0.0, 0.05, s.positions.shape)
    return s


CASES = {"cfg2md_L24_S3.mtp": (_cell_l24, 64), "cfg1md_L16_S2.mtp": (_cell_l16, 64)}
_cache = {}


def _case(name):
    if name not in _cache:
        make, stride = CASES[name]
        pot = read_mtp(potential_path(name))
        s = make()
        nd = synth.build_neighbors(s, pot.max_dist, n_pad=stride)
        ref = CpuMTP(pot).compute(nd.itypes, nd.rijs, nd.js, nd.jtypes, nd.counts)
        _cache[name] = (nd, ref)
    return _cache[name]


def _rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(1e-300, np.abs(b).max()))


@pytest.mark.parametrize("name", sorted(CASES))
def test_benchmark_potential_fp64_matches_oracle(name):
    nd, ref = _case(name)
    N, n = nd.js.shape
    with MTPEngine(potential_path(name), N, n) as eng:
        out = eng.compute(nd.itypes, nd.rijs, nd.js, nd.jtypes, nd.counts, eatom=True)
    assert abs(out["energy"] - ref["energy"]) <= REL * abs(ref["energy"])
    assert _rel(out["site_energies"], ref["site_energies"]) <= REL
    assert _rel(out["forces"], ref["forces"]) <= REL
    assert _rel(out["virial"], ref["virial"]) <= REL


@pytest.mark.parametrize("threads,apb", [(256, 2), (512, 4), (256, 1)])
@pytest.mark.parametrize("name", sorted(CASES))
def test_benchmark_potential_mixed_absolute_bars(name, threads, apb):
    nd, ref = _case(name)
    N, n = nd.js.shape
    with MTPEngine(potential_path(name), N, n, precision="mixed") as eng:
        eng.set_launch(threads, 0, apb)
        out = eng.compute(nd.itypes, nd.rijs, nd.js, nd.jtypes, nd.counts, eatom=True)
        ran = eng.launch()
    # the engine may narrow the lanes where that fits more blocks per SM (level 16)
    assert ran["atoms_per_block"] == apb and ran["threads"] in (threads, 256, 128)
    de_site = np.abs(out["site_energies"] - ref["site_energies"]).max() * 1e3
    de_total = abs(out["energy"] - ref["energy"]) / N * 1e3
    df = np.abs(out["forces"] - ref["forces"]).max() * 1e3
    assert de_site <= E_SITE_MEV, f"site energy error {de_site:.3g} meV"
    assert de_total <= E_TOTAL_MEV, f"total energy error {de_total:.3g} meV/atom"
    assert df <= F_MEV, f"force error {df:.3g} meV/A"
    # the forces are not trivially small: the bar is a real constraint
    assert np.abs(ref["forces"]).max() > 0.05
