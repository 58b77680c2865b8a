"""A potential whose basis was generated from its level runs in the engine (GPU).

mtp_b200.basis builds the tables of a level without a template file; with
seeded random coefficients the result is evaluated by the CUDA engine and by
the C++ FP64 oracle on a displaced crystal, and must agree to the drop-in bar
(1e-10 relative on energy, site energies, forces and virial).
"""

import numpy as np
import pytest

from mtp_b200 import basis as B
from mtp_b200 import synth
from mtp_b200.engine import MTPEngine
from mtp_b200.mtp_file import with_random_coeffs, write_mtp
from oracle.cpu_ref import CpuMTP

pytestmark = pytest.mark.gpu
REL = 1e-10


def _rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(1e-300, np.abs(b).max()))


@pytest.mark.parametrize("level", [12, 16, 20])
def test_generated_level_matches_oracle(tmp_path, level):
    pot = with_random_coeffs(B.template_potential(level, 2, min_dist=2.0, max_dist=5.0), seed=level)
    path = str(tmp_path / f"gen{level}.mtp")
    write_mtp(path, pot)
    s = synth.lattice_structure("bcc", 2.87, (3, 3, 3))
    s.types = (np.arange(s.natoms) % 2).astype(np.int32)
    s.positions = s.positions + np.random.default_rng(level).normal(0.0, 0.05, s.positions.shape)
    nd = synth.build_neighbors(s, pot.max_dist)
    ref = CpuMTP(pot).compute(nd.itypes, nd.rijs, nd.js, nd.jtypes, nd.counts)
    N, n = nd.js.shape
    with MTPEngine(path, N, n) as eng:
        out = eng.compute(nd.itypes, nd.rijs, nd.js, nd.jtypes, nd.counts, eatom=True)
    assert abs(out["energy"] - ref["energy"]) <= REL * abs(ref["energy"])
    assert _rel(out["site_energies"], ref["site_energies"]) <= REL
    assert _rel(out["forces"], ref["forces"]) <= REL
    assert _rel(out["virial"], ref["virial"]) <= REL
