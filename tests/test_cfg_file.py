"""MLIP .cfg reader/writer (CPU).

Checks the block grammar the reference's read_cfg accepts
(motep_original_files/old_io/mlip/cfg.py:49-135): Cartesian and fractional
coordinates, optional forces and cell, PlusStress in any column order and its
conversion to the training stress -PlusStress / V, features, errors on
malformed blocks, and a write -> read round trip.
"""

import numpy as np
import pytest

from mtp_b200.cfg_file import CfgFormatError, Configuration, format_cfg, parse_cfg_text

TEXT = """
BEGIN_CFG
 Size
    3
 SuperCell
     4.0 0.0 0.0
     0.0 5.0 0.0
     0.5 0.0 6.0
 AtomData:  id type       cartes_x      cartes_y      cartes_z           fx          fy          fz
             1    0       0.000000      0.000000      0.000000     0.10   -0.20    0.30
             2    1       1.000000      2.000000      3.000000    -0.10    0.20   -0.30
             3    1       2.000000      0.500000      1.000000     0.00    0.00    0.00
 Energy
         -11.25
 PlusStress:  xy          xx          yy          zz          yz          xz
         0.6    1.2   -0.3   0.9   0.0   0.15
 Feature   EFS_by	VASP
 Feature   mindist 1.5
END_CFG

BEGIN_CFG
 Size
    2
 Supercell
     3.0 0.0 0.0
     0.0 3.0 0.0
     0.0 0.0 3.0
 Atomic_data:  id type direct_x direct_y direct_z
             1    0   0.0  0.0  0.0
             2    0   0.5  0.5  0.5
END_CFG
"""


def test_parse_blocks():
    a, b = parse_cfg_text(TEXT)
    assert a.natoms == 3 and list(a.types) == [0, 1, 1]
    np.testing.assert_allclose(a.positions[1], [1.0, 2.0, 3.0])
    np.testing.assert_allclose(a.forces[0], [0.1, -0.2, 0.3])
    assert a.energy == -11.25
    np.testing.assert_allclose(a.plus_stress, [1.2, -0.3, 0.9, 0.0, 0.15, 0.6])   # xx yy zz yz xz xy
    assert a.volume == pytest.approx(4.0 * 5.0 * 6.0)
    np.testing.assert_allclose(a.stress, -a.plus_stress / 120.0)
    assert a.features == {"EFS_by": "VASP", "mindist": 1.5}
    # fractional coordinates go through the cell
    np.testing.assert_allclose(b.positions[1], [1.5, 1.5, 1.5])
    assert b.energy is None and b.forces is None and b.stress is None


def test_round_trip():
    rng = np.random.default_rng(3)
    cfgs = [Configuration(rng.integers(0, 3, n).astype(np.int32), rng.normal(size=(n, 3)),
                          np.diag(rng.uniform(3, 6, 3)) + 0.1 * rng.normal(size=(3, 3)), float(rng.normal()),
                          rng.normal(size=(n, 3)), rng.normal(size=6), {"note": "synthetic"})
            for n in (1, 4, 7)]
    back = parse_cfg_text(format_cfg(cfgs))
    assert len(back) == 3
    for x, y in zip(cfgs, back):
        assert np.array_equal(x.types, y.types)
        np.testing.assert_allclose(y.positions, x.positions, atol=1e-9)
        np.testing.assert_allclose(y.cell, x.cell, atol=1e-9)
        np.testing.assert_allclose(y.forces, x.forces, atol=1e-9)
        np.testing.assert_allclose(y.plus_stress, x.plus_stress, atol=1e-9)
        assert y.energy == pytest.approx(x.energy, abs=1e-11)
        assert y.features == {"note": "synthetic"}


@pytest.mark.parametrize("bad,msg", [
    ("BEGIN_CFG\n Size\n 1\n AtomData: id type cartes_x cartes_y cartes_z\n 1 0 0 0\nEND_CFG\n", "values for"),
    ("BEGIN_CFG\n Size\n 1\n AtomData: id type cartes_x cartes_y cartes_z\n 1 0 0 0 0\n", "without END_CFG"),
    ("BEGIN_CFG\n Size\n 1\n AtomData: id type direct_x direct_y direct_z\n 1 0 0 0 0\nEND_CFG\n", "Supercell"),
    ("BEGIN_CFG\n Size\n 1\n AtomData: id type cartes_x cartes_y cartes_z\n 1 0 0 0 0\n"
     " PlusStress: xx yy zz\n 1 2 3\nEND_CFG\n", "six components"),
    ("BEGIN_CFG\n Energy\n abc\nEND_CFG\n", "not a number"),
])
def test_malformed_blocks_raise(bad, msg):
    with pytest.raises(CfgFormatError, match=msg):
        parse_cfg_text(bad)
