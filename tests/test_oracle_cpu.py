"""The C++/OpenMP CPU restatement (the timed CPU baseline) against the torch oracle."""

import numpy as np
import pytest

from conftest import golden_case, potential_path
from mtp_b200.mtp_file import read_mtp
from oracle import mtp_oracle as O
from oracle.cpu_ref import CpuMTP


@pytest.mark.parametrize("tag", ["cfg0", "bcc54_L16", "small_L20", "fcc32_L24", "small_L28"])
def test_cpu_restatement_matches_oracle(tag):
    g = golden_case(tag)
    pot = read_mtp(potential_path(str(g["potential"])))
    a = CpuMTP(pot).compute(g["itypes"], g["rijs"], g["js"], g["jtypes"], g["counts"], nthreads=2)
    b = O.evaluate(pot, g["itypes"], g["rijs"], g["js"], g["jtypes"], float(g["volume"]))
    assert abs(a["energy"] - b["energy"]) <= 1e-12 * abs(b["energy"])
    np.testing.assert_allclose(a["forces"], b["forces"], rtol=0, atol=1e-12 * np.abs(b["forces"]).max())
    np.testing.assert_allclose(a["virial"], b["virial"], rtol=0, atol=1e-12 * np.abs(b["virial"]).max())
    np.testing.assert_allclose(a["site_energies"], g["site_energies_tables"], rtol=0,
                               atol=1e-12 * np.abs(g["site_energies_tables"]).max())


def test_cpu_restatement_thread_count_independent():
    g = golden_case("cfg0")
    pot = read_mtp(potential_path(str(g["potential"])))
    c = CpuMTP(pot)
    a = c.compute(g["itypes"], g["rijs"], g["js"], g["jtypes"], g["counts"], nthreads=1)
    b = c.compute(g["itypes"], g["rijs"], g["js"], g["jtypes"], g["counts"], nthreads=4)
    assert a["energy"] == b["energy"]
    assert np.array_equal(a["forces"], b["forces"])
