"""Basis generated from the level alone (CPU).

mtp_b200.basis enumerates the reference's scalar contractions of basic moment
tensors (moment_jax.py:116-212) and compiles them into MLIP tables.  The
reference itself checks its enumerated basis against the MLIP template of a
level by value (conversion.py:105-160, "they now agree perfectly"); here the
same check is made against the reference's own data -- its dense-tree basis
(levels 2-24) and the MLIP templates' basis (levels 2-28, 26 and 28 with the
templates' limits mu <= 5, nu <= 10) -- as sets of values on the reference's
test vectors, both ways, and against the tables of two benchmark potentials
(levels 16 and 20) on random neighbours.  The
compiled tables must reproduce the dense tensor contractions, and a generated
potential must load in the C++ parser and run through the schedule emulator.
"""

import os

import numpy as np
import pytest

from conftest import GOLDEN, potential_path
from mtp_b200 import basis as B
from mtp_b200.engine import parse_info, schedule_emulate
from mtp_b200.mtp_file import read_mtp, with_random_coeffs, write_mtp

TEMPLATES = {16: "cfg0_L16_S1.mtp", 20: "cfg3_L20_S2.mtp"}
LIMITS = {}


def _unmatched(a, b, rtol=1e-8):
    """How many values of a have no partner in b (each partner used once)."""
    free = np.ones(len(b), bool)
    miss = 0
    for x in a:
        hit = np.flatnonzero(free & (np.abs(b - x) <= rtol * abs(x)))
        if len(hit):
            free[hit[0]] = False
        else:
            miss += 1
    return miss


@pytest.mark.parametrize("level", list(range(2, 30, 2)))
def test_generated_basis_equals_the_reference_basis(level):
    """known_answer_basis.npz (made by tests/golden/make_golden.py from the
    reference's own code at its TEST_R_UNITS / TEST_RB_VALUES) holds, per
    level, the reference's dense-tree basis (levels 2-24, from its precomputed
    contraction lists) and the MLIP template's basis (levels 2-28).  The
    generated basis must equal both as sets of values (levels 26 and 28 with
    the templates' limits mu <= 5, nu <= 10)."""
    kat = np.load(os.path.join(GOLDEN, "known_answer_basis.npz"))
    u, rb = kat["test_r_units"], kat["test_rb_values"]
    tables = B.build_basis(level, **({} if level < 26 else dict(mu_max=5, nu_max=10)))
    ours = B.table_values(tables, u, rb)
    for kind in ("tree", "mlip"):
        key = f"L{level}_{kind}_basis"
        if key in kat.files:
            ref = kat[key]
            assert len(ref) == len(ours), key
            assert _unmatched(ref, ours) == 0 and _unmatched(ours, ref) == 0, key


@pytest.mark.parametrize("level", [16, 20])
def test_generated_basis_equals_the_template_basis(level):
    pot = read_mtp(potential_path(TEMPLATES[level]))
    tables = B.build_basis(level, **LIMITS.get(level, {}))
    assert len(tables.mapping) == pot.alpha_scalar_moments
    assert len(tables.basic) == pot.alpha_index_basic_count
    for seed in (3, 41):
        u, rb = B.test_inputs(tables.radial_funcs_count, seed=seed, neighbours=9)
        ours = B.table_values(tables, u, rb)
        theirs = B.mlip_values(pot, u, rb)
        assert _unmatched(theirs, ours) == 0 and _unmatched(ours, theirs) == 0


def test_level_28_without_the_template_limits_adds_ten_functions():
    # mu up to 6 and nu up to 12 (the level's own limits) add 10 functions,
    # every one with mu = 6 or nu >= 11
    assert len(B.enumerate_scalars(28)) == 2455


@pytest.mark.parametrize("level", [8, 12, 16, 20])
def test_tables_reproduce_the_dense_contractions(level):
    tables = B.build_basis(level)
    u, rb = B.test_inputs(tables.radial_funcs_count, seed=5, neighbours=8)
    ev = B.DenseEval(u, rb)
    dense = np.array([float(ev.value(s)) for s in tables.scalars])
    got = B.table_values(tables, u, rb)
    np.testing.assert_allclose(got, dense, rtol=1e-12, atol=1e-12 * np.abs(dense).max())
    assert tables.times[:, 2].max() <= B.MAX_MULT


@pytest.mark.parametrize("level,lanes,width", [(16, 256, 8), (20, 512, 16)])
def test_generated_potential_loads_and_runs_in_the_schedule(tmp_path, level, lanes, width):
    pot = with_random_coeffs(B.template_potential(level, 2), seed=9)
    path = tmp_path / f"gen{level}.mtp"
    write_mtp(str(path), pot)
    info = parse_info(str(path))
    assert info["alpha_scalar_moments"] == pot.alpha_scalar_moments
    rng = np.random.default_rng(2)
    basic = rng.normal(size=pot.alpha_index_basic_count)
    m, dm, e = schedule_emulate(str(path), lanes, basic, width)
    # the same tables evaluated directly
    ref = np.zeros(pot.alpha_moments_count)
    ref[: len(basic)] = basic
    for i1, i2, mult, i3 in pot.alpha_index_times:
        ref[i3] += mult * ref[i1] * ref[i2]
    np.testing.assert_allclose(m, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    e_ref = float(np.dot(pot.moment_coeffs, ref[pot.alpha_moment_mapping]))
    assert abs(e - e_ref) <= 1e-12 * max(1.0, abs(e_ref))


def test_coefficients_move_between_bases():
    """The level-16 benchmark potential's coefficients, remapped onto the
    generated level-16 basis (BasisConverter's matching by value), give the
    same potential: energies and forces of the C++ FP64 oracle agree."""
    from mtp_b200 import synth
    from oracle.cpu_ref import CpuMTP
    src = read_mtp(potential_path("cfg1md_L16_S2.mtp"))
    dst = B.template_potential(16, src.species_count, src.radial_basis_size, src.min_dist, src.max_dist)
    dst.radial_coeffs = np.array(src.radial_coeffs, copy=True)
    dst.species_coeffs = np.array(src.species_coeffs, copy=True)
    dst.scaling = src.scaling
    dst.moment_coeffs = B.remap_moment_coeffs(src, dst)
    s = synth.lattice_structure("bcc", 2.87, (3, 3, 3))
    s.types = (np.arange(s.natoms) % 2).astype(np.int32)
    s.positions = s.positions + np.random.default_rng(5).normal(0.0, 0.05, s.positions.shape)
    nd = synth.build_neighbors(s, src.max_dist)
    a = CpuMTP(src).compute(nd.itypes, nd.rijs, nd.js, nd.jtypes, nd.counts)
    b = CpuMTP(dst).compute(nd.itypes, nd.rijs, nd.js, nd.jtypes, nd.counts)
    assert abs(a["energy"] - b["energy"]) <= 1e-10 * abs(a["energy"])
    assert np.abs(a["forces"] - b["forces"]).max() <= 1e-10 * np.abs(a["forces"]).max()
