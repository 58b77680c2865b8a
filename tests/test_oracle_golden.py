"""The FP64 oracle against the reference's own known-answer vectors and fixtures.

The fixtures were produced by tests/golden/make_golden.py from the reference's
numpy modules (MLIPMomentBasis.calculate, the dense tensordot tree with
BasisConverter's coefficient remap, and finite differences of the reference
energy).  This pins the oracle before it is used to check the CUDA kernels.
"""

import numpy as np
import pytest
import torch

from conftest import GOLDEN, golden_case, potential_path
from mtp_b200.mtp_file import read_mtp
from oracle import mtp_oracle as O

CASES = ["cfg0", "bcc54_L16", "small_L20", "fcc32_L24", "small_L28"]


@pytest.mark.parametrize("level", list(range(2, 30, 2)))
def test_known_answer_basis(level):
    """Moments from the tables at TEST_RS equal the reference's MLIPMomentBasis values."""
    import os
    kat = np.load(os.path.join(GOLDEN, "known_answer_basis.npz"))
    ref_dir = os.path.join(GOLDEN, "potentials")
    # tables of the level come from the benchmark potential files where present,
    # else from the known-answer npz alone (levels without a benchmark potential
    # are checked through the dense tree below)
    u = torch.tensor(kat["test_r_units"])[None]          # [1, 4, 3]
    rb = torch.tensor(kat["test_rb_values"])              # [10, 4]
    name = {16: "cfg0_L16_S1.mtp", 20: "cfg3_L20_S2.mtp", 24: "cfg2_L24_S3.mtp", 28: "cfg4_L28_S4.mtp"}.get(level)
    want = kat[f"L{level}_mlip_basis"]
    if f"L{level}_tree_basis" in kat.files:
        # the reference's dense tree agrees with the MLIP tables (remap permutation)
        tree = kat[f"L{level}_tree_basis"]
        perm = kat[f"L{level}_tree_coeff_index"]
        np.testing.assert_allclose(tree, want[perm], rtol=1e-8, atol=0)
    if name is None:
        return
    pot = read_mtp(os.path.join(ref_dir, name))
    tab = O.OracleTables.from_potential(pot)
    f = rb[: tab.R].T[None]                                  # [1, 4, R]
    m = O.moments_from_tables(tab, u, f)
    got = m[0, torch.tensor(tab.mapping)].numpy()
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12 * np.abs(want).max())


@pytest.mark.parametrize("tag", CASES)
def test_oracle_site_energies_match_reference(tag):
    g = golden_case(tag)
    pot = read_mtp(potential_path(str(g["potential"])))
    r = O.evaluate(pot, g["itypes"], g["rijs"], g["js"], g["jtypes"], float(g["volume"]))
    ref = g["site_energies_tables"]
    scale = np.abs(ref).max()
    np.testing.assert_allclose(r["site_energies"], ref, rtol=0, atol=1e-12 * scale)
    if g["site_energies_tree"].size:
        np.testing.assert_allclose(r["site_energies"], g["site_energies_tree"], rtol=0, atol=1e-11 * scale)


@pytest.mark.parametrize("tag", CASES)
def test_oracle_forces_virial_match_finite_differences(tag):
    g = golden_case(tag)
    pot = read_mtp(potential_path(str(g["potential"])))
    r = O.evaluate(pot, g["itypes"], g["rijs"], g["js"], g["jtypes"], float(g["volume"]))
    F = r["forces"][g["fd_atoms"]]
    fscale = max(1.0, np.abs(r["forces"]).max())
    np.testing.assert_allclose(F, g["fd_forces"], rtol=0, atol=2e-6 * fscale)
    wscale = max(1.0, np.abs(r["virial"]).max())
    np.testing.assert_allclose(r["virial"], g["fd_virial"], rtol=0, atol=2e-6 * wscale)
    # the reference's stress is +sym(sum r g)/V in order xx,yy,zz,yz,xz,xy
    W = r["virial"]
    sig = -np.array([W[0], W[1], W[2], W[5], W[4], W[3]]) / float(g["volume"])
    np.testing.assert_allclose(r["stress"], sig, rtol=1e-12, atol=1e-14)


def test_training_loss_gradient_matches_finite_differences():
    """Loss gradient (double backward through forces) against central differences."""
    from mtp_b200 import synth
    pot = read_mtp(potential_path("cfg3_L20_S2.mtp"))
    tab = O.OracleTables.from_potential(pot)
    structs = synth.training_batch(2, 8, 12, 2, seed=21)
    nds = [synth.build_neighbors(s, pot.max_dist) for s in structs]
    nd, cfg, offs, vols = synth.pack_batch(nds)
    batch = (nd.itypes, nd.rijs, nd.js, nd.jtypes, cfg, len(structs), vols)
    rng = np.random.default_rng(0)
    targets = (rng.normal(size=2), rng.normal(size=(nd.natoms, 3)), rng.normal(size=(2, 6)) * 1e-2)
    params = {"species": pot.species_coeffs, "radial": pot.radial_coeffs, "basis": pot.moment_coeffs}
    L0, grads = O.loss_and_grad(tab, params, batch, targets)
    h = 1e-6
    for key, idx in [("basis", (3,)), ("basis", (40,)), ("radial", (1, 0, 2, 5)), ("radial", (0, 1, 0, 0)),
                     ("species", (1,))]:
        p1 = {k: np.array(v, dtype=np.float64) for k, v in params.items()}
        p1[key][idx] += h
        Lp, _ = O.loss_and_grad(tab, p1, batch, targets)
        p1[key][idx] -= 2 * h
        Lm, _ = O.loss_and_grad(tab, p1, batch, targets)
        fd = (Lp - Lm) / (2 * h)
        assert abs(fd - grads[key][idx]) <= 1e-6 * max(1.0, abs(fd)), (key, idx, fd, grads[key][idx])
