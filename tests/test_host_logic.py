"""Host-side logic of the library, checked without a GPU.

* the C ABI shared library loads and exports every function declared in
  include/mtp_b200.h;
* the C++ .mtp reader agrees with the Python one and rejects malformed files;
* the contraction schedule (lane programs with split/combine passes), run on
  the host, reproduces the oracle's moments and dE/dm exactly in structure
  (FP64 rounding only);
* the periodic ghosts and full lists handed to mtp_compute_positions, cut to
  the cutoff, are the neighbour rows of the direct periodic builder.
"""

import os
import re

import numpy as np
import pytest
import torch

from conftest import REPO, potential_path
from mtp_b200 import _lib, synth
from mtp_b200.engine import parse_info, schedule_emulate
from mtp_b200.mtp_file import format_mtp, read_mtp
from oracle import mtp_oracle as O


def _header_functions():
    text = open(os.path.join(REPO, "include", "mtp_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mtp_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_function():
    L = _lib.lib()
    names = _header_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(L, n), n
        assert n in _lib.SIGNATURES, f"{n} has no ctypes signature"
    assert L.mtp_abi_version() == 1


@pytest.mark.parametrize("name", ["cfg0_L16_S1.mtp", "cfg3_L20_S2.mtp", "cfg2_L24_S3.mtp", "cfg4_L28_S4.mtp"])
def test_cpp_parser_matches_python(name):
    p = read_mtp(potential_path(name))
    info = parse_info(potential_path(name))
    assert info["species_count"] == p.species_count
    assert info["radial_funcs_count"] == p.radial_funcs_count
    assert info["radial_basis_size"] == p.radial_basis_size
    assert info["alpha_moments_count"] == p.alpha_moments_count
    assert info["alpha_index_basic_count"] == p.alpha_index_basic_count
    assert info["alpha_index_times_count"] == p.alpha_index_times_count
    assert info["alpha_scalar_moments"] == p.alpha_scalar_moments
    assert info["max_degree"] == p.max_degree


def test_cpp_parser_rejects_bad_files(tmp_path):
    good = open(potential_path("cfg0_L16_S1.mtp")).read()
    cases = {
        "no_header": good.replace("MTP\n", "", 1),
        "bad_count": good.replace("alpha_index_basic_count = 130", "alpha_index_basic_count = 131"),
        "truncated_radial": good.split("\t\t0-0")[0] + "\t\t0-0\n",
        "bad_moment_ref": good.replace("alpha_moment_mapping = {0,", "alpha_moment_mapping = {9999,"),
        "not_chebyshev": good.replace("RBChebyshev", "RBShapeev"),
    }
    for tag, text in cases.items():
        f = tmp_path / f"{tag}.mtp"
        f.write_text(text)
        with pytest.raises(_lib.MTPError) as ei:
            parse_info(str(f))
        assert ei.value.code == 2, tag   # MTP_E_FORMAT
    # an untrained template (no coefficients) is not a usable potential
    tmpl = re.sub(r"\tradial_coeffs\n(\t\t.*\n)+", "", good)
    f = tmp_path / "template.mtp"
    f.write_text(tmpl)
    with pytest.raises(_lib.MTPError):
        parse_info(str(f))


@pytest.mark.parametrize("name,lanes,width", [("cfg0_L16_S1.mtp", 128, 4), ("cfg0_L16_S1.mtp", 512, 8),
                                              ("cfg3_L20_S2.mtp", 256, 16), ("cfg2_L24_S3.mtp", 256, 4),
                                              ("cfg2_L24_S3.mtp", 512, 8), ("cfg4_L28_S4.mtp", 512, 8)])
def test_schedule_reproduces_tree_and_adjoint(name, lanes, width):
    pot = read_mtp(potential_path(name))
    tab = O.OracleTables.from_potential(pot)
    rng = np.random.default_rng(7)
    basic = rng.normal(size=pot.alpha_index_basic_count)
    m, dm, e = schedule_emulate(potential_path(name), lanes, basic, width)
    # oracle: the same tree on the same basic moments, dE/dm by autograd
    b = torch.tensor(basic, requires_grad=True)
    mm = torch.cat([b, torch.zeros(tab.M - len(basic))])[None]
    for lev in tab.levels:
        i1 = torch.tensor(lev[:, 0]); i2 = torch.tensor(lev[:, 1]); i3 = torch.tensor(lev[:, 3])
        mm = mm.index_add(1, i3, torch.tensor(lev[:, 2], dtype=torch.float64) * mm[:, i1] * mm[:, i2])
    E = (mm[0, torch.tensor(tab.mapping)] * tab.moment_coeffs).sum()
    (gb,) = torch.autograd.grad(E, b)
    scale = np.abs(mm.detach().numpy()).max()
    np.testing.assert_allclose(m, mm[0].detach().numpy(), rtol=1e-12, atol=1e-12 * scale)
    assert abs(e - float(E.detach())) <= 1e-12 * max(1.0, abs(float(E.detach())))
    gscale = np.abs(gb.numpy()).max()
    np.testing.assert_allclose(dm[: len(basic)], gb.numpy(), rtol=1e-11, atol=1e-12 * gscale)


def test_python_writer_output_reads_back_in_cpp(tmp_path):
    p = read_mtp(potential_path("cfg3_L20_S2.mtp"))
    f = tmp_path / "rt.mtp"
    f.write_text(format_mtp(p))
    info = parse_info(str(f))
    assert info["alpha_index_times_count"] == p.alpha_index_times_count


@pytest.mark.parametrize("kind,a,reps", [("bcc", 2.87, (3, 3, 3)), ("fcc", 3.6, (4, 3, 3))])
def test_ghosts_and_lists_give_the_periodic_rows(kind, a, reps):
    s = synth.lattice_structure(kind, a, reps)
    s.positions = s.positions + np.random.default_rng(4).normal(0.0, 0.08, s.positions.shape)
    s.types = np.random.default_rng(5).integers(0, 3, s.natoms).astype(np.int32)
    cutoff, skin = 5.0, 0.3
    x, owner, lists = synth.ghosts_and_lists(s, cutoff + skin)
    N = s.natoms
    assert np.array_equal(owner[:N], np.arange(N)) and owner.min() >= 0 and owner.max() < N
    # every ghost is a lattice translate of its owner
    L = np.diag(s.cell)
    shift = (x - np.mod(s.positions, L)[owner]) / L
    assert np.allclose(shift, np.round(shift), atol=1e-12)
    nd = synth.build_neighbors(s, cutoff)
    for i, c in enumerate(lists):
        d = np.linalg.norm(x[c] - x[i], axis=1)
        assert np.all(d < cutoff + skin) and i not in c
        inside = c[d < cutoff]
        # the same neighbours (owner, distance) as the direct builder's row
        got = sorted(zip(owner[inside].tolist(), np.round(d[d < cutoff], 9).tolist()))
        row = nd.js[i, :nd.counts[i]]
        want = sorted(zip(row.tolist(), np.round(np.linalg.norm(nd.rijs[i, :nd.counts[i]], axis=1), 9).tolist()))
        assert got == want


def test_ghosts_and_lists_reject_small_or_skewed_cells():
    s = synth.lattice_structure("bcc", 2.87, (2, 2, 2))          # 5.74 A edges: not above 5.3 + a margin
    with pytest.raises(ValueError):
        synth.ghosts_and_lists(s, 6.0)
    h = synth.lattice_structure("hcp", 3.0, (3, 3, 3))
    with pytest.raises(ValueError):
        synth.ghosts_and_lists(h, 5.0)


def test_tile_candidates_and_batch_restride():
    """Neighbour-tile candidates of the training autotuner, and a batch restrided
    to a tile keeps every row's real slots (only padding changes)."""
    from mtp_b200.autotune import tile_candidates
    from mtp_b200.train import DeviceBatch
    assert tile_candidates(90) == (96,)
    assert tile_candidates(100) == (104, 112, 128)
    assert tile_candidates(130) == (136, 144, 160)
    assert tile_candidates(64) == (64,)
    pot = read_mtp(potential_path("cfg3_L20_S2.mtp"))
    structs = synth.training_batch(3, 8, 20, pot.species_count, seed=3)
    nds = [synth.build_neighbors(s, pot.max_dist) for s in structs]
    nd, cfg, offs, vols = synth.pack_batch(nds)
    b = DeviceBatch.from_numpy(nd, cfg, vols, device="cpu")
    longest = int(b.counts.max())
    for n in (longest, b.stride + 16):
        r = b.with_stride(n)
        assert r.stride == n
        for i in range(b.natoms):
            c = int(b.counts[i])
            assert torch.equal(r.rijs[i, :c], b.rijs[i, :c])
            assert torch.equal(r.js[i, :c], b.js[i, :c])
            assert torch.equal(r.jtypes[i, :c], b.jtypes[i, :c])
        assert bool((r.jtypes[:, b.stride:] == -1).all()) if n > b.stride else True
    with pytest.raises(ValueError):
        b.with_stride(longest - 1)
