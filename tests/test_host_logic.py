"""Host-side logic of the library, checked without a GPU.

* the C ABI shared library loads and exports every function declared in
  include/mtp_b200.h;
* the C++ .mtp reader agrees with the Python one and rejects malformed files;
* the contraction schedule (lane programs with split/combine passes), run on
  the host, reproduces the oracle's moments and dE/dm exactly in structure
  (FP64 rounding only).
"""

import os
import re

import numpy as np
import pytest
import torch

from conftest import REPO, potential_path
from mtp_b200 import _lib
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
