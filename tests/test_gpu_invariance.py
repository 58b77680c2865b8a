"""Symmetries of the CUDA evaluation (GPU).

The MTP energy is invariant under rotations of the neighbour vectors and
under relabelling (the order of a row's neighbour slots, the order of the
atoms); forces rotate with the vectors and the virial transforms as
R W R^T.  The FP64 kernel is held to relative 1e-11 (the rounding of
changed summation orders).  The mixed kernel's results differ from the exact
ones by its FP32 rounding, so its bar is four times its own largest relative
difference from the FP64 kernel on the unchanged input.
"""

import numpy as np
import pytest

from conftest import golden_case, potential_path
from mtp_b200.engine import MTPEngine

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-11


def _rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(1e-300, np.abs(b).max()))


def _sym(w):
    """LAMMPS virial order (xx, yy, zz, xy, xz, yz) to a symmetric 3x3 matrix."""
    xx, yy, zz, xy, xz, yz = w
    return np.array([[xx, xy, xz], [xy, yy, yz], [xz, yz, zz]])


def _tolerance(precision, path, N, n, out, it, rij, js, jt, cnt):
    if precision == "fp64":
        return FP64_TOL
    with MTPEngine(path, N, n) as e64:
        ref = e64.compute(it, rij, js, jt, cnt)
    err = max(_rel(out[k], ref[k]) for k in ("energy", "site_energies", "forces", "virial"))
    return FP64_TOL + 4 * err


def _case(tag):
    g = golden_case(tag)
    return (potential_path(str(g["potential"])), g["itypes"], g["rijs"], g["js"].astype(np.int32),
            g["jtypes"].astype(np.int32), g["counts"].astype(np.int32))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("tag", ["bcc54_L16", "fcc32_L24"])
def test_rotation(tag, precision):
    path, it, rij, js, jt, cnt = _case(tag)
    q, r = np.linalg.qr(np.random.default_rng(11).normal(size=(3, 3)))
    R = q @ np.diag(np.sign(np.diag(r)))
    if np.linalg.det(R) < 0:
        R[:, 0] = -R[:, 0]
    N, n = js.shape
    with MTPEngine(path, N, n, precision=precision) as eng:
        a = eng.compute(it, rij, js, jt, cnt)
        b = eng.compute(it, rij @ R.T, js, jt, cnt)
    tol = _tolerance(precision, path, N, n, a, it, rij, js, jt, cnt)
    assert abs(b["energy"] - a["energy"]) <= tol * abs(a["energy"])
    assert _rel(b["site_energies"], a["site_energies"]) <= tol
    assert _rel(b["forces"], a["forces"] @ R.T) <= tol
    assert _rel(_sym(b["virial"]), R @ _sym(a["virial"]) @ R.T) <= tol


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_slot_and_atom_relabelling(precision):
    path, it, rij, js, jt, cnt = _case("fcc32_L24")
    N, n = js.shape
    rng = np.random.default_rng(12)
    # permute the filled slots of every row
    rij2, js2, jt2 = rij.copy(), js.copy(), jt.copy()
    for i in range(N):
        p = rng.permutation(int(cnt[i]))
        rij2[i, :cnt[i]] = rij[i, p]
        js2[i, :cnt[i]] = js[i, p]
        jt2[i, :cnt[i]] = jt[i, p]
    # relabel the atoms: row k of the new system is atom perm[k] of the old one
    perm = rng.permutation(N)
    inv = np.append(np.argsort(perm), N)      # padded slots hold index N
    it3, rij3, cnt3 = it[perm], rij2[perm], cnt[perm]
    jt3 = jt2[perm]
    js3 = inv[js2[perm]].astype(np.int32)
    with MTPEngine(path, N, n, precision=precision) as eng:
        a = eng.compute(it, rij, js, jt, cnt)
        b = eng.compute(it, rij2, js2, jt2, cnt)
        c = eng.compute(it3, rij3, js3, jt3, cnt3)
    tol = _tolerance(precision, path, N, n, a, it, rij, js, jt, cnt)
    for o in (b, c):
        assert abs(o["energy"] - a["energy"]) <= tol * abs(a["energy"])
        assert _rel(o["virial"], a["virial"]) <= tol
    assert _rel(b["site_energies"], a["site_energies"]) <= tol
    assert _rel(b["forces"], a["forces"]) <= tol
    assert _rel(c["site_energies"], a["site_energies"][perm]) <= tol
    assert _rel(c["forces"], a["forces"][perm]) <= tol
