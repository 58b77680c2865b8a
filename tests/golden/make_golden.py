"""Generate the golden fixtures under tests/golden from the reference's own code.

Run with the path of a reference checkout (read-only is fine), given as the
first argument or in ``MTP_REFERENCE``:

    python tests/golden/make_golden.py <reference checkout>

What it does:

1. Copies the reference's numpy-only modules (``motep_original_files/{mtp,
   data}.py`` and ``jax_engine/{moment_jax,conversion,utils}.py`` with the
   precomputed moment JSON files) to a temporary directory.  They must be
   importable from a writable place because ``MomentBasis`` always writes its
   JSON back next to itself (moment_jax.py:159-167).  They are imported
   unmodified.
2. Known-answer basis vectors: for every untrained template level 2..24 the
   reference's ``MLIPMomentBasis.calculate`` (conversion.py:39-84) at the
   fixed ``TEST_R_UNITS`` / ``TEST_RB_VALUES`` (utils.py:3-13), plus the
   reference's own consistency check ``BasisConverter.remap_mlip_moment_coeffs``
   (conversion.py:112-168), which must find every MLIP basis function in the
   dense tensordot tree at rtol 1e-8.  Level 26/28 cannot be enumerated by
   the reference (moment_jax.py:44-46 returns None), so for those only the
   MLIP-table values are stored.
3. Benchmark potentials: each configuration's template tables with seeded
   coefficients, written with this repository's ``.mtp`` writer and read
   back with the reference's ``read_mtp`` (format interoperability).
4. Physical golden values for small structures: per-site energies through
   (a) the reference's MLIP-table route and (b) the reference's dense tree
   with ``BasisConverter``'s remapped coefficients; central finite-difference
   forces of the (a) energy on a few atoms, and a finite-difference virial
   under homogeneous strain.  The radial part (Chebyshev basis times the
   smooth cutoff, jax_backend.py:83-95 and 108-160) lives in the JAX module,
   which cannot be imported here (no JAX), so it is restated below in numpy.
"""

from __future__ import annotations

import os
import shutil
import sys
import tempfile
import warnings

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MTP_REFERENCE")
if not REF:
    sys.exit("usage: make_golden.py <reference checkout>  (or set MTP_REFERENCE)")
sys.path.insert(0, os.path.join(REPO, "jax-mtp_b200"))

from mtp_b200 import synth  # noqa: E402
from mtp_b200.mtp_file import read_mtp as my_read_mtp, with_random_coeffs, write_mtp  # noqa: E402

# Benchmark potentials: (name, template level, species, radial funcs (None = template),
# min_dist, max_dist, coefficient seed).  The template's radial_funcs_count is used
# where the configuration asked for fewer than the basis indexes.
POTENTIALS = [
    ("cfg0_L16_S1", 16, 1, None, 2.0, 5.0, 0),
    ("cfg1_L16_S2", 16, 2, None, 2.0, 5.0, 2),
    ("cfg2_L24_S3", 24, 3, None, 2.0, 5.0, 5),
    ("cfg3_L20_S2", 20, 2, None, 2.0, 5.0, 6),
    ("cfg3label_L20_S2", 20, 2, None, 2.0, 5.0, 7),
    ("cfg4_L28_S4", 28, 4, None, 2.0, 5.5, 8),
]


def _import_reference(tmp: str):
    src = os.path.join(REF, "motep_original_files")
    dst = os.path.join(tmp, "motep_original_files")
    os.makedirs(os.path.join(dst, "jax_engine"))
    for f in ("mtp.py", "data.py"):
        shutil.copy(os.path.join(src, f), dst)
    for f in ("__init__.py", "moment_jax.py", "conversion.py", "utils.py"):
        shutil.copy(os.path.join(src, "jax_engine", f), os.path.join(dst, "jax_engine"))
    shutil.copytree(os.path.join(src, "jax_engine", "precomputed_moments"),
                    os.path.join(dst, "jax_engine", "precomputed_moments"))
    sys.path.insert(0, tmp)
    import motep_original_files.mtp as rmtp
    import motep_original_files.jax_engine.conversion as rconv
    import motep_original_files.jax_engine.moment_jax as rmom
    import motep_original_files.jax_engine.utils as rutil
    return rmtp, rconv, rmom, rutil


def _radial_numpy(pot, d, itype, jtypes):
    """f[mu, j] = scaling * (Rc - d)^2 * sum_n c[it, jt, mu, n] T_n(x)  (jax_backend.py:83-95, 108-160)."""
    valid = (jtypes >= 0) & (d < pot.max_dist)
    x = (2.0 * d - (pot.min_dist + pot.max_dist)) / (pot.max_dist - pot.min_dist)
    K = pot.radial_basis_size
    T = [np.ones_like(x), x]
    for _ in range(K - 2):
        T.append(2.0 * x * T[-1] - T[-2])
    T = np.stack(T[:K], axis=1)                                   # [n, K]
    c = pot.radial_coeffs[itype, np.maximum(jtypes, 0)]           # [n, R, K]
    base = np.einsum("jmk,jk->mj", c, T)
    smooth = np.where(valid, (pot.max_dist - d) ** 2, 0.0)
    return pot.scaling * smooth[None, :] * base, valid


def _site_energies_ref(pot, nd, mlip, conv_route):
    """Per-site energies via the reference's MLIP-table basis and (optionally) its dense tree."""
    rconv, mb, remapped = conv_route if conv_route else (None, None, None)
    E_tab, E_tree = [], []
    for i in range(nd.natoms):
        c = nd.counts[i]
        r = nd.rijs[i, :c]
        jt = nd.jtypes[i, :c]
        d = np.linalg.norm(r, axis=1)
        rb, valid = _radial_numpy(pot, d, nd.itypes[i], jt)
        r, d, rb = r[valid], d[valid], rb[:, valid]
        u = r / d[:, None]
        basis = mlip.calculate(u, rb)
        E_tab.append(pot.species_coeffs[nd.itypes[i]] + pot.moment_coeffs @ basis)
        if rconv is not None:
            b2 = np.array(rconv._calc_moment_basis(u, rb, mb.basic_moments, mb.pair_contractions,
                                                   mb.scalar_contractions), dtype=np.float64)
            E_tree.append(pot.species_coeffs[nd.itypes[i]] + remapped @ b2)
    return np.array(E_tab), (np.array(E_tree) if E_tree else None)


def _total_energy(pot, s, cutoff, n_pad, mlip):
    nd = synth.build_neighbors(s, cutoff, n_pad=n_pad)
    e, _ = _site_energies_ref(pot, nd, mlip, None)
    return e.sum()


def main():
    out_pot = os.path.join(HERE, "potentials")
    os.makedirs(out_pot, exist_ok=True)
    tmp = tempfile.mkdtemp(prefix="mtp_ref_")
    rmtp, rconv, rmom, rutil = _import_reference(tmp)
    tdir = os.path.join(REF, "training", "untrained_mtps")

    # --- 2. known-answer basis vectors at TEST_RS --------------------------------
    kat = {}
    for L in range(2, 30, 2):
        d = rmtp.read_mtp(os.path.join(tdir, f"{L:02d}.mtp"))
        mlip = rconv.MLIPMomentBasis(d)
        R = int(d.alpha_index_basic[:, 0].max()) + 1
        vals = mlip.calculate(rutil.TEST_R_UNITS, rutil.TEST_RB_VALUES[:R])
        kat[f"L{L}_mlip_basis"] = vals
        if L <= 24:
            d.moment_coeffs = np.arange(1, d.alpha_scalar_moments + 1, dtype=np.float64)
            mb = rmom.MomentBasis(L)
            mb.init_moment_mappings()
            bc = rconv.BasisConverter(mb)
            with warnings.catch_warnings():
                warnings.simplefilter("error")
                bc.remap_mlip_moment_coeffs(d)       # raises if the two bases disagree
            tree = np.array(rconv._calc_moment_basis(rutil.TEST_R_UNITS, rutil.TEST_RB_VALUES[:R],
                                                     mb.basic_moments, mb.pair_contractions,
                                                     mb.scalar_contractions), dtype=np.float64)
            kat[f"L{L}_tree_basis"] = tree
            kat[f"L{L}_tree_coeff_index"] = bc.remapped_coeffs.astype(np.int64) - 1
    kat["test_r_units"] = rutil.TEST_R_UNITS
    kat["test_rb_values"] = rutil.TEST_RB_VALUES
    np.savez_compressed(os.path.join(HERE, "known_answer_basis.npz"), **kat)
    print("known-answer basis vectors: levels 2..28")

    # --- 3. benchmark potentials ---------------------------------------------------
    pots = {}
    for name, L, S, R, rmin, rmax, seed in POTENTIALS:
        tmpl = my_read_mtp(os.path.join(tdir, f"{L:02d}.mtp"), require_coeffs=False)
        pot = with_random_coeffs(tmpl, seed, species_count=S, radial_funcs_count=R,
                                 min_dist=rmin, max_dist=rmax)
        path = os.path.join(out_pot, f"{name}.mtp")
        write_mtp(path, pot)
        back = rmtp.read_mtp(path)                   # the reference reader accepts the file
        assert np.array_equal(back.radial_coeffs, pot.radial_coeffs)
        assert np.array_equal(back.alpha_index_times, pot.alpha_index_times)
        assert np.array_equal(back.moment_coeffs, pot.moment_coeffs)
        pots[name] = (pot, back)
        print("potential", name)

    # --- 4. physical golden values -------------------------------------------------
    cases = []
    # configuration 0 itself: 256 atoms fcc a=4.05, level 16, one species
    cases.append(("cfg0", "cfg0_L16_S1", synth.config0(), 5.0, 16, [0, 17, 101], True))
    # small two-species bcc cell, level 16
    s1 = synth.lattice_structure("bcc", 2.87, (3, 3, 3))
    s1.positions += np.random.default_rng(11).normal(0, 0.05, s1.positions.shape)
    s1.types = np.random.default_rng(12).integers(0, 2, s1.natoms).astype(np.int32)
    cases.append(("bcc54_L16", "cfg1_L16_S2", s1, 5.0, 16, [0, 7], True))
    # small cell with multiple periodic images, level 20, two species
    s3 = synth.training_batch(1, 24, 24, 2, seed=13)[0]
    cases.append(("small_L20", "cfg3_L20_S2", s3, 5.0, 20, [0, 5], True))
    # fcc a=3.6 2x2x2 (32 atoms), level 24, three species
    s2 = synth.lattice_structure("fcc", 3.6, (2, 2, 2))
    s2.positions += np.random.default_rng(14).normal(0, 0.08, s2.positions.shape)
    s2.types = np.random.default_rng(15).integers(0, 3, s2.natoms).astype(np.int32)
    cases.append(("fcc32_L24", "cfg2_L24_S3", s2, 5.0, 24, [3], True))
    # level 28, four species, 16 atoms (MLIP-table route only)
    s4 = synth.training_batch(1, 16, 16, 4, seed=16)[0]
    cases.append(("small_L28", "cfg4_L28_S4", s4, 5.5, 28, [2], False))

    for tag, pname, s, rc, L, fd_atoms, with_tree in cases:
        pot, back = pots[pname]
        nd = synth.build_neighbors(s, rc)
        mlip = rconv.MLIPMomentBasis(back)
        conv_route = None
        if with_tree:
            mb = rmom.MomentBasis(L)
            mb.init_moment_mappings()
            bc = rconv.BasisConverter(mb)
            bc.remap_mlip_moment_coeffs(back)
            conv_route = (rconv, mb, bc.remapped_coeffs)
        e_tab, e_tree = _site_energies_ref(back, nd, mlip, conv_route)
        h = 1e-5
        fd_f = np.zeros((len(fd_atoms), 3))
        for a_i, a in enumerate(fd_atoms):
            for k in range(3):
                sp = synth.Structure(s.positions.copy(), s.cell, s.types)
                sp.positions[a, k] += h
                ep = _total_energy(back, sp, rc, nd.n_pad, mlip)
                sp.positions[a, k] -= 2 * h
                em = _total_energy(back, sp, rc, nd.n_pad, mlip)
                fd_f[a_i, k] = -(ep - em) / (2 * h)
        # virial W_ab = -dE/d(eps_ab) for x -> (1 + eps) x, symmetric part, order xx,yy,zz,xy,xz,yz
        pairs = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
        fd_w = np.zeros(6)
        for v, (a, b) in enumerate(pairs):
            es = []
            for sgn in (1, -1):
                eps = np.zeros((3, 3))
                eps[a, b] += 0.5 * sgn * h
                eps[b, a] += 0.5 * sgn * h
                F = np.eye(3) + eps
                sp = synth.Structure(s.positions @ F.T, s.cell @ F.T, s.types)
                es.append(_total_energy(back, sp, rc, nd.n_pad, mlip))
            fd_w[v] = -(es[0] - es[1]) / (2 * h)
        np.savez_compressed(
            os.path.join(HERE, f"phys_{tag}.npz"), potential=pname + ".mtp", cutoff=rc,
            positions=s.positions, cell=s.cell, types=s.types,
            itypes=nd.itypes, rijs=nd.rijs, js=nd.js, jtypes=nd.jtypes, counts=nd.counts,
            volume=nd.volume, site_energies_tables=e_tab,
            site_energies_tree=(e_tree if e_tree is not None else np.zeros(0)),
            fd_atoms=np.array(fd_atoms), fd_forces=fd_f, fd_virial=fd_w, fd_step=h)
        msg = f"case {tag}: N={s.natoms} n_pad={nd.n_pad} E={e_tab.sum():.10f}"
        if e_tree is not None:
            msg += f" max|tab-tree|={np.abs(e_tab - e_tree).max():.2e}"
        print(msg)
    shutil.rmtree(tmp, ignore_errors=True)


if __name__ == "__main__":
    main()
