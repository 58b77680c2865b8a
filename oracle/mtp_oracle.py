"""FP64 CPU oracle for the MTP energy / force / stress path.

TEST INFRASTRUCTURE ONLY.  This module is the checker: ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may import it;
no product code path does.

It restates, in PyTorch CPU ``float64`` with autograd (the stand-in for the
reference's ``jax.value_and_grad``), the reference evaluator
``jax_backend.py`` of sebastian57/JAX-MTP:

* masks and smoothing ``(R_cut - d)^2``       jax_backend.py:83-90
* Chebyshev basis, T_{n+1} = 2 x T_n - T_{n-1} jax_backend.py:108-144
* radial functions f_mu = s * smooth * sum_n c[t_i, t_j, mu, n] T_n
                                              jax_backend.py:92-95, 146-160
* per-atom energy E_i = xi[t_i] + theta . basis jax_backend.py:97-106
* forces: autograd of E_i w.r.t. r_ij, then the Newton-3rd accumulation
                                              jax_backend.py:20-57, 263-303
* stress: sym(sum r (x) g) / V in Voigt (xx, yy, zz, yz, xz, xy)
                                              jax_backend.py:355-370
* masked total energy                         jax_backend.py:431-456

The basis is evaluated from the ``.mtp`` tables exactly as the reference's
``MLIPMomentBasis.calculate`` does (motep_original_files/jax_engine/
conversion.py:39-102): basic moments ``m_k = sum_j f_{mu_k}(d_j) u_x^a u_y^b
u_z^c``, then ``m[i3] += mult * m[i1] * m[i2]`` over ``alpha_index_times`` in
table order, then ``basis = m[alpha_moment_mapping]``.  The reference's
``BasisConverter`` proves that this basis equals the dense tensordot tree
that ``jax_backend._calc_basis_symmetric`` executes (conversion.py:112-168);
``tests/golden`` pins both against each other with the reference's own code.

This module reproduces the jax_backend math in float64 without deviations.
The training restatement below uses the *correct*
Chebyshev recurrence and Newton-3rd forces, not motep_original_files/
jax_engine/jax.py's off-by-one basis (jax.py:199-209) and j-less forces
(jax.py:96).
"""

from __future__ import annotations

import dataclasses
from typing import Dict, Optional, Sequence

import numpy as np
import torch

torch.set_default_dtype(torch.float64)

VOIGT_REF = (0, 4, 8, 5, 2, 1)   # xx, yy, zz, yz, xz, xy of a flattened 3x3 (jax_backend.py:359)


@dataclasses.dataclass
class OracleTables:
    """The ``.mtp`` fields the evaluator needs, as tensors."""

    scaling: float
    min_dist: float
    max_dist: float
    K: int
    R: int
    S: int
    radial: torch.Tensor          # [S, S, R, K]
    basic: np.ndarray             # [B, 4] (mu, a, b, c)
    times: np.ndarray             # [T, 4] (i1, i2, mult, i3)
    mapping: np.ndarray           # [Sa]
    M: int
    species_coeffs: torch.Tensor  # [S]
    moment_coeffs: torch.Tensor   # [Sa]
    levels: list                  # [(i1, i2, mult, i3) arrays] grouped by target depth

    @staticmethod
    def from_potential(pot) -> "OracleTables":
        t = np.asarray(pot.alpha_index_times, dtype=np.int64).reshape(-1, 4)
        M = int(pot.alpha_moments_count)
        depth = np.zeros(M, dtype=np.int64)
        for i1, i2, _, i3 in t:
            depth[i3] = max(depth[i3], max(depth[i1], depth[i2]) + 1)
        # Level-by-level evaluation equals the sequential loop of
        # conversion.py:95-102 when every moment is fully written before it
        # is read; check that, else keep the sequential order.
        sequential_ok = True
        last_write = np.full(M, -1)
        first_read = np.full(M, np.iinfo(np.int64).max)
        for e, (i1, i2, _, i3) in enumerate(t):
            last_write[i3] = e
            first_read[i1] = min(first_read[i1], e)
            first_read[i2] = min(first_read[i2], e)
        if np.any((last_write >= 0) & (first_read <= last_write)):
            sequential_ok = False
        levels = []
        if sequential_ok and len(t):
            td = depth[t[:, 3]]
            for L in range(1, int(td.max()) + 1):
                levels.append(t[td == L])
        elif len(t):
            levels = [t[e:e + 1] for e in range(len(t))]
        return OracleTables(
            scaling=float(pot.scaling), min_dist=float(pot.min_dist), max_dist=float(pot.max_dist),
            K=int(pot.radial_basis_size), R=int(pot.radial_funcs_count), S=int(pot.species_count),
            radial=torch.tensor(np.asarray(pot.radial_coeffs, dtype=np.float64)),
            basic=np.asarray(pot.alpha_index_basic, dtype=np.int64).reshape(-1, 4), times=t,
            mapping=np.asarray(pot.alpha_moment_mapping, dtype=np.int64), M=M,
            species_coeffs=torch.tensor(np.asarray(pot.species_coeffs, dtype=np.float64)),
            moment_coeffs=torch.tensor(np.asarray(pot.moment_coeffs, dtype=np.float64)),
            levels=levels)


def chebyshev(d: torch.Tensor, K: int, rmin: float, rmax: float) -> torch.Tensor:
    """T_0..T_{K-1} of x = (2d - (rmin + rmax)) / (rmax - rmin)   (jax_backend.py:108-144)."""
    if K == 0:
        return d.new_zeros(d.shape + (0,))
    x = (2.0 * d - (rmin + rmax)) * (1.0 / (rmax - rmin))
    T = [torch.ones_like(x)]
    if K > 1:
        T.append(x)
    for _ in range(K - 2):
        T.append(2.0 * x * T[-1] - T[-2])
    return torch.stack(T, dim=-1)


def radial_values(tab: OracleTables, rij: torch.Tensor, itypes: torch.Tensor, jtypes: torch.Tensor,
                  radial: Optional[torch.Tensor] = None):
    """Returns (d [N,n], valid [N,n], f [N,n,R]) following jax_backend.py:83-95, 146-160.

    Invalid slots (neighbour species < 0, or d >= max_dist) get f = 0 exactly;
    their r is replaced by a unit dummy so that no 0/0 enters the graph (the
    reference feeds finite sentinels there, with the same zero result).
    """
    radial = tab.radial if radial is None else radial
    r2 = (rij * rij).sum(-1)
    d0 = torch.sqrt(torch.where(r2 > 0, r2, torch.ones_like(r2)))
    valid = (jtypes >= 0) & (d0 < tab.max_dist) & (r2 > 0)
    safe = torch.where(valid[..., None], rij, torch.tensor([1.0, 0.0, 0.0]).expand_as(rij))
    d = torch.sqrt((safe * safe).sum(-1))
    smooth = torch.where(valid, (tab.max_dist - d) ** 2, torch.zeros_like(d))
    T = chebyshev(d, tab.K, tab.min_dist, tab.max_dist)                      # [N, n, K]
    it = itypes.clamp(min=0).long()
    jt = jtypes.clamp(min=0).long()
    coeffs = radial[it[:, None], jt]                                         # [N, n, R, K]
    base = torch.einsum("anmk,ank->anm", coeffs, T)
    f = tab.scaling * smooth[..., None] * base
    return d, valid, f, safe


def moments_from_tables(tab: OracleTables, u: torch.Tensor, f: torch.Tensor) -> torch.Tensor:
    """All alpha moments [N, M] from unit vectors u [N,n,3] and radial values f [N,n,R].

    Basic moments as conversion.py:66-81, contractions as conversion.py:95-102.
    """
    N = u.shape[0]
    B = tab.basic.shape[0]
    mu, a, b, c = (torch.tensor(tab.basic[:, k]) for k in range(4))
    maxp = int(tab.basic[:, 1:].max()) if B else 0
    pw = [torch.ones_like(u)]
    for _ in range(maxp):
        pw.append(pw[-1] * u)
    pw = torch.stack(pw, dim=0)                                              # [P+1, N, n, 3]
    mono = pw[a, :, :, 0] * pw[b, :, :, 1] * pw[c, :, :, 2]                  # [B, N, n]
    fk = f.permute(2, 0, 1)[mu]                                              # [B, N, n]
    basic = (fk * mono).sum(-1).T                                            # [N, B]
    m = torch.cat([basic, u.new_zeros(N, tab.M - B)], dim=1)
    for lev in tab.levels:
        i1 = torch.tensor(lev[:, 0]); i2 = torch.tensor(lev[:, 1])
        mult = torch.tensor(lev[:, 2], dtype=torch.float64); i3 = torch.tensor(lev[:, 3])
        prod = mult * m[:, i1] * m[:, i2]
        m = m.index_add(1, i3, prod)
    return m


def site_energies(tab: OracleTables, rij: torch.Tensor, itypes: torch.Tensor, jtypes: torch.Tensor,
                  params: Optional[Dict[str, torch.Tensor]] = None) -> torch.Tensor:
    """Per-atom energies E_i (jax_backend.py:59-106)."""
    params = params or {}
    radial = params.get("radial", tab.radial)
    xi = params.get("species", tab.species_coeffs)
    theta = params.get("basis", tab.moment_coeffs)
    d, valid, f, safe = radial_values(tab, rij, itypes, jtypes, radial)
    u = safe / d[..., None]
    m = moments_from_tables(tab, u, f)
    basis = m[:, torch.tensor(tab.mapping)]
    return xi[itypes.clamp(min=0).long()] + basis @ theta


def accumulate_forces(g: torch.Tensor, js: torch.Tensor, natoms: int) -> torch.Tensor:
    """F_k = sum_s g_ks - sum_{(i,s): j_is = k} g_is, masked as jax_backend.py:263-303."""
    A, n, _ = g.shape
    amask = (torch.arange(A) < natoms)
    gr = torch.where(amask[:, None, None], g, torch.zeros_like(g))
    Fi = gr.sum(1)
    jf = js.reshape(-1).long()
    vmask = amask.repeat_interleave(n) & (jf < natoms) & (jf >= 0)
    gf = torch.where(vmask[:, None], gr.reshape(-1, 3), torch.zeros(1, 3))
    Fj = torch.zeros(A, 3).index_add(0, torch.where(vmask, jf, torch.zeros_like(jf)), -gf)
    return Fi + Fj


def stress_voigt(rij: torch.Tensor, g: torch.Tensor, volume: float, cell_rank: int = 3) -> torch.Tensor:
    """sym(sum_{a,s} r (x) g) / V in the reference's Voigt order (jax_backend.py:355-370)."""
    if cell_rank != 3:
        return torch.full((6,), float("nan"))
    W = torch.einsum("aij,aik->jk", rij, g)
    sym = (W + W.T) * (0.5 / volume)
    return sym.reshape(-1)[list(VOIGT_REF)]


def evaluate(pot_or_tab, itypes, rijs, js, jtypes, volume: float, natoms: Optional[int] = None,
             cell_rank: int = 3) -> Dict[str, np.ndarray]:
    """Reference semantics of calc_energy_forces_stress_padded (jax_backend.py:374-460), FP64.

    Returns energy, site energies, forces [A,3], per-slot gradients g = dE_i/dr_ij,
    the reference stress (Voigt xx,yy,zz,yz,xz,xy, /V) and the LAMMPS virial
    W = -sum r (x) g symmetrised, in order xx,yy,zz,xy,xz,yz (energy units).
    """
    tab = pot_or_tab if isinstance(pot_or_tab, OracleTables) else OracleTables.from_potential(pot_or_tab)
    itypes_t = torch.as_tensor(np.asarray(itypes), dtype=torch.int64)
    A = itypes_t.shape[0]
    natoms = A if natoms is None else int(natoms)
    rij = torch.tensor(np.asarray(rijs, dtype=np.float64), requires_grad=True)
    jt = torch.as_tensor(np.asarray(jtypes), dtype=torch.int64)
    js_t = torch.as_tensor(np.asarray(js), dtype=torch.int64)
    E_i = site_energies(tab, rij, itypes_t, jt)
    (g,) = torch.autograd.grad(E_i.sum(), rij)
    with torch.no_grad():
        F = accumulate_forces(g, js_t, natoms)
        sig = stress_voigt(rij, g, volume, cell_rank)
        W = -torch.einsum("aij,aik->jk", rij, g)
        W = 0.5 * (W + W.T)
        vir = torch.stack([W[0, 0], W[1, 1], W[2, 2], W[0, 1], W[0, 2], W[1, 2]])
        E = E_i[:natoms].sum()
    return {
        "energy": float(E), "site_energies": E_i.detach().numpy(), "forces": F.numpy(),
        "pair_grads": g.numpy(), "stress": sig.numpy(), "virial": vir.numpy(),
    }


# ----------------------------------------------------------------------------
# Training loss (training/motep_jax_train_function.py:67-74) with autograd
# ----------------------------------------------------------------------------

def batch_predictions(tab: OracleTables, params: Dict[str, torch.Tensor], itypes, rijs, js, jtypes,
                      cfg_of_atom, ncfg: int, volumes, create_graph: bool = True):
    """Differentiable (E [C], F [Ntot,3], sigma [C,6]) for a flat batch of configurations.

    Forces use the correct Newton-3rd accumulation of jax_backend.py:263-303
    (global neighbour indices), stress follows jax_backend.py:355-370 per
    configuration.
    """
    it = torch.as_tensor(np.asarray(itypes), dtype=torch.int64)
    rij = torch.as_tensor(np.asarray(rijs, dtype=np.float64)).clone().requires_grad_(True)
    jt = torch.as_tensor(np.asarray(jtypes), dtype=torch.int64)
    jsl = torch.as_tensor(np.asarray(js), dtype=torch.int64)
    cfg = torch.as_tensor(np.asarray(cfg_of_atom), dtype=torch.int64)
    E_i = site_energies(tab, rij, it, jt, params)
    (g,) = torch.autograd.grad(E_i.sum(), rij, create_graph=create_graph)
    A = it.shape[0]
    F = accumulate_forces(g, jsl, A)
    E = torch.zeros(ncfg).index_add(0, cfg, E_i)
    W = torch.einsum("aij,aik->ajk", rij, g)                                  # per atom
    Wc = torch.zeros(ncfg, 3, 3).index_add(0, cfg, W)
    vol = torch.as_tensor(np.asarray(volumes, dtype=np.float64))
    sym = (Wc + Wc.transpose(1, 2)) * (0.5 / vol)[:, None, None]
    sig = sym.reshape(ncfg, 9)[:, list(VOIGT_REF)]
    return E, F, sig


def loss_and_grad(tab: OracleTables, params: Dict[str, np.ndarray], batch, targets,
                  weights=(1.0, 0.01, 0.001)):
    """Loss we*sum(dE^2) + wf*sum(dF^2) + ws*sum(dsigma^2) and its gradient
    w.r.t. species, radial and basis coefficients (double backward through forces)."""
    p = {k: torch.tensor(np.asarray(v, dtype=np.float64), requires_grad=True) for k, v in params.items()}
    itypes, rijs, js, jtypes, cfg, ncfg, vols = batch
    E, F, sig = batch_predictions(tab, p, itypes, rijs, js, jtypes, cfg, ncfg, vols, create_graph=True)
    Et, Ft, St = (torch.as_tensor(np.asarray(x, dtype=np.float64)) for x in targets)
    we, wf, ws = weights
    L = we * ((E - Et) ** 2).sum() + wf * ((F - Ft) ** 2).sum() + ws * ((sig - St) ** 2).sum()
    grads = torch.autograd.grad(L, [p["species"], p["radial"], p["basis"]])
    return float(L.detach()), {"species": grads[0].numpy(), "radial": grads[1].numpy(), "basis": grads[2].numpy()}
