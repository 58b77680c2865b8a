"""The hand-written adjoint (training gradient) against the oracle (GPU).

Bar: gradients of the E/F/stress loss with respect to species, moment and
radial coefficients match torch double-backward on the FP64 oracle to <= 1e-8
relative (the target is 1e-6), and central finite differences of the GPU
loss (h = 1e-6, FP64) on randomly chosen coefficients.
"""

import numpy as np
import pytest
import torch

from conftest import potential_path
from mtp_b200 import synth
from mtp_b200.engine import MTPEngine
from mtp_b200.mtp_file import read_mtp
from mtp_b200.train import DeviceBatch, predict, weighted_loss
from oracle import mtp_oracle as O

pytestmark = pytest.mark.gpu


def _setup(name, nconf, nmin, nmax, seed):
    pot = read_mtp(potential_path(name))
    structs = synth.training_batch(nconf, nmin, nmax, pot.species_count, seed=seed)
    nds = [synth.build_neighbors(s, pot.max_dist) for s in structs]
    nd, cfg, offs, vols = synth.pack_batch(nds)
    rng = np.random.default_rng(seed + 1)
    targets = (rng.normal(size=nconf) * 10, rng.normal(size=(nd.natoms, 3)), rng.normal(size=(nconf, 6)) * 1e-2)
    return pot, nd, cfg, vols, targets


def _rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(1e-300, np.abs(np.asarray(b)).max()))


@pytest.mark.parametrize("name,nconf,nmin,nmax", [("cfg3_L20_S2.mtp", 4, 8, 24), ("cfg0_L16_S1.mtp", 3, 6, 16),
                                                  ("cfg4_L28_S4.mtp", 2, 6, 10)])
def test_adjoint_matches_oracle_double_backward(name, nconf, nmin, nmax):
    pot, nd, cfg, vols, targets = _setup(name, nconf, nmin, nmax, seed=41)
    tab = O.OracleTables.from_potential(pot)
    params = {"species": pot.species_coeffs, "radial": pot.radial_coeffs, "basis": pot.moment_coeffs}
    L_ref, g_ref = O.loss_and_grad(tab, params, (nd.itypes, nd.rijs, nd.js, nd.jtypes, cfg, nconf, vols), targets)
    dev = torch.device("cuda")
    batch = DeviceBatch.from_numpy(nd, cfg, vols, device=dev)
    tt = tuple(torch.as_tensor(t, dtype=torch.float64, device=dev) for t in targets)
    with MTPEngine(potential_path(name), nd.natoms, nd.n_pad) as eng:
        p = {k: torch.tensor(v, dtype=torch.float64, device=dev, requires_grad=True) for k, v in params.items()}
        E, F, S = predict(p, eng, batch)
        L = weighted_loss(E, F, S, tt)
        L.backward()
        eng.sync_status()
    assert abs(float(L) - L_ref) <= 1e-10 * abs(L_ref)
    for k in ("species", "radial", "basis"):
        assert _rel(p[k].grad.cpu().numpy(), g_ref[k]) <= 1e-8, k


def test_adjoint_matches_finite_differences():
    name = "cfg3_L20_S2.mtp"
    pot, nd, cfg, vols, targets = _setup(name, 3, 8, 20, seed=43)
    dev = torch.device("cuda")
    batch = DeviceBatch.from_numpy(nd, cfg, vols, device=dev)
    tt = tuple(torch.as_tensor(t, dtype=torch.float64, device=dev) for t in targets)
    base = {"species": pot.species_coeffs, "radial": pot.radial_coeffs, "basis": pot.moment_coeffs}
    with MTPEngine(potential_path(name), nd.natoms, nd.n_pad) as eng:
        def loss(pp, grad=False):
            p = {k: torch.tensor(v, dtype=torch.float64, device=dev, requires_grad=grad) for k, v in pp.items()}
            L = weighted_loss(*predict(p, eng, batch), tt)
            if grad:
                L.backward()
                return float(L), {k: p[k].grad.cpu().numpy() for k in p}
            return float(L)
        L0, g = loss(base, grad=True)
        rng = np.random.default_rng(5)
        picks = [("basis", (int(i),)) for i in rng.choice(pot.alpha_scalar_moments, 12, replace=False)]
        picks += [("radial", tuple(int(x) for x in rng.integers(0, s))) for s in [pot.radial_coeffs.shape] * 16]
        picks += [("species", (0,)), ("species", (1,))]
        h = 1e-6
        for key, idx in picks:
            pp = {k: np.array(v, dtype=np.float64) for k, v in base.items()}
            pp[key][idx] += h
            lp = loss(pp)
            pp[key][idx] -= 2 * h
            lm = loss(pp)
            fd = (lp - lm) / (2 * h)
            assert abs(fd - g[key][idx]) <= 1e-6 * max(1.0, abs(fd)) + 1e-7 * abs(L0), (key, idx, fd, g[key][idx])


def test_adjoint_deterministic():
    name = "cfg3_L20_S2.mtp"
    pot, nd, cfg, vols, targets = _setup(name, 3, 8, 20, seed=47)
    dev = torch.device("cuda")
    batch = DeviceBatch.from_numpy(nd, cfg, vols, device=dev)
    gE = torch.ones(3, dtype=torch.float64, device=dev)
    gF = torch.ones((nd.natoms, 3), dtype=torch.float64, device=dev)
    gS = torch.ones((3, 6), dtype=torch.float64, device=dev)
    with MTPEngine(potential_path(name), nd.natoms, nd.n_pad) as eng:
        a = eng.adjoint_device(batch.itypes, batch.rijs, batch.js, batch.jtypes, batch.counts, batch.cfg,
                               batch.volumes, 3, gE, gF, gS)
        b = eng.adjoint_device(batch.itypes, batch.rijs, batch.js, batch.jtypes, batch.counts, batch.cfg,
                               batch.volumes, 3, gE, gF, gS)
        torch.cuda.synchronize()
    for x, y in zip(a, b):
        assert torch.equal(x, y)


def _teacher_batch(name, nconf, nmin, nmax, seed, noise):
    """Structures labelled by the potential itself (FP64 oracle) plus noise."""
    pot = read_mtp(potential_path(name))
    structs = synth.training_batch(nconf, nmin, nmax, pot.species_count, seed=seed)
    nds = [synth.build_neighbors(s, pot.max_dist) for s in structs]
    nd, cfg, offs, vols = synth.pack_batch(nds)
    tab = O.OracleTables.from_potential(pot)
    p = {"species": torch.tensor(pot.species_coeffs), "radial": torch.tensor(pot.radial_coeffs),
         "basis": torch.tensor(pot.moment_coeffs)}
    E, F, S = O.batch_predictions(tab, p, nd.itypes, nd.rijs, nd.js, nd.jtypes, cfg, nconf, vols, create_graph=False)
    rng = np.random.default_rng(seed + 7)
    E = E.detach().numpy() + noise * rng.normal(size=nconf)
    F = F.detach().numpy() + noise * rng.normal(size=(nd.natoms, 3))
    S = S.detach().numpy() + 0.01 * noise * rng.normal(size=(nconf, 6))
    return pot, structs, nd, cfg, vols, tab, (E, F, S)


def test_lls_basis_matches_dense_lstsq():
    """solve_lls_basis (matrix-free CG on the GPU) reaches the loss minimum
    that a dense least-squares solve over the oracle's Jacobian reaches
    (the reference's jacfwd + lstsq, motep_jax_train_import.py:604-683)."""
    from mtp_b200.train import solve_lls_basis
    name = "cfg1_L16_S2.mtp"
    pot, _, nd, cfg, vols, tab, targets = _teacher_batch(name, 5, 4, 10, seed=61, noise=0.05)
    nconf = len(vols)
    w = (1.0, 0.01, 0.001)
    sw = np.sqrt(w)
    sp, ra = torch.tensor(pot.species_coeffs), torch.tensor(pot.radial_coeffs)

    def flat(basis):
        E, F, S = O.batch_predictions(tab, {"species": sp, "radial": ra, "basis": torch.as_tensor(basis)},
                                      nd.itypes, nd.rijs, nd.js, nd.jtypes, cfg, nconf, vols, create_graph=False)
        return np.concatenate([sw[0] * E.detach().numpy(), sw[1] * F.detach().numpy().ravel(),
                               sw[2] * S.detach().numpy().ravel()])

    Sa = pot.alpha_scalar_moments
    off = flat(np.zeros(Sa))
    X = np.stack([flat(np.eye(Sa)[a]) - off for a in range(Sa)], axis=1)
    y = np.concatenate([sw[0] * targets[0], sw[1] * targets[1].ravel(), sw[2] * targets[2].ravel()]) - off
    th_ref = np.linalg.lstsq(X, y, rcond=None)[0]
    loss_ref = float(np.sum((X @ th_ref - y) ** 2))
    dev = torch.device("cuda")
    batch = DeviceBatch.from_numpy(nd, cfg, vols, device=dev)
    tt = tuple(torch.as_tensor(t, dtype=torch.float64, device=dev) for t in targets)
    with MTPEngine(potential_path(name), nd.natoms, nd.n_pad) as eng:
        theta, info = solve_lls_basis(eng, batch, tt, pot.species_coeffs, pot.radial_coeffs, w)
        theta_cg, info_cg = solve_lls_basis(eng, batch, tt, pot.species_coeffs, pot.radial_coeffs, w, method="cg",
                                            max_iter=1000)
        eng.sync_status()
    th = theta.cpu().numpy()
    loss_gpu = float(np.sum((X @ th - y) ** 2))
    assert loss_gpu <= loss_ref * (1 + 1e-9) + 1e-15, (loss_gpu, loss_ref, info)
    assert abs(info["loss"] - loss_gpu) <= 1e-9 * loss_gpu
    # both minimum-norm solutions and their predictions agree
    assert np.abs(X @ th - X @ th_ref).max() <= 1e-8 * np.abs(y).max()
    assert _rel(th, th_ref) <= 1e-6
    # the matrix-free variant gets close without storing X (CG on the normal
    # equations converges slowly on this ill-conditioned basis)
    assert info_cg["loss"] <= 1.1 * loss_ref


def test_cfg_to_lls_to_lbfgs_pipeline(tmp_path):
    """.cfg ingest -> least-squares basis -> L-BFGS on all coefficients
    (the reference's training flow, motep_jax_train_function.py:150-213),
    all on the GPU forward and adjoint; the loss falls at every stage."""
    from mtp_b200.cfg_file import Configuration, read_cfg, write_cfg
    from mtp_b200.train import batch_from_configs, fit_lbfgs, solve_lls_basis
    name = "cfg1_L16_S2.mtp"
    pot, structs, nd, cfg, vols, tab, (E, F, S) = _teacher_batch(name, 8, 4, 12, seed=71, noise=0.01)
    offs = np.concatenate([[0], np.cumsum([s.natoms for s in structs])])
    configs = [Configuration(s.types, s.positions, s.cell, float(E[c]), F[offs[c]:offs[c + 1]],
                             -S[c] * s.volume, {"origin": "synthetic"}) for c, s in enumerate(structs)]
    write_cfg(tmp_path / "train.cfg", configs)
    back = read_cfg(tmp_path / "train.cfg")
    dev = torch.device("cuda")
    batch, tt = batch_from_configs(back, pot.max_dist, device=dev)
    np.testing.assert_allclose(tt[2].cpu().numpy(), S, rtol=1e-8, atol=1e-12)
    rng = np.random.default_rng(9)
    with MTPEngine(potential_path(name), batch.natoms, int(batch.rijs.shape[1])) as eng:
        # start from a perturbed potential
        params = {"species": torch.tensor(pot.species_coeffs + 0.1, device=dev),
                  "basis": torch.tensor(pot.moment_coeffs * (1 + 0.5 * rng.normal(size=pot.alpha_scalar_moments)),
                                        device=dev),
                  "radial": torch.tensor(pot.radial_coeffs * (1 + 0.02 * rng.normal(size=pot.radial_coeffs.shape)),
                                         device=dev)}
        with torch.no_grad():
            L0 = float(weighted_loss(*predict(params, eng, batch), tt))
        theta, info = solve_lls_basis(eng, batch, tt, params["species"].cpu().numpy(),
                                      params["radial"].cpu().numpy())
        params["basis"] = theta.clone()
        with torch.no_grad():
            L1 = float(weighted_loss(*predict(params, eng, batch), tt))
        out = fit_lbfgs(eng, batch, tt, params, steps=30)
        with torch.no_grad():
            E_fit, F_fit, _ = predict(params, eng, batch)
        eng.sync_status()
    # write-out: the trained potential reloaded in a new engine predicts the same
    from mtp_b200.mtp_file import write_mtp
    trained = pot.copy()
    trained.species_coeffs = params["species"].detach().cpu().numpy()
    trained.moment_coeffs = params["basis"].detach().cpu().numpy()
    trained.radial_coeffs = params["radial"].detach().cpu().numpy()
    write_mtp(tmp_path / "trained.mtp", trained)
    with MTPEngine(str(tmp_path / "trained.mtp"), batch.natoms, int(batch.rijs.shape[1])) as eng2:
        E2, F2, _ = eng2.batch_device(batch.itypes, batch.rijs, batch.js, batch.jtypes, batch.counts, batch.cfg,
                                      batch.volumes, batch.nconfig)
        eng2.sync_status()
    assert _rel(E2.cpu().numpy(), E_fit.cpu().numpy()) <= 1e-12
    assert _rel(F2.cpu().numpy(), F_fit.cpu().numpy()) <= 1e-10
    assert L1 < L0
    assert abs(L1 - info["loss"]) <= 1e-6 * L1
    hist = out["loss_history"]
    # every accepted L-BFGS step lowers the loss (Armijo); the radial and
    # species coefficients move the loss below the least-squares optimum
    assert all(np.isfinite(hist)) and out["steps"] >= 10
    assert all(b <= a for a, b in zip([L1] + hist[:-1], hist)), hist
    assert hist[-1] < 0.995 * L1, (L0, L1, hist)


def _cfg4_batch(nconf, seed):
    """The first `nconf` configurations of the config-4 generator (32-512 atoms,
    fcc/bcc/hcp, a in [2.8, 4.2] A, strain 3 %, sigma 0.1 A) whose pairs all lie
    at or beyond the potential's min_dist.  The generator also makes pairs down
    to ~1.45 A (fcc near a = 2.8 A with thermal displacement); there the
    Chebyshev basis is evaluated outside [-1, 1], site energies of this random
    potential reach ~1e9 eV, and a central difference in FP64 keeps no
    significant digits, so those configurations are not used for this check."""
    pot = read_mtp(potential_path("cfg4_L28_S4.mtp"))
    structs, nds = [], []
    for s in synth.training_batch(4 * nconf, 32, 512, pot.species_count, seed=seed):
        nd = synth.build_neighbors(s, pot.max_dist)
        d = np.linalg.norm(nd.rijs, axis=2)[nd.jtypes >= 0]
        if d.size and d.min() >= pot.min_dist:
            structs.append(s)
            nds.append(nd)
        if len(nds) == nconf:
            break
    assert len(nds) == nconf
    nd, cfg, offs, vols = synth.pack_batch(nds)
    return pot, nd, cfg, offs, vols


def test_cfg4_adjoint_matches_central_differences():
    """Config 4's stated gradient check: central differences (h = 1e-6, FP64) of
    the E/F/stress loss (weights 1, 0.01, 0.001; training/motep_jax_train_function.py:67-74)
    on 32 random coefficients of the level-28, 4-species potential (2 species,
    14 radial, 16 basis), over 8 configurations labelled by the potential
    itself plus the stated noise (1 meV/atom, 10 meV/A, 0.1 GPa).

    The difference is the fourth-order central stencil
    (-L(+2h) + 8 L(+h) - 8 L(-h) + L(-2h)) / 12h: the random level-28
    coefficients give gradients up to ~1e7, whose third derivatives make the
    two-point stencil's O(h^2) error reach ~1e-6 relative on its own."""
    pot, nd, cfg, offs, vols = _cfg4_batch(8, seed=81)
    dev = torch.device("cuda")
    batch = DeviceBatch.from_numpy(nd, cfg, vols, device=dev)
    base = {"species": pot.species_coeffs, "radial": pot.radial_coeffs, "basis": pot.moment_coeffs}
    with MTPEngine(potential_path("cfg4_L28_S4.mtp"), nd.natoms, nd.n_pad) as eng:
        def predict_np(pp, grad=False):
            p = {k: torch.tensor(v, dtype=torch.float64, device=dev, requires_grad=grad) for k, v in pp.items()}
            return p, predict(p, eng, batch)

        with torch.no_grad():
            _, (E0, F0, S0) = predict_np(base)
        rng = np.random.default_rng(82)
        natom_c = torch.as_tensor(np.diff(offs), dtype=torch.float64, device=dev)
        tt = (E0 + 1e-3 * natom_c * torch.as_tensor(rng.normal(size=E0.shape), device=dev),
              F0 + 1e-2 * torch.as_tensor(rng.normal(size=F0.shape), device=dev),
              S0 + 6.2415e-4 * torch.as_tensor(rng.normal(size=S0.shape), device=dev))

        def loss(pp):
            with torch.no_grad():
                return float(weighted_loss(*predict_np(pp)[1], tt))

        p, (E, F, S) = predict_np(base, grad=True)
        L0 = weighted_loss(E, F, S, tt)
        L0.backward()
        g = {k: p[k].grad.cpu().numpy() for k in p}
        L0 = float(L0)
        eng.sync_status()
        picks = [("species", (int(i),)) for i in rng.choice(pot.species_count, 2, replace=False)]
        picks += [("radial", tuple(int(x) for x in rng.integers(0, s))) for s in [pot.radial_coeffs.shape] * 14]
        picks += [("basis", (int(i),)) for i in rng.choice(pot.alpha_scalar_moments, 16, replace=False)]
        assert len(picks) == 32
        h = 1e-6
        gmax = max(np.abs(v).max() for v in g.values())
        for key, idx in picks:
            def at(step):
                pp = {k: np.array(v, dtype=np.float64) for k, v in base.items()}
                pp[key][idx] += step
                return loss(pp)
            fd = (-at(2 * h) + 8 * at(h) - 8 * at(-h) + at(-2 * h)) / (12 * h)
            # 1e-6 relative to the component, or to the gradient's scale for
            # components near zero (FP64 roundoff of the loss over h)
            assert abs(fd - g[key][idx]) <= 1e-6 * max(abs(fd), 1e-3 * gmax), (key, idx, fd, g[key][idx], gmax)


def test_autotuned_training_launches_agree():
    """The training autotuner (neighbour tile, threads, atoms per block) changes
    only the launch: the tuned batched forward and the tuned training gradient
    equal the untuned ones (FP64, <= 1e-10 relative)."""
    from mtp_b200.autotune import tile_candidates, tune_batch, tune_step
    name = "cfg3_L20_S2.mtp"
    pot, nd, cfg, vols, targets = _setup(name, 4, 8, 40, seed=91)
    dev = torch.device("cuda")
    batch = DeviceBatch.from_numpy(nd, cfg, vols, device=dev)
    tt = tuple(torch.as_tensor(t, dtype=torch.float64, device=dev) for t in targets)
    tiles = tile_candidates(int(nd.counts.max()))
    base = {"species": pot.species_coeffs, "radial": pot.radial_coeffs, "basis": pot.moment_coeffs}
    with MTPEngine(potential_path(name), nd.natoms, max(tiles)) as eng:
        def grads(b):
            p = {k: torch.tensor(v, dtype=torch.float64, device=dev, requires_grad=True) for k, v in base.items()}
            L = weighted_loss(*predict(p, eng, b), tt)
            L.backward()
            return [p[k].grad.cpu().numpy() for k in ("species", "radial", "basis")]

        E0, F0, S0 = eng.batch_device(batch.itypes, batch.rijs, batch.js, batch.jtypes, batch.counts, batch.cfg,
                                      batch.volumes, batch.nconfig)
        g0 = grads(batch)
        r = tune_batch(eng, batch, tiles=tiles, calls=1)
        b = r["batch"]
        assert r["n_pad"] in tiles and b.stride == r["n_pad"] and len(r["timings"]) >= len(tiles)
        E1, F1, S1 = eng.batch_device(b.itypes, b.rijs, b.js, b.jtypes, b.counts, b.cfg, b.volumes, b.nconfig)
        r2 = tune_step(eng, batch, lambda bb: grads(bb), candidates=((256, 1), (512, 1), (256, 2)), tiles=tiles,
                       calls=1)
        g1 = grads(r2["batch"])
        eng.sync_status()
    assert _rel(E1.cpu().numpy(), E0.cpu().numpy()) <= 1e-10
    assert _rel(F1.cpu().numpy(), F0.cpu().numpy()) <= 1e-10
    assert _rel(S1.cpu().numpy(), S0.cpu().numpy()) <= 1e-10
    for a, c in zip(g1, g0):
        assert _rel(a, c) <= 1e-10
