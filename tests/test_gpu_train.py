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
