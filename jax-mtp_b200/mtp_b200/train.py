"""Training on the CUDA engine: batched E/F/stress with a hand-written adjoint.

``MTPFunction`` is a ``torch.autograd.Function`` whose forward is the batched
evaluation kernel (one persistent launch over all atoms of all
configurations) and whose backward is the dual-number adjoint kernel
(mtp_adjoint_batch_device): gradients of any loss of (E, F, sigma) with
respect to the species, moment (basis) and radial coefficients, including the
second derivatives the force and stress terms need.  The moment tensors are
recomputed in the backward pass; nothing per-atom is kept between the two.

The loss is the reference's (training/motep_jax_train_function.py:67-74):
``we * sum (E - E*)^2 + wf * sum (F - F*)^2 + ws * sum (sigma - sigma*)^2``
with weights (1, 0.01, 0.001), on forces computed with the Newton-3rd term
(jax_backend.py:263-303); the reference training code's own forward omits
that term (motep_original_files/jax_engine/jax.py:96), which is not
reproduced.
"""

from __future__ import annotations

import dataclasses
from typing import Optional, Sequence

import numpy as np
import torch

from .engine import MTPEngine

__all__ = ["DeviceBatch", "MTPFunction", "predict", "weighted_loss", "Trainer", "batch_from_configs",
           "solve_lls_basis", "fit_lbfgs"]


@dataclasses.dataclass
class DeviceBatch:
    """A packed batch of configurations resident on the GPU."""

    itypes: torch.Tensor     # [N] int32
    rijs: torch.Tensor       # [N, n, 3] float64
    js: torch.Tensor         # [N, n] int32 (global atom indices)
    jtypes: torch.Tensor     # [N, n] int32
    counts: torch.Tensor     # [N] int32
    cfg: torch.Tensor        # [N] int32, non-decreasing
    volumes: torch.Tensor    # [C] float64
    nconfig: int

    @staticmethod
    def from_numpy(nd, cfg, volumes, device="cuda") -> "DeviceBatch":
        T = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=device)
        return DeviceBatch(T(nd.itypes, torch.int32), T(nd.rijs, torch.float64), T(nd.js, torch.int32),
                           T(nd.jtypes, torch.int32), T(nd.counts, torch.int32), T(cfg, torch.int32),
                           T(volumes, torch.float64), int(len(volumes)))

    @property
    def natoms(self) -> int:
        return int(self.itypes.shape[0])

    @property
    def stride(self) -> int:
        return int(self.rijs.shape[1])

    def with_stride(self, n: int) -> "DeviceBatch":
        """The same batch with rows of `n` slots (every row's count must fit;
        slots past a row's count are never read, so narrowing drops padding only)."""
        longest = int(self.counts.max()) if self.natoms else 0
        if n <= 0 or n < longest:
            raise ValueError(f"rows of {n} slots cannot hold the longest row ({longest})")
        if n <= self.stride:
            sl = slice(0, n)
            return dataclasses.replace(self, rijs=self.rijs[:, sl].contiguous(), js=self.js[:, sl].contiguous(),
                                       jtypes=self.jtypes[:, sl].contiguous())
        pad = n - self.stride
        N = self.natoms
        dev = self.rijs.device
        return dataclasses.replace(
            self, rijs=torch.cat([self.rijs, torch.zeros((N, pad, 3), dtype=self.rijs.dtype, device=dev)], 1),
            js=torch.cat([self.js, torch.full((N, pad), -1, dtype=self.js.dtype, device=dev)], 1),
            jtypes=torch.cat([self.jtypes, torch.full((N, pad), -1, dtype=self.jtypes.dtype, device=dev)], 1))


class MTPFunction(torch.autograd.Function):
    """(species, moment, radial) -> (E [C], F [N,3], sigma [C,6])."""

    @staticmethod
    def forward(ctx, species, moment, radial, engine: MTPEngine, batch: DeviceBatch):
        engine.set_coeffs(species.detach().double().cpu().numpy(), moment.detach().double().cpu().numpy(),
                          radial.detach().double().cpu().numpy())
        b = batch
        E, F, S = engine.batch_device(b.itypes, b.rijs, b.js, b.jtypes, b.counts, b.cfg, b.volumes, b.nconfig)
        ctx.engine = engine
        ctx.batch = batch
        ctx.coeffs = (species.detach(), moment.detach(), radial.detach())
        ctx.devices = (species.device, moment.device, radial.device)
        return E, F, S

    @staticmethod
    def backward(ctx, gE, gF, gS):
        b = ctx.batch
        eng = ctx.engine
        sp, mo, ra = ctx.coeffs
        # the handle may have seen other coefficients since the forward
        eng.set_coeffs(sp.double().cpu().numpy(), mo.double().cpu().numpy(), ra.double().cpu().numpy())
        dev = b.rijs.device
        z = lambda shape: torch.zeros(shape, dtype=torch.float64, device=dev)
        gE = z(b.nconfig) if gE is None else gE.to(dev, torch.float64).contiguous()
        gF = z((b.natoms, 3)) if gF is None else gF.to(dev, torch.float64).contiguous()
        gS = z((b.nconfig, 6)) if gS is None else gS.to(dev, torch.float64).contiguous()
        gsp, gmo, gra = eng.adjoint_device(b.itypes, b.rijs, b.js, b.jtypes, b.counts, b.cfg, b.volumes, b.nconfig,
                                           gE, gF, gS)
        d0, d1, d2 = ctx.devices
        return gsp.to(d0), gmo.to(d1), gra.to(d2), None, None


def predict(params: dict, engine: MTPEngine, batch: DeviceBatch):
    return MTPFunction.apply(params["species"], params["basis"], params["radial"], engine, batch)


def weighted_loss(E, F, S, targets, weights=(1.0, 0.01, 0.001)):
    Et, Ft, St = targets
    we, wf, ws = weights
    return we * ((E - Et) ** 2).sum() + wf * ((F - Ft) ** 2).sum() + ws * ((S - St) ** 2).sum()


class Trainer:
    """Minimal gradient-descent loop (the optimiser itself is plain torch)."""

    def __init__(self, engine: MTPEngine, species, moment, radial, lr: float = 1e-3, device="cuda"):
        self.engine = engine
        self.params = {
            "species": torch.tensor(np.asarray(species), dtype=torch.float64, device=device, requires_grad=True),
            "basis": torch.tensor(np.asarray(moment), dtype=torch.float64, device=device, requires_grad=True),
            "radial": torch.tensor(np.asarray(radial), dtype=torch.float64, device=device, requires_grad=True),
        }
        self.opt = torch.optim.Adam(self.params.values(), lr=lr)

    def step(self, batch: DeviceBatch, targets, weights=(1.0, 0.01, 0.001)) -> float:
        self.opt.zero_grad(set_to_none=True)
        E, F, S = predict(self.params, self.engine, batch)
        L = weighted_loss(E, F, S, targets, weights)
        L.backward()
        self.opt.step()
        return float(L.detach())


# ----------------------------------------------------------------------------
# Training pipeline around the adjoint: data, linear least squares, L-BFGS
# ----------------------------------------------------------------------------

def batch_from_configs(configs, cutoff: float, n_pad: Optional[int] = None, device="cuda"):
    """DeviceBatch and (E, F, sigma) targets from ``cfg_file.Configuration`` s.

    Neighbour rows hold every periodic image inside ``cutoff``; the stress
    target is -PlusStress / V (motep_original_files/old_io/mlip/cfg.py:131-134).
    Every configuration needs a Supercell, energy, forces and PlusStress.
    """
    from . import synth
    nds, E, F, S = [], [], [], []
    for k, c in enumerate(configs):
        if c.cell is None or c.energy is None or c.forces is None or c.plus_stress is None:
            raise ValueError(f"configuration {k} lacks a Supercell, Energy, forces or PlusStress")
        st = synth.Structure(np.asarray(c.positions, dtype=np.float64), np.asarray(c.cell, dtype=np.float64),
                             np.asarray(c.types, dtype=np.int32))
        nds.append(synth.build_neighbors(st, cutoff, n_pad))
        E.append(c.energy)
        F.append(np.asarray(c.forces, dtype=np.float64))
        S.append(c.stress)
    nd, cfg, _, vols = synth.pack_batch(nds, n_pad)
    batch = DeviceBatch.from_numpy(nd, cfg, vols, device=device)
    T = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64), device=device)
    return batch, (T(E), T(np.concatenate(F)), T(np.stack(S)))


def solve_lls_basis(engine: MTPEngine, batch: DeviceBatch, targets, species, radial,
                    weights=(1.0, 0.01, 0.001), method: str = "dense", max_iter: int = 500, rtol: float = 1e-10):
    """Moment (basis) coefficients minimising the weighted loss with the
    species and radial coefficients held fixed.

    The reference builds the Jacobian of all (E, F, sigma) targets with
    ``jax.jacfwd`` and calls ``lstsq`` (motep_jax_train_import.py:604-683).
    The predictions are affine in the basis coefficients theta,
    pred(theta) = pred(0) + X theta, so:

    * ``method="dense"`` (default, the reference's solve): column a of X is
      one batched GPU forward with theta = e_a minus pred(0) (Sa forwards);
      the weighted problem is solved on the GPU by a thin SVD with the
      minimum-norm cut-off of lstsq(rcond=None): singular values below
      eps * max(rows, Sa) * s_max are dropped.
    * ``method="cg"``: matrix-free conjugate gradients on the normal
      equations (one forward and one adjoint launch per iteration, no
      Jacobian in memory); slow to converge on ill-conditioned bases.

    Returns (theta [Sa] tensor on the batch's device, info dict).
    """
    b = batch
    dev = b.rijs.device
    sw = [float(np.sqrt(w)) for w in weights]
    sp = np.asarray(species, dtype=np.float64)
    ra = np.asarray(radial, dtype=np.float64)
    Sa = engine.alpha_scalar_moments

    def fwd(theta: torch.Tensor):
        engine.set_coeffs(sp, theta.detach().double().cpu().numpy(), ra)
        E, F, S = engine.batch_device(b.itypes, b.rijs, b.js, b.jtypes, b.counts, b.cfg, b.volumes, b.nconfig)
        return torch.cat([sw[0] * E, sw[1] * F.reshape(-1), sw[2] * S.reshape(-1)])

    nE, nF = b.nconfig, 3 * b.natoms

    def adj(u: torch.Tensor):
        gE = (sw[0] * u[:nE]).contiguous()
        gF = (sw[1] * u[nE:nE + nF]).reshape(b.natoms, 3).contiguous()
        gS = (sw[2] * u[nE + nF:]).reshape(b.nconfig, 6).contiguous()
        _, gmo, _ = engine.adjoint_device(b.itypes, b.rijs, b.js, b.jtypes, b.counts, b.cfg, b.volumes, b.nconfig,
                                          gE, gF, gS)
        return gmo

    zero = torch.zeros(Sa, dtype=torch.float64, device=dev)
    offset = fwd(zero)
    Et, Ft, St = targets
    y = torch.cat([sw[0] * Et.to(dev, torch.float64), sw[1] * Ft.to(dev, torch.float64).reshape(-1),
                   sw[2] * St.to(dev, torch.float64).reshape(-1)]) - offset
    if method == "dense":
        X = torch.empty((y.shape[0], Sa), dtype=torch.float64, device=dev)
        for a in range(Sa):
            e = zero.clone()
            e[a] = 1.0
            X[:, a] = fwd(e) - offset
        U, sv, Vh = torch.linalg.svd(X, full_matrices=False)
        cut = torch.finfo(torch.float64).eps * max(X.shape) * sv[0]
        keep = sv > cut
        theta = Vh[keep].T @ ((U[:, keep].T @ y) / sv[keep])
        resid = X @ theta - y
        return theta, {"method": "dense", "rank": int(keep.sum()), "loss": float(resid @ resid)}
    if method != "cg":
        raise ValueError("method must be 'dense' or 'cg'")
    theta = zero.clone()
    r = adj(y)
    p = r.clone()
    rs = float(r @ r)
    rs0 = rs
    it = 0
    while it < max_iter and rs > (rtol ** 2) * rs0 and rs > 0.0:
        q = fwd(p) - offset
        qq = float(q @ q)
        if qq <= 0.0:
            break
        alpha = rs / qq
        theta += alpha * p
        r -= alpha * adj(q)
        rs_new = float(r @ r)
        p = r + (rs_new / rs) * p
        rs = rs_new
        it += 1
    resid = fwd(theta) - offset - y
    return theta, {"method": "cg", "iterations": it, "normal_residual": (rs / rs0) ** 0.5 if rs0 > 0 else 0.0,
                   "loss": float(resid @ resid)}


def fit_lbfgs(engine: MTPEngine, batch: DeviceBatch, targets, params: dict, weights=(1.0, 0.01, 0.001),
              steps: int = 100, lr: float = 1.0, decay_rate: float = 1.0, transition_steps: int = 1000,
              clip_norm: Optional[float] = None, threshold: float = 0.0, min_steps: int = 0,
              val_batch: Optional[DeviceBatch] = None, val_targets=None, history_size: int = 10,
              max_backtrack: int = 40):
    """L-BFGS on all coefficients with the GPU forward and adjoint.

    Follows the reference's loop (training/motep_jax_train_function.py:103-213):
    per step one loss-and-gradient evaluation (forward + adjoint launch), a
    search direction from the two-loop recursion over the last
    ``history_size`` curvature pairs (initial scaling s.y / y.y), the
    gradient clipped to a global norm ``clip_norm`` for the direction, a
    learning rate ``lr * decay_rate ** (step // transition_steps)`` (staircase
    exponential decay), and a stop once at least ``min_steps`` steps are done
    and the loss fell by no more than ``threshold``.  The step length comes
    from a backtracking Armijo search that needs forward launches only; the
    first step, before any curvature pair exists, starts from
    2 L / |g|^2 along -g (the Gauss-Newton length of a least-squares loss
    along the gradient), so badly scaled problems, where gradients of 1e7
    meet losses of 1e-2, start sensibly.  ``params`` holds float64 tensors
    ``species``, ``basis``, ``radial`` (updated in place).  Returns a dict with
    the loss history (and the validation loss history for a validation batch).
    """
    keys = ("species", "basis", "radial")
    shapes = [params[k].shape for k in keys]
    sizes = [params[k].numel() for k in keys]

    def unflat(x):
        out, o = {}, 0
        for k, sh, n in zip(keys, shapes, sizes):
            out[k] = x[o:o + n].view(sh)
            o += n
        return out

    def f_only(x, b=batch, t=targets):
        with torch.no_grad():
            return float(weighted_loss(*predict(unflat(x), engine, b), t, weights))

    def f_and_g(x):
        q = {k: v.detach().clone().requires_grad_(True) for k, v in unflat(x).items()}
        L = weighted_loss(*predict(q, engine, batch), targets, weights)
        L.backward()
        return float(L.detach()), torch.cat([q[k].grad.reshape(-1) for k in keys])

    x = torch.cat([params[k].detach().reshape(-1).to(torch.float64) for k in keys])
    f, g = f_and_g(x)
    S, Y = [], []
    hist, vhist = [], []
    for step in range(steps):
        lr_t = lr * decay_rate ** (step // transition_steps)
        gd = g
        if clip_norm is not None:
            n = float(g.norm())
            if n > clip_norm:
                gd = g * (clip_norm / n)
        # two-loop recursion
        q = gd.clone()
        alphas = []
        for s_, y_ in zip(reversed(S), reversed(Y)):
            a = float(s_ @ q) / float(y_ @ s_)
            q -= a * y_
            alphas.append(a)
        if S:
            q *= float(S[-1] @ Y[-1]) / float(Y[-1] @ Y[-1])
        else:
            gg = float(gd @ gd)
            q *= (2.0 * f / gg) if gg > 0 else 0.0
        for (s_, y_), a in zip(zip(S, Y), reversed(alphas)):
            b_ = float(y_ @ q) / float(y_ @ s_)
            q += (a - b_) * s_
        d = -q
        slope = float(g @ d)
        if not slope < 0.0:          # not a descent direction: restart from the gradient
            S.clear()
            Y.clear()
            gg = float(gd @ gd)
            d = -gd * ((2.0 * f / gg) if gg > 0 else 0.0)
            slope = float(g @ d)
        t = lr_t
        f_new = f
        accepted = False
        for _ in range(max_backtrack):
            f_try = f_only(x + t * d)
            if np.isfinite(f_try) and f_try <= f + 1e-4 * t * slope:
                f_new = f_try
                accepted = True
                break
            t *= 0.5
        if accepted:
            x_new = x + t * d
            f_new, g_new = f_and_g(x_new)
            s_, y_ = x_new - x, g_new - g
            if float(s_ @ y_) > 1e-12 * float(s_.norm()) * float(y_.norm()):
                S.append(s_)
                Y.append(y_)
                if len(S) > history_size:
                    S.pop(0)
                    Y.pop(0)
            x, g = x_new, g_new
        prev, f = f, f_new
        hist.append(f)
        if val_batch is not None:
            vhist.append(f_only(x, val_batch, val_targets))
        if not accepted or (step + 1 >= min_steps and prev > f and prev - f <= threshold):
            break
    with torch.no_grad():
        for k, v in unflat(x).items():
            params[k].copy_(v)
    out = {"loss_history": hist, "steps": len(hist)}
    if val_batch is not None:
        out["val_loss_history"] = vhist
    return out
