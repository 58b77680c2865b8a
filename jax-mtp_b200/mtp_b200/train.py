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

__all__ = ["DeviceBatch", "MTPFunction", "predict", "weighted_loss", "Trainer"]


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
