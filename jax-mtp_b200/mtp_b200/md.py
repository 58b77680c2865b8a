"""Device-resident NVE molecular dynamics on the CUDA engine.

One MD step (LAMMPS 'metal' units, velocity Verlet as in LAMMPS fix nve):

    v += dt/2 F/m ; x += dt v              (mtp_verlet_device, stage 1)
    every `rebuild_every` steps: neighbour rows from a device cell list with
        cutoff max_dist + skin             (mtp_neighbors_device)
    r_ij = x_j - x_i + image . H           (mtp_pack_rij_device)
    E, F, W                                (mtp_compute_device)
    v += dt/2 F/m                          (mtp_verlet_device, stage 2)

Everything stays on the GPU; a step can be captured as a CUDA graph (one
graph for a rebuild step, one for a reuse step).  This replaces the
reference's per-step host work in PairJaxMTP::compute
(pair_style_files/pair_jax_mtp.cpp:69-207) and the CPython call of the
bridge (zero_overhead.cpp:171-272) for device-resident runs.
"""

from __future__ import annotations

import math
from typing import Optional, Sequence

import numpy as np
import torch

from .engine import MTPEngine
from .synth import MVV2E, Structure

__all__ = ["DeviceMD"]


class DeviceMD:
    def __init__(self, engine: MTPEngine, s: Structure, masses: Sequence[float], velocities: Optional[np.ndarray] = None,
                 dt: float = 0.001, skin: float = 0.3, rebuild_every: int = 10, stride: int = 64,
                 list_cutoff: float = 5.0, device="cuda"):
        self.eng = engine
        self.dev = torch.device(device)
        self.N = s.natoms
        self.cell = np.asarray(s.cell, dtype=np.float64)
        self.volume = float(abs(np.linalg.det(self.cell)))
        self.masses = np.asarray(masses, dtype=np.float64)
        self.dt = float(dt)
        self.rebuild_every = int(rebuild_every)
        self.cutoff = float(list_cutoff) + float(skin)
        self.stride = int(stride)
        T = lambda a, dt_: torch.as_tensor(np.ascontiguousarray(a), dtype=dt_, device=self.dev)
        self.x = T(s.positions, torch.float64)
        self.v = T(np.zeros((self.N, 3)) if velocities is None else velocities, torch.float64)
        self.types = T(s.types, torch.int32)
        self.f = torch.zeros((self.N, 3), dtype=torch.float64, device=self.dev)
        self.energy = torch.zeros(1, dtype=torch.float64, device=self.dev)
        self.virial = torch.zeros(6, dtype=torch.float64, device=self.dev)
        self.js = torch.empty((self.N, self.stride), dtype=torch.int32, device=self.dev)
        self.image = torch.empty((self.N, self.stride), dtype=torch.int32, device=self.dev)
        self.jtypes = torch.empty((self.N, self.stride), dtype=torch.int32, device=self.dev)
        self.counts = torch.empty(self.N, dtype=torch.int32, device=self.dev)
        self.rijs = torch.empty((self.N, self.stride, 3), dtype=torch.float64, device=self.dev)
        self.mass_of_atom = T(self.masses[np.asarray(s.types)], torch.float64)
        self.step_count = 0
        self._graphs = None
        # initial list and forces
        self._rebuild()
        self._forces(reuse=False)

    # -- pieces -------------------------------------------------------------
    def _rebuild(self):
        self.eng.neighbors_device(self.x, self.cell, self.types, self.cutoff, self.stride, self.js, self.image,
                                  self.jtypes, self.counts)

    def _forces(self, reuse: bool):
        self.eng.pack_rij_device(self.x, self.cell, self.js, self.image, self.counts, self.rijs)
        self.eng.compute_device(self.types, self.rijs, self.js, self.jtypes, self.counts, energy=self.energy,
                                forces=self.f, virial=self.virial, reuse_neighbors=reuse)

    def _step(self, rebuild: bool):
        self.eng.verlet_device(self.x, self.v, self.f, self.types, self.masses, self.dt, 1)
        if rebuild:
            self._rebuild()
        self._forces(reuse=not rebuild)
        self.eng.verlet_device(self.x, self.v, self.f, self.types, self.masses, self.dt, 2)

    # -- public ---------------------------------------------------------------
    def capture(self) -> None:
        """Capture the two step variants as CUDA graphs (after one warm-up of each)."""
        s = torch.cuda.Stream(self.dev)
        s.wait_stream(torch.cuda.current_stream(self.dev))
        with torch.cuda.stream(s):
            # warm-ups allocate every lazily sized buffer before capture
            saved = [t.clone() for t in (self.x, self.v, self.f)]
            self._step(True)
            self._step(False)
            for t, c in zip((self.x, self.v, self.f), saved):
                t.copy_(c)
            self._rebuild()
            self._forces(reuse=False)
        torch.cuda.current_stream(self.dev).wait_stream(s)
        torch.cuda.synchronize(self.dev)
        g_rebuild = torch.cuda.CUDAGraph()
        g_reuse = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g_rebuild):
            self._step(True)
        with torch.cuda.graph(g_reuse):
            self._step(False)
        self._graphs = (g_rebuild, g_reuse)
        self.eng.set_stream(torch.cuda.current_stream(self.dev).cuda_stream)

    def run(self, nsteps: int, graphs: bool = False) -> None:
        for _ in range(nsteps):
            self.step_count += 1
            rebuild = (self.step_count % self.rebuild_every) == 0
            if graphs:
                if self._graphs is None:
                    raise RuntimeError("call capture() first")
                self._graphs[0 if rebuild else 1].replay()
            else:
                self._step(rebuild)

    def kinetic_energy(self) -> float:
        ke = 0.5 * (self.mass_of_atom[:, None] * self.v * self.v).sum() * MVV2E
        return float(ke)

    def potential_energy(self) -> float:
        return float(self.energy[0])

    def total_energy(self) -> float:
        return self.kinetic_energy() + self.potential_energy()

    def temperature(self) -> float:
        from .synth import KB_EV
        return 2.0 * self.kinetic_energy() / (3.0 * self.N * KB_EV)

    def release(self) -> None:
        self._graphs = None
