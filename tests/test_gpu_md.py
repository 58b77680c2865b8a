"""Device neighbour rows, device MD and CUDA-graph capture (GPU)."""

import numpy as np
import pytest
import torch

from conftest import potential_path
from mtp_b200 import synth
from mtp_b200.engine import MTPEngine
from mtp_b200.md import DeviceMD

pytestmark = pytest.mark.gpu


def _rows(js, rij, counts):
    out = []
    for i in range(len(counts)):
        c = counts[i]
        keys = sorted((int(js[i, s]), tuple(np.round(rij[i, s], 9))) for s in range(c))
        out.append(keys)
    return out


@pytest.mark.parametrize("kind,a,reps,cut", [("fcc", 3.6, (4, 4, 4), 5.3), ("bcc", 2.87, (5, 5, 5), 5.0),
                                           ("hcp", 3.0, (4, 4, 3), 5.0), ("fcc", 3.6, (2, 2, 2), 5.3)])
def test_device_rows_match_host_builder(kind, a, reps, cut):
    s = synth.lattice_structure(kind, a, reps)
    rng = np.random.default_rng(3)
    s.positions = s.positions + rng.normal(0, 0.1, s.positions.shape)
    s.positions[::7] += s.cell[0] * 1.0      # some atoms outside the home cell
    s.types = rng.integers(0, 2, s.natoms).astype(np.int32)
    host = synth.build_neighbors(s, cut)
    stride = max(64, host.n_pad)
    dev = torch.device("cuda")
    with MTPEngine(potential_path("cfg1_L16_S2.mtp"), s.natoms, stride) as eng:
        x = torch.as_tensor(s.positions, device=dev)
        t = torch.as_tensor(s.types, device=dev)
        js = torch.empty((s.natoms, stride), dtype=torch.int32, device=dev)
        im = torch.empty_like(js)
        jt = torch.empty_like(js)
        cnt = torch.empty(s.natoms, dtype=torch.int32, device=dev)
        rij = torch.empty((s.natoms, stride, 3), dtype=torch.float64, device=dev)
        eng.neighbors_device(x, s.cell, t, cut, stride, js, im, jt, cnt)
        eng.pack_rij_device(x, s.cell, js, im, cnt, rij)
        torch.cuda.synchronize()
        eng.sync_status()
    c = cnt.cpu().numpy()
    assert np.array_equal(c, host.counts)
    assert _rows(js.cpu().numpy(), rij.cpu().numpy(), c) == _rows(host.js, host.rijs, host.counts)
    jtn = jt.cpu().numpy()
    for i in range(s.natoms):
        assert np.array_equal(jtn[i, :c[i]], s.types[js.cpu().numpy()[i, :c[i]]])


def test_row_overflow_reported():
    s = synth.lattice_structure("fcc", 3.6, (3, 3, 3))
    dev = torch.device("cuda")
    with MTPEngine(potential_path("cfg0_L16_S1.mtp"), s.natoms, 64) as eng:
        x = torch.as_tensor(s.positions, device=dev)
        t = torch.zeros(s.natoms, dtype=torch.int32, device=dev)
        js = torch.empty((s.natoms, 16), dtype=torch.int32, device=dev)
        im, jt = torch.empty_like(js), torch.empty_like(js)
        cnt = torch.empty(s.natoms, dtype=torch.int32, device=dev)
        eng.neighbors_device(x, s.cell, t, 5.0, 16, js, im, jt, cnt)
        from mtp_b200._lib import MTPError
        with pytest.raises(MTPError) as ei:
            eng.sync_status()
        assert ei.value.code == 3
        assert int(cnt.max()) == 16


def test_nve_energy_conservation_and_graph_replay():
    s = synth.lattice_structure("bcc", 2.87, (4, 4, 4))
    rng = np.random.default_rng(9)
    s.types = rng.integers(0, 2, s.natoms).astype(np.int32)
    v0 = synth.maxwell_boltzmann(s.natoms, 300.0, 55.845, seed=4)
    path = potential_path("cfg1md_L16_S2.mtp")
    with MTPEngine(path, s.natoms, 64) as eng:
        md = DeviceMD(eng, s, [55.845, 55.845], velocities=v0, dt=0.001, skin=0.3, rebuild_every=10, stride=64)
        e0 = md.total_energy()
        md.run(200)
        e1 = md.total_energy()
        eng.sync_status()
        drift = abs(e1 - e0) / s.natoms
        assert drift < 1e-4, drift            # eV/atom over 0.1 ps
        x_ref = md.x.clone()
    with MTPEngine(path, s.natoms, 64) as eng:
        md = DeviceMD(eng, s, [55.845, 55.845], velocities=v0, dt=0.001, skin=0.3, rebuild_every=10, stride=64)
        md.capture()
        md.run(200, graphs=True)
        torch.cuda.synchronize()
        eng.sync_status()
        assert torch.equal(md.x, x_ref)
        md.release()
