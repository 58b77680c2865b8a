"""The allocation-free entry point against the regular one (GPU).

mtp_compute_device_noalloc serves callers that cannot let a library allocate
device memory (for example code running inside CUDA-graph stream capture, or
under a memory pool that owns the GPU).  It keeps its scratch in one fixed
device array shared by every call, so this checks, through the C ABI, that two
calls in a row both reproduce mtp_compute_device to the same tolerance the
other GPU tests use, and that inputs above its stated limits are rejected.

This file is collected last on purpose: a failure here leaves every other test
already run.  It passes alone in a fresh process as well.
"""

import numpy as np
import pytest
import torch

from conftest import golden_case, potential_path
from mtp_b200 import _lib
from mtp_b200.engine import MTPEngine

pytestmark = pytest.mark.gpu
# FP64: the bar of every FP64 parity test.  Mixed: both entry points may pick
# different launch shapes (summation orders) in FP32, so the bar is the FP32
# rounding level, far inside the mixed error budget (0.1 meV/atom, 1 meV/A).
REL = {"fp64": 1e-10, "mixed": 1e-5}


def _rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(1e-300, np.abs(b).max()))


@pytest.mark.parametrize("tag,precision", [("bcc54_L16", "fp64"), ("small_L20", "fp64"), ("fcc32_L24", "fp64"),
                                           ("cfg0", "mixed")])
def test_noalloc_matches_regular_entry_point_twice(tag, precision):
    g = golden_case(tag)
    path = potential_path(str(g["potential"]))
    N, n = g["js"].shape
    dev = torch.device("cuda")
    T = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=dev)
    it, rij, js, jt, cnt = (T(g["itypes"], torch.int32), T(g["rijs"], torch.float64), T(g["js"], torch.int32),
                            T(g["jtypes"], torch.int32), T(g["counts"], torch.int32))
    with MTPEngine(path, N, n, precision=precision) as eng:
        E0, F0, W0 = eng.compute_device(it, rij, js, jt, cnt)
        torch.cuda.synchronize()
        eng.sync_status()
        ref = (float(E0.cpu()[0]), F0.cpu().numpy(), W0.cpu().numpy())
        for _ in range(2):
            E = torch.full((1,), float("nan"), dtype=torch.float64, device=dev)
            F = torch.full((N, 3), float("nan"), dtype=torch.float64, device=dev)
            W = torch.full((6,), float("nan"), dtype=torch.float64, device=dev)
            eng.compute_device_noalloc(it, rij, js, jt, cnt, E, F, W)
            torch.cuda.synchronize()
            eng.sync_status()
            tol = REL[precision]
            assert abs(float(E.cpu()[0]) - ref[0]) <= tol * abs(ref[0])
            assert _rel(F.cpu().numpy(), ref[1]) <= tol
            assert _rel(W.cpu().numpy(), ref[2]) <= tol


def test_noalloc_rejects_inputs_above_its_limits():
    path = potential_path("cfg0_L16_S1.mtp")
    n_over = _lib.NOALLOC_MAX_ATOMS + 1
    dev = torch.device("cuda")
    with MTPEngine(path, n_over, 16) as eng:
        it = torch.zeros(n_over, dtype=torch.int32, device=dev)
        rij = torch.zeros((n_over, 16, 3), dtype=torch.float64, device=dev)
        js = torch.full((n_over, 16), -1, dtype=torch.int32, device=dev)
        cnt = torch.zeros(n_over, dtype=torch.int32, device=dev)
        E = torch.zeros(1, dtype=torch.float64, device=dev)
        F = torch.zeros((n_over, 3), dtype=torch.float64, device=dev)
        W = torch.zeros(6, dtype=torch.float64, device=dev)
        with pytest.raises(_lib.MTPError) as ei:
            eng.compute_device_noalloc(it, rij, js, js, cnt, E, F, W)
        assert ei.value.code == 3
        assert "allocation-free limit" in str(ei.value)
    # too many neighbour slots for the fixed scratch, with an atom count under
    # the atom limit: 8,193 atoms x 32 slots = 262,176 > MTP_NOALLOC_MAX_SLOTS
    m, stride = _lib.NOALLOC_MAX_SLOTS // 32 + 1, 32
    assert m <= _lib.NOALLOC_MAX_ATOMS and m * stride > _lib.NOALLOC_MAX_SLOTS
    with MTPEngine(path, m, stride) as eng:
        it = torch.zeros(m, dtype=torch.int32, device=dev)
        rij = torch.zeros((m, stride, 3), dtype=torch.float64, device=dev)
        js = torch.full((m, stride), -1, dtype=torch.int32, device=dev)
        cnt = torch.zeros(m, dtype=torch.int32, device=dev)
        E = torch.zeros(1, dtype=torch.float64, device=dev)
        F = torch.zeros((m, 3), dtype=torch.float64, device=dev)
        W = torch.zeros(6, dtype=torch.float64, device=dev)
        with pytest.raises(_lib.MTPError) as ei:
            eng.compute_device_noalloc(it, rij, js, js, cnt, E, F, W)
        assert ei.value.code == 3
        assert "neighbour slots" in str(ei.value)
