"""ctypes wrapper of the C++ CPU restatement (oracle/mtp_cpu.cpp).

TEST INFRASTRUCTURE ONLY (checker and CPU baseline), never a product path.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

_SO = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_build", "libmtp_cpu.so")
_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            raise RuntimeError(f"{_SO} missing: run `make -C oracle`")
        L = ctypes.CDLL(_SO)
        P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.mtpcpu_create.restype = P
        L.mtpcpu_create.argtypes = [I, I, I, I, I, I, I, D, D, D, P, P, P, P, P, P]
        L.mtpcpu_destroy.argtypes = [P]
        L.mtpcpu_compute.restype = I
        L.mtpcpu_compute.argtypes = [P, I, I, P, P, P, P, P, I, P, P, P, P, P]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class CpuMTP:
    """The potential on the host, evaluated by the OpenMP restatement."""

    def __init__(self, pot):
        L = _load()
        self._keep = [np.ascontiguousarray(pot.radial_coeffs, dtype=np.float64),
                      np.ascontiguousarray(pot.alpha_index_basic, dtype=np.int32),
                      np.ascontiguousarray(pot.alpha_index_times, dtype=np.int32).reshape(-1, 4),
                      np.ascontiguousarray(pot.alpha_moment_mapping, dtype=np.int32),
                      np.ascontiguousarray(pot.species_coeffs, dtype=np.float64),
                      np.ascontiguousarray(pot.moment_coeffs, dtype=np.float64)]
        r, b, t, m, s, mo = self._keep
        self._h = L.mtpcpu_create(pot.species_count, pot.radial_funcs_count, pot.radial_basis_size,
                                  pot.alpha_moments_count, len(b), len(t), len(m), pot.scaling, pot.min_dist,
                                  pot.max_dist, _p(r), _p(b), _p(t), _p(m), _p(s), _p(mo))

    def __del__(self):
        if getattr(self, "_h", None):
            _load().mtpcpu_destroy(self._h)
            self._h = None

    def compute(self, itypes, rijs, js, jtypes, counts=None, nthreads: int = 0):
        it = np.ascontiguousarray(itypes, dtype=np.int32)
        N = len(it)
        r = np.ascontiguousarray(rijs, dtype=np.float64)
        stride = r.shape[1]
        j = np.ascontiguousarray(js, dtype=np.int32)
        t = np.ascontiguousarray(jtypes, dtype=np.int32)
        c = None if counts is None else np.ascontiguousarray(counts, dtype=np.int32)
        e = np.zeros(1)
        site = np.zeros(N)
        F = np.zeros((N, 3))
        W = np.zeros(6)
        g = np.zeros((N, stride, 3))
        bad = _load().mtpcpu_compute(self._h, N, stride, _p(it), _p(r), _p(j), _p(t),
                                     None if c is None else _p(c), int(nthreads), _p(e), _p(site), _p(F), _p(W), _p(g))
        if bad:
            raise ValueError("species index out of range")
        return {"energy": float(e[0]), "site_energies": site, "forces": F, "virial": W, "pair_grads": g}
