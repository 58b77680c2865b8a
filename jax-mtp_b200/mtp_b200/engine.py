"""Python front end of the CUDA engine (host NumPy and device PyTorch paths).

``MTPEngine`` wraps one handle of the C ABI.  Its arguments follow the
reference evaluator's dynamic arguments (jax_backend.py:374-392):
``itypes [A]``, ``js [A, n]``, ``rijs [A, n, 3]``, ``jtypes [A, n]`` and the
cell volume; neighbour counts are optional (empty slots carry ``jtype < 0``,
as the reference bridge pads them, zero_overhead.cpp:76-92).
"""

from __future__ import annotations

import ctypes
from typing import Dict, Optional

import numpy as np

from . import _lib
from ._lib import EATOM, EFLAG, REUSE_NEIGHBORS, VATOM, VFLAG, check, lib

__all__ = ["MTPEngine", "pinned_empty", "stress_from_virial", "virial_from_stress"]


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _c(a, dtype) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=dtype)


class _PinnedBlock:
    """Page-locked bytes from mtp_host_alloc, freed with the last array viewing them."""

    def __init__(self, nbytes: int):
        p = ctypes.c_void_p()
        check(lib().mtp_host_alloc(nbytes, ctypes.byref(p)), None)
        self.ptr = p.value
        self.__array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (self.ptr, False), "version": 3}

    def __del__(self):
        if getattr(self, "ptr", None):
            lib().mtp_host_free(self.ptr)
            self.ptr = None


def pinned_empty(shape, dtype=np.float64) -> np.ndarray:
    """Uninitialised page-locked host array: ``compute`` moves it by DMA
    instead of through the driver's staging copy of pageable memory."""
    dt = np.dtype(dtype)
    n = int(np.prod(shape, dtype=np.int64)) * dt.itemsize
    raw = np.asarray(_PinnedBlock(max(n, dt.itemsize)))
    return raw[:n].view(dt).reshape(shape)


def stress_from_virial(virial: np.ndarray, volume: float) -> np.ndarray:
    """LAMMPS virial (xx,yy,zz,xy,xz,yz, energy) -> reference stress (xx,yy,zz,yz,xz,xy, /V)."""
    w = np.asarray(virial)
    return -np.array([w[..., 0], w[..., 1], w[..., 2], w[..., 5], w[..., 4], w[..., 3]]).T / volume


def virial_from_stress(stress: np.ndarray, volume: float) -> np.ndarray:
    s = np.asarray(stress)
    return -volume * np.array([s[..., 0], s[..., 1], s[..., 2], s[..., 5], s[..., 4], s[..., 3]]).T


class MTPEngine:
    """One evaluator handle (owns device buffers sized by max_atoms x max_nbr)."""

    def __init__(self, mtp_path: str, max_atoms: int, max_nbr: int, cutoff: Optional[float] = None,
                 precision: str = "fp64", debug_level: int = 0):
        L = lib()
        self.precision = precision
        prec = {"fp64": _lib.PRECISION_FP64, "mixed": _lib.PRECISION_MIXED}[precision]
        h = ctypes.c_void_p()
        code = L.mtp_create(str(mtp_path).encode(), int(max_atoms), int(max_nbr),
                            float(cutoff if cutoff is not None else 1e30), int(debug_level), prec,
                            ctypes.byref(h))
        check(code, None)
        self._h = h
        self.max_atoms = int(max_atoms)
        self.max_nbr = int(max_nbr)
        info = np.zeros(8, dtype=np.int32)
        check(L.mtp_get_info(self._h, _ptr(info)), self._h)
        (self.species_count, self.radial_funcs_count, self.radial_basis_size, self.alpha_moments_count,
         self.alpha_index_basic_count, self.alpha_index_times_count, self.alpha_scalar_moments,
         self.max_degree) = (int(x) for x in info)

    # ------------------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().mtp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    def stats(self) -> Dict[str, float]:
        """Host-buffer call statistics (mtp_get_stats)."""
        out = np.zeros(4)
        check(lib().mtp_get_stats(self._h, _ptr(out)), self._h)
        return {"calls": int(out[0]), "total_ms": float(out[1]), "graph_captures": int(out[2]),
                "graph_replays": int(out[3])}

    def set_coeffs(self, species=None, moment=None, radial=None) -> None:
        sp = None if species is None else _c(species, np.float64)
        mo = None if moment is None else _c(moment, np.float64)
        ra = None if radial is None else _c(radial, np.float64)
        check(lib().mtp_set_coeffs(self._h, _ptr(sp), _ptr(mo), _ptr(ra)), self._h)

    def set_stream(self, stream_handle: int) -> None:
        """Work on this cudaStream_t (0 = the legacy default stream, as torch's default)."""
        check(lib().mtp_set_stream(self._h, ctypes.c_void_p(stream_handle)), self._h)

    def use_own_stream(self) -> None:
        check(lib().mtp_use_own_stream(self._h), self._h)

    def set_launch(self, threads: int, blocks_per_sm: int = 0, atoms_per_block: int = 0) -> None:
        check(lib().mtp_set_launch(self._h, int(threads), int(blocks_per_sm), int(atoms_per_block)), self._h)

    def launch(self) -> Dict[str, int]:
        out = np.zeros(5, dtype=np.int32)
        check(lib().mtp_get_launch(self._h, _ptr(out)), self._h)
        return {"threads": int(out[0]), "blocks": int(out[1]), "smem": int(out[2]), "blocks_per_sm": int(out[3]),
                "atoms_per_block": int(out[4])}

    def sync_status(self) -> None:
        check(lib().mtp_sync_status(self._h), self._h)

    # ------------------------------------------------------------------
    def compute(self, itypes, rijs, js, jtypes, counts=None, eatom: bool = True, vatom: bool = False):
        """Host arrays in, host arrays out (synchronous).  Returns energy, forces,
        LAMMPS virial (xx,yy,zz,xy,xz,yz), site energies and optionally per-atom virials."""
        it = _c(itypes, np.int32)
        N = it.shape[0]
        r = _c(rijs, np.float64)
        stride = r.shape[1] if N else max(1, self.max_nbr)
        j = _c(js, np.int32)
        t = _c(jtypes, np.int32)
        cnt = None if counts is None else _c(counts, np.int32)
        F = np.zeros((N, 3))
        vir = np.zeros(6)
        e = np.zeros(1)
        ea = np.zeros(N) if eatom else None
        va = np.zeros((N, 6)) if vatom else None
        flags = EFLAG | VFLAG | (EATOM if eatom else 0) | (VATOM if vatom else 0)
        code = lib().mtp_compute(self._h, N, stride, _ptr(it), _ptr(r), _ptr(j), _ptr(t), _ptr(cnt), flags,
                                 _ptr(e), _ptr(F), _ptr(vir), _ptr(ea), _ptr(va))
        check(code, self._h)
        out = {"energy": float(e[0]), "forces": F, "virial": vir}
        if eatom:
            out["site_energies"] = ea
        if vatom:
            out["vatom"] = va
        return out

    def compute_positions(self, nlocal: int, x, species, owner, neigh, numneigh, eatom: bool = True,
                          vatom: bool = False):
        """Host arrays in, rows built on the device (mtp_compute_positions):
        x [nall, 3] local atoms then ghosts, species [nall] (0-based), owner
        [nall] (local owner index or -1), neigh [nlocal, list_stride] candidate
        indices into [0, nall), numneigh [nlocal].  Returns what ``compute`` returns."""
        xa = _c(x, np.float64)
        sp = _c(species, np.int32)
        ow = _c(owner, np.int32)
        nb = _c(neigh, np.int32)
        nn = _c(numneigh, np.int32)
        nall = int(sp.shape[0])
        stride = int(nb.shape[1]) if nb.ndim == 2 else 0
        F = np.zeros((nlocal, 3))
        vir = np.zeros(6)
        e = np.zeros(1)
        ea = np.zeros(nlocal) if eatom else None
        va = np.zeros((nlocal, 6)) if vatom else None
        flags = EFLAG | VFLAG | (EATOM if eatom else 0) | (VATOM if vatom else 0)
        code = lib().mtp_compute_positions(self._h, nlocal, nall, _ptr(xa), _ptr(sp), _ptr(ow), stride, _ptr(nb),
                                           _ptr(nn), flags, _ptr(e), _ptr(F), _ptr(vir), _ptr(ea), _ptr(va))
        check(code, self._h)
        out = {"energy": float(e[0]), "forces": F, "virial": vir}
        if eatom:
            out["site_energies"] = ea
        if vatom:
            out["vatom"] = va
        return out

    def execute_potential(self, itypes, rijs, js, jtypes, counts, volume: float):
        """The reference bridge signature (zero_overhead.hpp:58-64): per-atom row
        pointers in, (ok, energy, forces [N,3], stress [6] in the reference's
        convention) out."""
        it = _c(itypes, np.int32)
        N = it.shape[0]
        rows_r = [_c(rijs[i], np.float64) for i in range(N)]
        rows_j = [_c(js[i], np.int32) for i in range(N)]
        rows_t = [_c(jtypes[i], np.int32) for i in range(N)]
        cnt = _c(counts, np.int32)
        P = ctypes.c_void_p * max(1, N)
        pr = P(*[x.ctypes.data for x in rows_r])
        pj = P(*[x.ctypes.data for x in rows_j])
        pt = P(*[x.ctypes.data for x in rows_t])
        F = np.zeros((N, 3))
        pf = P(*[F[i].ctypes.data for i in range(N)])
        e = np.zeros(1)
        st = np.zeros(6)
        code = lib().mtp_execute_potential(self._h, N, int(cnt.sum()), ctypes.cast(pr, ctypes.c_void_p),
                                           _ptr(it), ctypes.cast(pj, ctypes.c_void_p), _ptr(cnt),
                                           ctypes.cast(pt, ctypes.c_void_p), float(volume), _ptr(e),
                                           ctypes.cast(pf, ctypes.c_void_p), _ptr(st))
        check(code, self._h)
        return float(e[0]), F, st

    # ------------------------------------------------------------------
    # device (PyTorch) paths
    # ------------------------------------------------------------------
    def compute_device(self, itypes, rijs, js, jtypes, counts=None, *, energy=None, forces=None, virial=None,
                       eatom=None, vatom=None, reuse_neighbors: bool = False, stream=None):
        """Device tensors in/out (torch, contiguous).  Asynchronous on ``stream``
        (default: torch's current stream).  Outputs are allocated when not given."""
        import torch
        N = int(itypes.shape[0])
        stride = int(rijs.shape[1])
        dev = rijs.device
        if forces is None:
            forces = torch.empty((N, 3), dtype=torch.float64, device=dev)
        if energy is None:
            energy = torch.empty(1, dtype=torch.float64, device=dev)
        if virial is None:
            virial = torch.empty(6, dtype=torch.float64, device=dev)
        flags = EFLAG | VFLAG
        if eatom is not None:
            flags |= EATOM
        if vatom is not None:
            flags |= VATOM
        if reuse_neighbors:
            flags |= REUSE_NEIGHBORS
        st = torch.cuda.current_stream(dev) if stream is None else stream
        self.set_stream(st.cuda_stream)
        P = lambda t: None if t is None else ctypes.c_void_p(t.data_ptr())
        code = lib().mtp_compute_device(self._h, N, stride, P(itypes), P(rijs), P(js), P(jtypes), P(counts), flags,
                                        P(energy), P(forces), P(virial), P(eatom), P(vatom))
        check(code, self._h)
        return energy, forces, virial

    def compute_positions_device(self, nlocal: int, x, species, owner, neigh, numneigh, *, energy=None,
                                 forces=None, virial=None, eatom=None, vatom=None, stream=None):
        """Device tensors in/out (mtp_compute_positions_device): x [nall, 3]
        float64, species / owner [nall] int32, neigh [nlocal, list_stride] and
        numneigh [nlocal] int32.  Asynchronous on ``stream`` (default: torch's
        current stream); errors are read with ``sync_status``."""
        import torch
        dev = x.device
        nall = int(species.shape[0])
        stride = int(neigh.shape[1])
        if forces is None:
            forces = torch.empty((nlocal, 3), dtype=torch.float64, device=dev)
        if energy is None:
            energy = torch.empty(1, dtype=torch.float64, device=dev)
        if virial is None:
            virial = torch.empty(6, dtype=torch.float64, device=dev)
        flags = EFLAG | VFLAG | (EATOM if eatom is not None else 0) | (VATOM if vatom is not None else 0)
        st = torch.cuda.current_stream(dev) if stream is None else stream
        self.set_stream(st.cuda_stream)
        P = lambda t: None if t is None else ctypes.c_void_p(t.data_ptr())
        code = lib().mtp_compute_positions_device(self._h, nlocal, nall, P(x), P(species), P(owner), stride, P(neigh),
                                                  P(numneigh), flags, P(energy), P(forces), P(virial), P(eatom),
                                                  P(vatom))
        check(code, self._h)
        return energy, forces, virial

    def batch_device(self, itypes, rijs, js, jtypes, counts, cfg_of_atom, volumes, nconfig: int, stream=None):
        """Batched configurations: returns (energy [C], forces [N,3], stress [C,6] reference convention)."""
        import torch
        N = int(itypes.shape[0])
        dev = rijs.device
        E = torch.empty(nconfig, dtype=torch.float64, device=dev)
        F = torch.empty((N, 3), dtype=torch.float64, device=dev)
        S = torch.empty((nconfig, 6), dtype=torch.float64, device=dev)
        st = torch.cuda.current_stream(dev) if stream is None else stream
        self.set_stream(st.cuda_stream)
        P = lambda t: None if t is None else ctypes.c_void_p(t.data_ptr())
        code = lib().mtp_compute_batch_device(self._h, N, int(rijs.shape[1]), int(nconfig), P(itypes), P(rijs), P(js),
                                              P(jtypes), P(counts), P(cfg_of_atom), P(volumes), P(E), P(F), P(S))
        check(code, self._h)
        return E, F, S

    def adjoint_device(self, itypes, rijs, js, jtypes, counts, cfg_of_atom, volumes, nconfig: int, gE, gF, gS,
                       stream=None):
        """Gradient of sum(gE*E) + sum(gF*F) + sum(gS*S) w.r.t. (species, moment, radial) coefficients."""
        import torch
        N = int(itypes.shape[0])
        dev = rijs.device
        gsp = torch.empty(self.species_count, dtype=torch.float64, device=dev)
        gmo = torch.empty(self.alpha_scalar_moments, dtype=torch.float64, device=dev)
        gra = torch.empty((self.species_count, self.species_count, self.radial_funcs_count, self.radial_basis_size),
                          dtype=torch.float64, device=dev)
        st = torch.cuda.current_stream(dev) if stream is None else stream
        self.set_stream(st.cuda_stream)
        P = lambda t: None if t is None else ctypes.c_void_p(t.data_ptr())
        code = lib().mtp_adjoint_batch_device(self._h, N, int(rijs.shape[1]), int(nconfig), P(itypes), P(rijs), P(js),
                                              P(jtypes), P(counts), P(cfg_of_atom), P(volumes), P(gE.contiguous()),
                                              P(gF.contiguous()), P(gS.contiguous()), P(gsp), P(gmo), P(gra))
        check(code, self._h)
        return gsp, gmo, gra


def parse_info(path: str) -> Dict[str, int]:
    """Host-only parse of an .mtp file through the C++ reader."""
    out = np.zeros(8, dtype=np.int32)
    err = ctypes.create_string_buffer(512)
    code = lib().mtp_parse_info(str(path).encode(), _ptr(out), err, 512)
    if code != _lib.MTP_OK:
        raise _lib.MTPError(code, err.value.decode())
    keys = ["species_count", "radial_funcs_count", "radial_basis_size", "alpha_moments_count",
            "alpha_index_basic_count", "alpha_index_times_count", "alpha_scalar_moments", "max_degree"]
    return dict(zip(keys, (int(x) for x in out)))


def schedule_emulate(path: str, lanes: int, basic: np.ndarray, width: int = 4):
    """Run the contraction schedule on the host (test hook)."""
    info = parse_info(path)
    b = _c(basic, np.float64)
    m = np.zeros(info["alpha_moments_count"])
    dm = np.zeros(info["alpha_moments_count"])
    e = np.zeros(1)
    code = lib().mtp_schedule_emulate(str(path).encode(), int(lanes), int(width), _ptr(b), _ptr(m), _ptr(dm),
                                      _ptr(e))
    if code != _lib.MTP_OK:
        raise _lib.MTPError(code, "schedule emulation failed")
    return m, dm, float(e[0])


def measure_fma_peak():
    d = ctypes.c_double()
    f = ctypes.c_double()
    check(lib().mtp_measure_fma_peak(ctypes.byref(d), ctypes.byref(f)))
    return d.value, f.value


# ----------------------------------------------------------------------------
# device MD helpers (bound as methods below)
# ----------------------------------------------------------------------------
def _tp(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _neighbors_device(self, pos, cell, types, cutoff: float, stride: int, js, image, jtypes, counts, stream=None):
    """Device cell-list rows (see mtp_neighbors_device)."""
    import torch
    st = torch.cuda.current_stream(pos.device) if stream is None else stream
    self.set_stream(st.cuda_stream)
    c9 = _c(np.asarray(cell, dtype=np.float64).reshape(9), np.float64)
    code = lib().mtp_neighbors_device(self._h, int(pos.shape[0]), _tp(pos), _ptr(c9), _tp(types), float(cutoff),
                                      int(stride), _tp(js), _tp(image), _tp(jtypes), _tp(counts))
    check(code, self._h)


def _pack_rij_device(self, pos, cell, js, image, counts, rijs, stream=None):
    import torch
    st = torch.cuda.current_stream(pos.device) if stream is None else stream
    self.set_stream(st.cuda_stream)
    c9 = _c(np.asarray(cell, dtype=np.float64).reshape(9), np.float64)
    code = lib().mtp_pack_rij_device(self._h, int(pos.shape[0]), int(js.shape[1]), _tp(pos), _ptr(c9), _tp(js),
                                     _tp(image), _tp(counts), _tp(rijs))
    check(code, self._h)


def _verlet_device(self, x, v, f, types, masses, dt: float, stage: int, stream=None):
    import torch
    st = torch.cuda.current_stream(x.device) if stream is None else stream
    self.set_stream(st.cuda_stream)
    m = _c(masses, np.float64)
    code = lib().mtp_verlet_device(self._h, int(x.shape[0]), _tp(x), _tp(v), _tp(f), _tp(types), _ptr(m), len(m),
                                   float(dt), int(stage))
    check(code, self._h)


def _profile(self, enable: bool) -> None:
    check(lib().mtp_profile(self._h, 1 if enable else 0), self._h)


def _profile_read(self):
    ms = ctypes.c_double()
    n = ctypes.c_int()
    check(lib().mtp_profile_read(self._h, ctypes.byref(ms), ctypes.byref(n)), self._h)
    return ms.value, n.value


MTPEngine.neighbors_device = _neighbors_device
MTPEngine.pack_rij_device = _pack_rij_device
MTPEngine.verlet_device = _verlet_device
MTPEngine.profile = _profile
MTPEngine.profile_read = _profile_read


def _compute_device_noalloc(self, itypes, rijs, js, jtypes, counts, energy, forces, virial, stream=None):
    """mtp_compute_device_noalloc: the evaluation with no device allocation at all.

    For callers that cannot allocate device memory (inside CUDA-graph capture,
    under an external memory pool, or where an allocation's implicit device
    synchronisation is not allowed).  Outputs must be preallocated device
    tensors: energy [1], forces [N, 3], virial [6] (float64).  Calls that
    overlap on the GPU share one scratch array and race.
    """
    import torch
    st = torch.cuda.current_stream(rijs.device) if stream is None else stream
    self.set_stream(st.cuda_stream)
    code = lib().mtp_compute_device_noalloc(self._h, int(itypes.shape[0]), int(rijs.shape[1]), _tp(itypes),
                                             _tp(rijs), _tp(js), _tp(jtypes), _tp(counts), _tp(energy), _tp(forces),
                                             _tp(virial))
    check(code, self._h)


MTPEngine.compute_device_noalloc = _compute_device_noalloc
