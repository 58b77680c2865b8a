"""Profiling harness (not part of the library's API): a bounded evaluation case
for profilers (ncu) and quick timing, the command every ncu summary of the
evaluation and adjoint kernels was captured with.

    python -m mtp_b200.profile_case --potential <file.mtp> --reps 32 --precision mixed --calls 3

Builds an fcc a=3.6 A crystal of reps^3 cells (4 reps^3 atoms) with thermal
displacements, device neighbour rows (cutoff max_dist + 0.3 A), and calls the
evaluation `--calls` times; prints the evaluation-kernel time per call
measured with CUDA events.  reps=32 gives 131,072 atoms and 200 MB of r_ij,
larger than the 126 MB L2, while staying a few GB on the device.
"""

from __future__ import annotations

import argparse
import json
import os

import numpy as np
import torch

from . import synth
from .engine import MTPEngine
from .mtp_file import read_mtp


_BYTE_UNITS = {"byte": 1.0, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9, "Tbyte": 1e12,
               "KB": 1e3, "MB": 1e6, "GB": 1e9}


def write_traffic(json_path: str, csv_path: str, key: str, kernel: str, scale: float, captured_atoms: int) -> dict:
    """DRAM bytes per launch of `kernel` from `ncu -i <rep> --page raw --csv`
    output (dram__bytes_read.sum + dram__bytes_write.sum, averaged over the
    captured launches), scaled by `scale` to the full workload, merged into
    the JSON data file under `key`."""
    import csv
    rows = list(csv.reader(open(csv_path)))
    # the header row names the columns (lines the profiled program printed may precede it)
    at = next(i for i, r in enumerate(rows) if "Kernel Name" in r)
    head, units, rows = rows[at], rows[at + 1], rows[at:]
    iname = head.index("Kernel Name")
    irx, iwx = head.index("dram__bytes_read.sum"), head.index("dram__bytes_write.sum")
    per = []
    for r in rows[2:]:
        if len(r) <= max(irx, iwx) or kernel not in r[iname]:
            continue
        rb = float(r[irx].replace(",", "")) * _BYTE_UNITS[units[irx]]
        wb = float(r[iwx].replace(",", "")) * _BYTE_UNITS[units[iwx]]
        per.append(rb + wb)
    if not per:
        raise SystemExit(f"no launch of {kernel!r} in {csv_path}")
    entry = {"bytes_per_launch_captured": sum(per) / len(per), "launches": len(per), "scale": scale,
             "captured_atoms": captured_atoms, "bytes_per_launch_full_workload": scale * sum(per) / len(per),
             "kernel": kernel}
    try:
        with open(json_path) as fh:
            data = json.load(fh)
    except (OSError, ValueError):
        data = {}
    data[key] = entry
    with open(json_path, "w") as fh:
        json.dump(data, fh, indent=1, sort_keys=True)
        fh.write("\n")
    return entry


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--write-traffic", metavar="JSON",
                    help="instead: merge the DRAM bytes per launch of --ncu-csv (ncu --page raw --csv) into JSON "
                         "under --key, scaled by --scale to the full workload")
    ap.add_argument("--ncu-csv")
    ap.add_argument("--key")
    ap.add_argument("--kernel", default="k_mtp_eval")
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--potential")
    ap.add_argument("--reps", type=int, default=32)
    ap.add_argument("--stride", type=int, default=64)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    ap.add_argument("--calls", type=int, default=3)
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--apb", type=int, default=0, help="atoms per block (0: automatic)")
    ap.add_argument("--sweep", action="store_true", help="time every (threads, atoms per block) shape")
    ap.add_argument("--training", type=int, default=0,
                    help="instead: a batch of this many training configurations (synth.training_batch, "
                         "32-512 atoms, seed 8); one batched forward, then --calls adjoint launches")
    ap.add_argument("--pair-call", action="store_true",
                    help="instead: the LAMMPS-size force call, bcc a=2.87 A 10^3 cells (2,000 atoms, 50/50 "
                         "species) with periodic ghosts and full lists (skin 0.3 A), --calls calls of "
                         "mtp_compute_positions on page-locked buffers (max_nbr 60, cutoff 5.0 A)")
    a = ap.parse_args(argv)
    if a.write_traffic:
        e = write_traffic(a.write_traffic, a.ncu_csv, a.key, a.kernel, a.scale, 4 * a.reps ** 3)
        print(json.dumps(e))
        return 0
    if not a.potential:
        ap.error("--potential is required")
    pot = read_mtp(a.potential)
    if a.pair_call:
        return pair_call_case(a, pot)
    if a.training:
        return training_case(a, pot)
    s = synth.config2_structure(a.reps)
    s.types = s.types % pot.species_count
    dev = torch.device("cuda")
    N = s.natoms
    with MTPEngine(a.potential, N, a.stride, precision=a.precision) as eng:
        if a.threads or a.apb:
            eng.set_launch(a.threads or 256, 0, a.apb)
        x = torch.as_tensor(s.positions, device=dev)
        t = torch.as_tensor(s.types, device=dev)
        js = torch.empty((N, a.stride), dtype=torch.int32, device=dev)
        im, jt = torch.empty_like(js), torch.empty_like(js)
        cnt = torch.empty(N, dtype=torch.int32, device=dev)
        rij = torch.empty((N, a.stride, 3), dtype=torch.float64, device=dev)
        eng.neighbors_device(x, s.cell, t, pot.max_dist + 0.3, a.stride, js, im, jt, cnt)
        eng.pack_rij_device(x, s.cell, js, im, cnt, rij)
        shapes = [(None, None)]
        if a.sweep:
            apbs = (1, 2) if a.precision == "fp64" else (1, 2, 4)
            shapes = [(th, ap) for th in (256, 512) for ap in apbs]
        for th, ap in shapes:
            if th is not None:
                eng.set_launch(th, 0, ap)
            eng.compute_device(t, rij, js, jt, cnt)          # warm-up, builds the incoming lists
            eng.profile(True)
            for k in range(a.calls):
                eng.compute_device(t, rij, js, jt, cnt, reuse_neighbors=True)
            ms, n = eng.profile_read()
            eng.profile(False)
            eng.sync_status()
            print(json.dumps({"atoms": N, "precision": a.precision, "eval_ms_per_call": ms / max(1, n),
                              "launch": eng.launch()}), flush=True)


def training_case(a, pot):
    """Batched forward + adjoint (training gradient) on synthetic configurations."""
    from .train import DeviceBatch
    dev = torch.device("cuda")
    structs = synth.training_batch(a.training, 32, 512, pot.species_count, seed=8)
    nds = [synth.build_neighbors(st, pot.max_dist) for st in structs]
    nd, cfg, _, vols = synth.pack_batch(nds)
    b = DeviceBatch.from_numpy(nd, cfg, vols, device=dev)
    with MTPEngine(a.potential, nd.natoms, nd.n_pad, precision=a.precision) as eng:
        E, F, S = eng.batch_device(b.itypes, b.rijs, b.js, b.jtypes, b.counts, b.cfg, b.volumes, b.nconfig)
        gE, gF, gS = torch.ones_like(E), 0.01 * torch.ones_like(F), 0.001 * torch.ones_like(S)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(a.calls):
            eng.adjoint_device(b.itypes, b.rijs, b.js, b.jtypes, b.counts, b.cfg, b.volumes, b.nconfig, gE, gF, gS)
        e1.record()
        torch.cuda.synchronize()
        eng.sync_status()
        print(json.dumps({"configs": b.nconfig, "atoms": nd.natoms, "n_pad": nd.n_pad,
                          "adjoint_ms_per_call": e0.elapsed_time(e1) / max(1, a.calls)}), flush=True)



def pair_call_case(a, pot):
    """Host wall clock of synchronous mtp_compute_positions calls (graph replay)."""
    import ctypes
    import time

    from ._lib import EFLAG, VFLAG, check, lib
    from .engine import pinned_empty
    s = synth.config1()
    s.types = s.types % pot.species_count
    x, owner, lists = synth.ghosts_and_lists(s, 5.3)
    N = s.natoms
    stride = max(len(c) for c in lists)
    buf = {"x": pinned_empty(x.shape), "sp": pinned_empty((len(x),), np.int32),
           "own": pinned_empty((len(x),), np.int32), "nb": pinned_empty((N, stride), np.int32),
           "num": pinned_empty((N,), np.int32), "e": pinned_empty((1,)), "F": pinned_empty((N, 3)),
           "w": pinned_empty((6,))}
    buf["x"][...] = x
    buf["sp"][...] = s.types[owner]
    buf["own"][...] = owner
    buf["nb"][...] = -1
    for i, c in enumerate(lists):
        buf["nb"][i, :len(c)] = c
        buf["num"][i] = len(c)
    P = lambda v: v.ctypes.data_as(ctypes.c_void_p)
    with MTPEngine(a.potential, N, 60, cutoff=5.0, precision=a.precision) as eng:
        eng.use_own_stream()

        def call():
            check(lib().mtp_compute_positions(eng.handle, N, len(x), P(buf["x"]), P(buf["sp"]), P(buf["own"]),
                                              stride, P(buf["nb"]), P(buf["num"]), EFLAG | VFLAG, P(buf["e"]),
                                              P(buf["F"]), P(buf["w"]), None, None), eng.handle)
        for _ in range(3):
            call()
        t0 = time.perf_counter()
        for _ in range(a.calls):
            call()
        us = (time.perf_counter() - t0) / max(1, a.calls) * 1e6
        print(json.dumps({"atoms": N, "atoms_with_ghosts": len(x), "precision": a.precision, "calls": a.calls,
                          "us_per_call": us, "stats": eng.stats()}), flush=True)


if __name__ == "__main__":
    main()
