#!/usr/bin/env python3
"""Benchmark: MD atom-steps/s of the mixed-precision MTP kernel against the FP64
kernel at a stated force error (the headline metric), on the mixed-vs-FP64
workload at scale:

    level-24 MTP (template tables, R=6, K=8), 3 species, cutoff 5.0 A,
    fcc a = 3.6 A, 64^3 cells = 1,048,576 atoms, thermal displacement 0.08 A,
    species uniform 1/3, NVE at 600 K, dt = 1 fs, device neighbour rebuild
    every 10 steps (skin 0.3 A), each MD step captured as a CUDA graph.

One "step" = one velocity-Verlet MD step (integration, r_ij packing, energy +
forces + virial, and the neighbour rebuild at its cadence).  Inputs (1.6 GB of
r_ij per step) are far larger than the 126 MB L2, so no flush is needed.

Our arm (default) prints one JSON line with the mixed value, the FP64 value,
the force/energy error of mixed vs FP64, the roofline of the evaluation
kernel, the CPU baseline (C++/OpenMP FP64 restatement on the host cores) and
the end-to-end number through the C ABI with host buffers.

`--impl reference` times the reference algorithm's CPU implementation (the
oracle port: JAX, which the reference needs, is not installed here) on the
host cores for the same workload and metric.

Multi-GPU: the path does not shard (one MD system per GPU); N ranks run N
independent replicas ("scaling": "weak").
"""

from __future__ import annotations

import argparse
import gc
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "jax-mtp_b200"))
sys.path.insert(0, ROOT)

# level-24 tables, radial coefficients N(0, 0.1^2) from seed 5, moment coefficients
# normalised per basis function to an RMS force of 0.5 eV/A (tests/golden/make_md_potentials.py)
POT = os.path.join(ROOT, "tests", "golden", "potentials", "cfg2md_L24_S3.mtp")
MASS = 55.845          # amu, one stated mass for every species
REPS = 64
STRIDE = 64
SKIN = 0.3
REBUILD = 10
DT = 0.001
TEMP = 600.0
METRIC = "MD atom-steps/s, mixed vs FP64 kernel at stated force error; train cfg/s"


def workload_config():
    return {"workload": "MD NVE, level-24 MTP, 3 species, fcc a=3.6 A 64^3 = 1,048,576 atoms, 600 K, dt 1 fs, "
                        "rebuild every 10 steps, CUDA-graph step",
            "level": 24, "species": 3, "atoms": REPS ** 3 * 4, "nbr_stride": STRIDE, "cutoff": 5.0, "skin": SKIN,
            "precision_headline": "mixed (FP32 radial/moments/tree, FP64 energy/virial/force accumulation)",
            "l2_policy": "inputs (r_ij 1.6 GB/step) larger than L2; no flush",
            "mass_amu": MASS, "parallelism": "replicas",
            "potential": "cfg2md_L24_S3.mtp: radial N(0,0.1^2) seed 5, moment coefficients normalised per basis "
                         "function to RMS force 0.5 eV/A (the N(0,0.01^2) draw gives 10^3 eV/A forces: no MD)"}


def structure():
    from mtp_b200 import synth
    return synth.config2_structure(REPS)


def algorithmic_flops(pot, counts_real: np.ndarray) -> float:
    """Per launch: sum_i n_i (10 B + 6 R K + 6 K + 2 P + 75) + N (9 T + 2 Sa) (FMA = 2)."""
    B = pot.alpha_index_basic_count
    P = len({tuple(r) for r in pot.alpha_index_basic[:, 1:].tolist()})
    R, K, T, Sa = pot.radial_funcs_count, pot.radial_basis_size, pot.alpha_index_times_count, pot.alpha_scalar_moments
    per_nbr = 10 * B + 6 * R * K + 6 * K + 2 * P + 75
    return float(counts_real.sum()) * per_nbr + len(counts_real) * (9 * T + 2 * Sa)


def read_traffic(threads: int, atoms_per_block: int, precision: str = "mixed"):
    """DRAM bytes per evaluation launch of the bench workload for the launch
    shape that ran, from the data file that `python -m mtp_b200.profile_case
    --write-traffic` makes out of an ncu capture (profiles/eval_kernel_traffic.json)."""
    f = os.path.join(ROOT, "profiles", "eval_kernel_traffic.json")
    try:
        with open(f) as fh:
            d = json.load(fh)
    except (OSError, ValueError):
        return None
    e = d.get(f"{precision}_t{threads}_a{atoms_per_block}")
    if not e:
        return None
    return {"bytes_per_launch": float(e["bytes_per_launch_full_workload"]), "source": "eval_kernel_traffic.json",
            "captured_atoms": e.get("captured_atoms"), "scale": e.get("scale")}


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during a timed region."""

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join("/tmp", f"mtp_clocks_{os.getpid()}_{gpu_index}.csv")

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------------------
def cpu_baseline(pot, s, seconds: float = 12.0, sample_atoms: int = 2048):
    """C++/OpenMP FP64 restatement on the host cores, bounded sample of the workload."""
    from mtp_b200 import synth
    from oracle.cpu_ref import CpuMTP
    # a sample of centre atoms with their full neighbour rows
    sub = synth.lattice_structure("fcc", 3.6, (8, 8, 8))       # 2048 atoms, same lattice / density
    rng = np.random.default_rng(51)
    sub.positions = sub.positions + rng.normal(0.0, 0.08, sub.positions.shape)
    sub.types = np.random.default_rng(52).integers(0, 3, sub.natoms).astype(np.int32)
    nd = synth.build_neighbors(sub, pot.max_dist, n_pad=STRIDE)
    cpu = CpuMTP(pot)
    cores = os.cpu_count() or 1
    cpu.compute(nd.itypes, nd.rijs, nd.js, nd.jtypes, nd.counts, nthreads=cores)   # warm-up
    t0 = time.perf_counter()
    reps = 0
    while True:
        cpu.compute(nd.itypes, nd.rijs, nd.js, nd.jtypes, nd.counts, nthreads=cores)
        reps += 1
        if time.perf_counter() - t0 >= seconds:
            break
    dt = time.perf_counter() - t0
    return {"value": nd.natoms * reps / dt, "unit": "atom-steps/s", "cores": cores, "kind": "port",
            "sample": f"{nd.natoms}-atom fcc a=3.6 cell of the same workload (energy+forces+virial, FP64), "
                      f"{reps} evaluations in {dt:.1f} s"}


# ----------------------------------------------------------------------------
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from mtp_b200.mtp_file import read_mtp
    pot = read_mtp(POT)
    steps, warm = args.steps, args.warmup
    from mtp_b200 import synth
    from oracle.cpu_ref import CpuMTP
    sub = synth.lattice_structure("fcc", 3.6, (8, 8, 8))
    rng = np.random.default_rng(51)
    sub.positions = sub.positions + rng.normal(0.0, 0.08, sub.positions.shape)
    sub.types = np.random.default_rng(52).integers(0, 3, sub.natoms).astype(np.int32)
    nd = synth.build_neighbors(sub, pot.max_dist, n_pad=STRIDE)
    cpu = CpuMTP(pot)
    cores = os.cpu_count() or 1
    for _ in range(warm):
        cpu.compute(nd.itypes, nd.rijs, nd.js, nd.jtypes, nd.counts, nthreads=cores)
    t0 = time.perf_counter()
    for _ in range(steps):
        cpu.compute(nd.itypes, nd.rijs, nd.js, nd.jtypes, nd.counts, nthreads=cores)
    dt = time.perf_counter() - t0
    value = nd.natoms * steps / dt
    line = {"metric": METRIC, "value": value, "unit": "atom-steps/s", "n_gpus": args.gpus, "steps": steps,
            "warmup": warm, "ms_per_step": 1e3 * dt / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": workload_config(),
            "cpu_baseline": {"value": value, "unit": "atom-steps/s", "cores": cores, "kind": "port",
                             "sample": f"each step: energy+forces+virial of a {nd.natoms}-atom sample of the "
                                       "workload (same lattice, density, species, potential) on the host cores; "
                                       "the reference's JAX path cannot run (jax not installed)"},
            "e2e": {"value": value, "unit": "atom-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------
def max_over_ranks(ms: float, dist, device) -> float:
    """The job time is the slowest rank's (every rank runs one replica)."""
    if dist is None:
        return ms
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t[0])


def job_value(atoms_per_rank: int, world: int, steps: int, ms: float) -> float:
    """Whole-job atom-steps/s: all replicas' atoms x steps over the slowest rank's time."""
    return world * atoms_per_rank * steps / (ms * 1e-3)


def time_md(md, steps: int, warmup: int, dist, device, sampler=None):
    import torch
    md.run(warmup, graphs=True)
    torch.cuda.synchronize(device)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(device)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    stream = torch.cuda.current_stream(device)
    if sampler is not None:
        sampler.__enter__()
    e0.record(stream)
    md.run(steps, graphs=True)
    e1.record(stream)
    torch.cuda.synchronize(device)
    if sampler is not None:
        sampler.__exit__()
    ms = max_over_ranks(e0.elapsed_time(e1), dist, device)
    if dist is not None:
        dist.barrier()
    return ms


def launches_per_step(rebuild: bool) -> int:
    # verlet x2, pack, eval, gather, totals (partial + final)
    n = 7
    if rebuild:
        # cell assign, scan (3), fill, sort, rows; incoming count, scan (3), fill, sort
        n += 7 + 6
    return n


def run_ours(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as tdist
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        dist = tdist
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)

    from mtp_b200 import synth
    from mtp_b200.engine import MTPEngine, measure_fma_peak
    from mtp_b200.md import DeviceMD
    from mtp_b200.mtp_file import read_mtp

    pot = read_mtp(POT)
    s = structure()
    N = s.natoms
    v0 = synth.maxwell_boltzmann(N, TEMP, MASS, seed=53 + rank)
    masses = [MASS] * pot.species_count

    results = {}
    eng = {p: MTPEngine(POT, N, STRIDE, precision=p) for p in ("mixed", "fp64")}
    mds = {}
    for p in ("mixed", "fp64"):
        mds[p] = DeviceMD(eng[p], s, masses, velocities=v0, dt=DT, skin=SKIN, rebuild_every=REBUILD, stride=STRIDE)
    torch.cuda.synchronize(device)
    # accuracy of mixed vs FP64 at the starting configuration (same neighbour rows)
    fm, f64 = mds["mixed"].f.clone(), mds["fp64"].f.clone()
    em, e64 = float(mds["mixed"].energy[0]), float(mds["fp64"].energy[0])
    dF = (fm - f64).abs()
    force_err = {"max_meV_per_A": float(dF.max()) * 1e3,
                 "rms_meV_per_A": float(torch.sqrt(((fm - f64) ** 2).sum(1).mean())) * 1e3,
                 "energy_meV_per_atom": abs(em - e64) / N * 1e3,
                 "force_scale_eV_per_A": float(f64.abs().max())}
    parity = None
    if rank == 0 and not args.skip_cpu:
        parity = parity_sample(pot, mds["fp64"], mds["mixed"])
    # real neighbours (d < max_dist) per atom, for the algorithmic FLOP count
    rn = mds["fp64"].rijs.norm(dim=2)
    valid = (mds["fp64"].jtypes >= 0) & (rn < pot.max_dist) & (rn > 0)
    counts_real = valid.sum(1).cpu().numpy()
    flops = algorithmic_flops(pot, counts_real)

    # launch shapes by the autotuner (timed on these rows)
    from mtp_b200.autotune import tune
    tuning = {}
    for p in ("mixed", "fp64"):
        md = mds[p]
        r = tune(eng[p], md.types, md.rijs, md.js, md.jtypes, md.counts, use_cache=False)
        tuning[p] = {"threads": r["threads"], "atoms_per_block": r["atoms_per_block"],
                     "eval_ms": r["ms"], "ran": r["ran"]}
        md._forces(reuse=False)       # rebuild the incoming lists after tuning
    torch.cuda.synchronize(device)
    e_start = {p: mds[p].total_energy() for p in ("mixed", "fp64")}
    for p in ("mixed", "fp64"):
        mds[p].capture()
    # timed regions
    sampler = ClockSampler(local)
    for p in ("fp64", "mixed"):
        ms = time_md(mds[p], args.steps, args.warmup, dist, device, sampler if p == "mixed" else None)
        eng[p].sync_status()
        results[p] = {"ms": ms}
    # the evaluation kernel alone: CUDA events around each launch (direct
    # launches on the same rows; graph replays bypass the host-side hooks)
    for p in ("fp64", "mixed"):
        eng[p].set_stream(torch.cuda.current_stream(device).cuda_stream)
        eng[p].profile(True)
        for _ in range(max(3, min(args.steps, 10))):
            mds[p]._forces(reuse=True)
        kms, kn = eng[p].profile_read()
        eng[p].profile(False)
        results[p]["eval_ms_per_launch"] = kms / max(1, kn)
        results[p]["eval_launches"] = kn
    clocks = sampler.summary()
    # NVE drift from step 0 over `--drift-steps` steps (untimed continuation of
    # the graph replays; one replica per process, so only without peers)
    drift = {}
    nd_steps = args.drift_steps if world == 1 else 0
    for p in ("mixed", "fp64"):
        drift[p] = drift_leg(mds[p], e_start[p], max(nd_steps, mds[p].step_count))
    for p in ("mixed", "fp64"):
        mds[p].release()
    fp64_peak, fp32_peak = measure_fma_peak()

    value = job_value(N, world, args.steps, results["mixed"]["ms"])
    value64 = job_value(N, world, args.steps, results["fp64"]["ms"])
    k_mixed = results["mixed"]["eval_ms_per_launch"] * 1e-3
    k_64 = results["fp64"]["eval_ms_per_launch"] * 1e-3
    achieved = flops / k_mixed / 1e12
    achieved64 = flops / k_64 / 1e12
    ran = tuning["mixed"]["ran"]
    traffic_rec = read_traffic(ran["threads"], ran["atoms_per_block"])
    traffic = traffic_rec["bytes_per_launch"] if traffic_rec else None
    ran64 = tuning["fp64"]["ran"]
    traffic64_rec = read_traffic(ran64["threads"], ran64["atoms_per_block"], "fp64")
    # the same launch against HBM: algorithmic bytes per atom-step through the
    # evaluation (28 n_pad + 36: r_ij and neighbour index in, force and energy out)
    alg_bytes = (28 * STRIDE + 36) * N
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            hbm_peak = float(json.load(fh)["hbm_gbs"])
        hbm_src = "MEASURED_PEAKS.json"
    except (OSError, ValueError, KeyError):
        hbm_peak, hbm_src = 6650.0, "fallback"
    hbm_view = {"achieved_gbs": alg_bytes / k_mixed / 1e9, "peak_gbs": hbm_peak,
                "frac": alg_bytes / k_mixed / 1e9 / hbm_peak, "algorithmic_bytes_per_launch": alg_bytes,
                "peak_source": hbm_src}
    nrebuild = sum(1 for k in range(args.warmup + 1, args.warmup + args.steps + 1) if k % REBUILD == 0)
    launches = nrebuild * launches_per_step(True) + (args.steps - nrebuild) * launches_per_step(False)

    # end to end through the C ABI with pinned host buffers (the pair-style boundary)
    e2e = None
    if rank == 0 and not args.skip_e2e:
        e2e = run_e2e(eng["mixed"], mds["mixed"], N, args)

    # the LAMMPS-size legs run with the 1M-atom engines and their pinned
    # buffers released (with them alive the small calls ran up to 1.9x slower)
    for p in ("mixed", "fp64"):
        eng[p].close()
    del mds
    torch.cuda.empty_cache()

    pair_call = None
    if rank == 0 and not args.skip_e2e:
        pair_call = run_pair_call(args)

    cpu = None
    if rank == 0 and not args.skip_cpu:
        cpu = cpu_baseline(pot, s, seconds=args.cpu_seconds)

    pair_nve = None
    if rank == 0 and world == 1 and not args.skip_e2e and args.pair_nve_steps > 0:
        pair_nve = run_pair_style_nve(args.pair_nve_steps)
    train = None
    if not args.skip_train:
        train = run_train(args, device, dist)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "atom-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": results["mixed"]["ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (mixed; FP64 accumulation)", "data": "synthetic",
            "config": workload_config(),
            "fp64": {"value": value64, "unit": "atom-steps/s", "ms_per_step": results["fp64"]["ms"] / args.steps},
            "mixed_over_fp64": value / value64,
            "force_error_mixed_vs_fp64": force_err,
            "nve_drift": drift,
            "parity_sample": parity,
            "autotuned_launch": tuning,
            "train": train,
            "roofline": {"bound": "fp32-fma", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                         "frac": achieved / fp32_peak if fp32_peak else None, "traffic": traffic,
                         "traffic_record": traffic_rec,
                         "kernel": "k_mtp_eval<float> (mixed)", "flops_per_launch": flops,
                         "kernel_ms": k_mixed * 1e3, "hbm_view": hbm_view,
                         "peak_source": "measured live: FP32 FMA-chain kernel (no FP32/FP64 CUDA-core peak in "
                                        "MEASURED_PEAKS.json)",
                         "fp64_kernel": {"achieved": achieved64, "peak": fp64_peak, "frac": achieved64 / fp64_peak
                                         if fp64_peak else None, "kernel_ms": k_64 * 1e3,
                                         "traffic": traffic64_rec["bytes_per_launch"] if traffic64_rec else None}},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "pair_style_call": pair_call,
            "pair_style_nve_config1": pair_nve,
            "gpu_launches": launches * 1,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def parity_sample(pot, md64, mdmx, nsample: int = 512, seed: int = 54):
    """Oracle spot-check of the bench's own rows: `nsample` random atoms of the
    1,048,576-atom system at the starting configuration, their site energies
    and forces from the FP64 and mixed kernels against the C++ FP64 oracle
    (oracle/mtp_cpu.cpp).  The oracle evaluates the sampled atoms and every
    neighbour of theirs (the full lists are symmetric, so every slot that points
    at a sampled atom belongs to that set), which makes the sampled forces
    exact."""
    import torch
    from oracle.cpu_ref import CpuMTP
    N = md64.N
    out = {}
    gpu = {}
    for tag, md in (("fp64", md64), ("mixed", mdmx)):
        eat = torch.empty(N, dtype=torch.float64, device=md.x.device)
        E, F, W = md.eng.compute_device(md.types, md.rijs, md.js, md.jtypes, md.counts, eatom=eat)
        torch.cuda.synchronize()
        gpu[tag] = (eat.cpu().numpy(), F.cpu().numpy())
    rng = np.random.default_rng(seed)
    pick = np.sort(rng.choice(N, nsample, replace=False))
    js = md64.js.cpu().numpy()
    jt = md64.jtypes.cpu().numpy()
    cnt = md64.counts.cpu().numpy()
    rows = js[pick]
    nb = rows[(jt[pick] >= 0) & (np.arange(js.shape[1])[None, :] < cnt[pick][:, None]) & (rows >= 0)]
    closure = np.unique(np.concatenate([pick, nb]))
    remap = np.full(N, -1, dtype=np.int64)
    remap[closure] = np.arange(len(closure))
    sub_js = js[closure]
    sub_js = np.where(sub_js >= 0, remap[np.clip(sub_js, 0, N - 1)], -1).astype(np.int32)
    rij = md64.rijs.cpu().numpy()[closure]
    ref = CpuMTP(pot).compute(md64.types.cpu().numpy()[closure], rij, sub_js, jt[closure], cnt[closure],
                              nthreads=os.cpu_count() or 1)
    at = remap[pick]
    e_ref, f_ref = ref["site_energies"][at], ref["forces"][at]
    for tag in ("fp64", "mixed"):
        e, f = gpu[tag][0][pick], gpu[tag][1][pick]
        out[tag] = {"site_energy_max_rel": float(np.abs(e - e_ref).max() / np.abs(e_ref).max()),
                    "force_max_rel": float(np.abs(f - f_ref).max() / np.abs(f_ref).max()),
                    "site_energy_max_abs_meV": float(np.abs(e - e_ref).max() * 1e3),
                    "force_max_abs_meV_per_A": float(np.abs(f - f_ref).max() * 1e3)}
    out["atoms_sampled"] = int(nsample)
    out["oracle_atoms_evaluated"] = int(len(closure))
    out["reference"] = "C++ FP64 restatement (oracle/mtp_cpu.cpp), same rows"
    out["bars"] = {"fp64_rel": 1e-10, "mixed_site_energy_meV": 0.1, "mixed_force_meV_per_A": 1.0}
    return out


def drift_leg(md, e0: float, nsteps: int, every: int = 10):
    """NVE total-energy record from step 0 (`e0`) to `nsteps` MD steps,
    continuing the graph replays of the timed run (untimed).  The drift is
    the least-squares slope of E_total(t); the end-point difference and the
    largest excursion are reported beside it."""
    ts, es = [0], [e0]
    if md.step_count > 0:
        ts.append(md.step_count)
        es.append(md.total_energy())
    while md.step_count < nsteps:
        md.run(min(every, nsteps - md.step_count), graphs=True)
        ts.append(md.step_count)
        es.append(md.total_energy())
    t = np.asarray(ts, dtype=np.float64) * DT
    e = np.asarray(es, dtype=np.float64)
    slope = float(np.polyfit(t, e, 1)[0]) if len(t) > 1 else 0.0
    N = md.N
    return {"steps": int(md.step_count), "samples": len(ts),
            "meV_per_atom_per_ps": slope / N * 1e3,
            "endpoint_meV_per_atom_per_ps": (e[-1] - e[0]) / N * 1e3 / max(t[-1], 1e-30),
            "max_excursion_meV_per_atom": float(np.abs(e - e[0]).max() / N * 1e3),
            "method": "least-squares slope of total energy over the run"}


def run_pair_style_nve(steps: int = 1000):
    """Config 1 through the pair style: `pair_style jax/mtp` driven by the mini
    LAMMPS host driver (host neighbour list with ghosts, rebuild every 10 steps,
    skin 0.3 A, rows built on the GPU from positions), level-16 MD potential,
    2 species, bcc a = 2.87 A, 10^3 cells = 2,000 atoms, MAX_ATOMS_PER_NEIGHBOR
    60, Maxwell-Boltzmann 300 K (seed 4), dt 1 fs.  atom-steps/s is the
    driver's host wall clock over the whole MD loop (integration, lists,
    pair-style calls)."""
    import tempfile
    from mtp_b200 import synth
    from mtp_b200.lammps_data import write_data
    pdir = os.path.join(ROOT, "jax-mtp_b200", "pair_style")
    r = subprocess.run(["make", "-C", pdir], capture_output=True, text=True)
    if r.returncode != 0:
        return {"unavailable": "mini LAMMPS driver did not build: " + r.stderr[-300:]}
    s = synth.config1()
    v = synth.maxwell_boltzmann(s.natoms, 300.0, MASS, seed=4)
    pot = os.path.join(ROOT, "tests", "golden", "potentials", "cfg1md_L16_S2.mtp")
    out = {"workload": "pair_style jax/mtp NVE, level-16 MD potential, 2 species, bcc a=2.87 A 10^3 = 2,000 atoms, "
                       "300 K, dt 1 fs, rebuild every 10 steps (skin 0.3 A), 60 slots per row",
           "steps": steps, "timer": "host wall clock of the driver's MD loop"}
    with tempfile.TemporaryDirectory() as td:
        data = os.path.join(td, "data.txt")
        write_data(data, s, v, 2)
        for prec in ("fp64", "mixed"):
            r = subprocess.run([os.path.join(pdir, "_build", "mini_lammps"), data, pot, str(s.natoms), "60", "5.0",
                                str(MASS), str(DT), str(steps), "10", "0.3", prec, "100"],
                               capture_output=True, text=True, timeout=900)
            if r.returncode != 0:
                out[prec] = {"error": r.stderr[-300:]}
                continue
            lines = r.stdout.strip().splitlines()
            summ = json.loads(lines[-1])
            th = [l.split() for l in lines if l.startswith("step")]
            t = np.array([float(x[1]) for x in th]) * DT
            et = np.array([float(x[7]) for x in th])
            slope = float(np.polyfit(t, et, 1)[0]) if len(t) > 1 else 0.0
            out[prec] = {"atom_steps_per_s": summ["atom_steps_per_s"], "pair_ms_per_step": summ["pair_ms_per_step"],
                         "drift_meV_per_atom_per_ps": slope / s.natoms * 1e3,
                         "endpoint_drift_meV_per_atom": summ["energy_drift_eV_per_atom"] * 1e3,
                         "temperature_end_K": float(th[-1][9]), "pair_calls": summ["pair_calls"]}
    return out


def batch_diagnostics(nds, min_dist: float):
    """How much of a training batch lies below the potential's min_dist, where
    the Chebyshev basis is evaluated outside [-1, 1] (the stated lattice range
    a in [2.8, 4.2] A puts fcc nearest neighbours at 1.98-2.97 A)."""
    n_pairs = n_bad = n_cfg_bad = 0
    dmin = float("inf")
    for nd in nds:
        d = np.linalg.norm(nd.rijs, axis=2)[nd.jtypes >= 0]
        b = int((d < min_dist).sum())
        n_pairs += d.size
        n_bad += b
        n_cfg_bad += b > 0
        if d.size:
            dmin = min(dmin, float(d.min()))
    return {"pairs_below_min_dist_frac": n_bad / max(1, n_pairs), "configs_with_pairs_below_min_dist": n_cfg_bad,
            "configs": len(nds), "min_pair_distance_A": dmin, "min_dist_A": min_dist}


def rmse_per_atom(E, F, E_t, F_t, natom_c):
    """Energy RMSE per atom (meV/atom) over configurations and force RMSE (meV/A) over components."""
    import torch
    de = ((E - E_t) / natom_c)
    return {"energy_rmse_meV_per_atom": float(torch.sqrt((de * de).mean())) * 1e3,
            "force_rmse_meV_per_A": float(torch.sqrt(((F - F_t) ** 2).mean())) * 1e3}


def run_train(args, device, dist):
    """Training throughput: configuration 3 (level 20, 2 species, 512 periodic
    configurations, N in [16, 256], batched forward in mixed precision) and
    configuration 4 (level 28, 4 species, 256 configurations, N in [32, 512],
    FP64 forward + hand-written adjoint of the E/F/stress loss)."""
    import torch
    from mtp_b200 import synth
    from mtp_b200.engine import MTPEngine
    from mtp_b200.mtp_file import read_mtp
    from mtp_b200.train import DeviceBatch, predict, weighted_loss
    potdir = os.path.join(ROOT, "tests", "golden", "potentials")
    out = {}

    def timed(fn, steps, warm):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize(device)
        if dist is not None:
            dist.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize(device)
        return max_over_ranks(e0.elapsed_time(e1), dist, device)

    world = 1 if dist is None else dist.get_world_size()
    # ---- configuration 3: batched forward, mixed precision
    pot3 = read_mtp(os.path.join(potdir, "cfg3_L20_S2.mtp"))
    structs = synth.training_batch(512, 16, 256, 2, seed=6)
    nds = [synth.build_neighbors(st, pot3.max_dist) for st in structs]
    nd, cfg, offs, vols = synth.pack_batch(nds)
    batch = DeviceBatch.from_numpy(nd, cfg, vols, device=device)
    with MTPEngine(os.path.join(potdir, "cfg3label_L20_S2.mtp"), nd.natoms, nd.n_pad) as lab:
        E_l, F_l, S_l = lab.batch_device(batch.itypes, batch.rijs, batch.js, batch.jtypes, batch.counts, batch.cfg,
                                         batch.volumes, batch.nconfig)
    diag3 = batch_diagnostics(nds, pot3.min_dist)
    g = torch.Generator(device="cpu").manual_seed(7)
    natom_c = torch.as_tensor(np.diff(offs), dtype=torch.float64, device=device)
    diag3["label_energy_rms_eV_per_atom"] = float(torch.sqrt(((E_l / natom_c) ** 2).mean()))
    diag3["label_force_rms_eV_per_A"] = float(torch.sqrt((F_l ** 2).mean()))
    E_t = E_l + 1e-3 * natom_c * torch.randn(batch.nconfig, generator=g, dtype=torch.float64).to(device)
    F_t = F_l + 1e-2 * torch.randn(F_l.shape, generator=g, dtype=torch.float64).to(device)
    S_t = S_l + 6.2415e-4 * torch.randn(S_l.shape, generator=g, dtype=torch.float64).to(device)
    from mtp_b200.autotune import tile_candidates, tune_batch, tune_step
    tiles3 = tile_candidates(int(nd.counts.max()))
    with MTPEngine(os.path.join(potdir, "cfg3_L20_S2.mtp"), nd.natoms, max(tiles3), precision="mixed") as eng3:
        # neighbour tile, threads and atoms per block by the autotuner, on this batch
        tuned3 = tune_batch(eng3, batch, tiles=tiles3)
        b3 = tuned3["batch"]

        def fwd3():
            eng3.batch_device(b3.itypes, b3.rijs, b3.js, b3.jtypes, b3.counts, b3.cfg, b3.volumes, b3.nconfig)
        steps = max(3, min(args.steps, 10))
        ms = timed(fwd3, steps, 3)
        E_p, F_p, S_p = eng3.batch_device(b3.itypes, b3.rijs, b3.js, b3.jtypes, b3.counts, b3.cfg, b3.volumes,
                                          b3.nconfig)
        loss = float(weighted_loss(E_p, F_p, S_p, (E_t, F_t, S_t)))
        rmse3 = rmse_per_atom(E_p, F_p, E_t, F_t, natom_c)
        eng3.sync_status()
    # least-squares basis fit of configuration 3 (FP64): Jacobian by 289
    # batched forwards, then a thin SVD (the reference's jacfwd + lstsq)
    from mtp_b200.train import solve_lls_basis
    with MTPEngine(os.path.join(potdir, "cfg3_L20_S2.mtp"), nd.natoms, nd.n_pad, precision="fp64") as e64:
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        theta, info = solve_lls_basis(e64, batch, (E_t, F_t, S_t), pot3.species_coeffs, pot3.radial_coeffs)
        torch.cuda.synchronize(device)
        lls_s = time.perf_counter() - t0
        with torch.no_grad():
            E_f, F_f, _ = predict({"species": torch.as_tensor(pot3.species_coeffs, device=device),
                                   "basis": theta, "radial": torch.as_tensor(pot3.radial_coeffs, device=device)},
                                  e64, batch)
        rmse_fit = rmse_per_atom(E_f, F_f, E_t, F_t, natom_c)
        e64.sync_status()
    out["cfg3_lls_basis"] = {"seconds": lls_s, "forwards": pot3.alpha_scalar_moments + 1, "rank": info["rank"],
                             "loss_after": info["loss"], "loss_before": loss, "precision": "fp64",
                             "rmse_before": rmse3, "rmse_after": rmse_fit,
                             "rows": int(batch.nconfig * 7 + 3 * batch.natoms)}
    out["cfg3_batched_forward"] = {"value": world * batch.nconfig * steps / (ms * 1e-3), "unit": "cfg/s",
                                   "configs": batch.nconfig, "atoms": batch.natoms, "nbr_stride": b3.stride,
                                   "ms_per_batch": ms / steps, "precision": "mixed", "loss_vs_labels": loss,
                                   "autotuned": {"n_pad": tuned3["n_pad"], "threads": tuned3["threads"],
                                                 "atoms_per_block": tuned3["atoms_per_block"],
                                                 "candidates_ms": {k: (v["ms"] if isinstance(v, dict) else v)
                                                                   for k, v in tuned3["timings"].items()}},
                                   "rmse_vs_labels": rmse3, "data_diagnostics": diag3,
                                   "labels": "second random level-20 MTP (seed 7) + noise 1 meV/atom, "
                                             "10 meV/A, 0.1 GPa",
                                   "note": "the raw loss is dominated by the configurations with pairs below "
                                           "min_dist, where both random potentials extrapolate the Chebyshev "
                                           "basis; the throughput is unaffected"}
    del batch
    # ---- configuration 4: forward + adjoint training step, FP64
    pot4 = read_mtp(os.path.join(potdir, "cfg4_L28_S4.mtp"))
    structs = synth.training_batch(256, 32, 512, 4, seed=8)
    nds = [synth.build_neighbors(st, pot4.max_dist) for st in structs]
    diag4 = batch_diagnostics(nds, pot4.min_dist)
    nd, cfg, offs, vols = synth.pack_batch(nds)
    batch = DeviceBatch.from_numpy(nd, cfg, vols, device=device)
    tiles4 = tile_candidates(int(nd.counts.max()))
    with MTPEngine(os.path.join(potdir, "cfg4_L28_S4.mtp"), nd.natoms, max(tiles4), precision="fp64") as eng4:
        params = {k: torch.tensor(v, dtype=torch.float64, device=device, requires_grad=True)
                  for k, v in (("species", pot4.species_coeffs), ("basis", pot4.moment_coeffs),
                               ("radial", pot4.radial_coeffs))}
        with torch.no_grad():
            E0, F0, S0 = predict(params, eng4, batch)
        g = torch.Generator(device="cpu").manual_seed(9)
        tgt = (E0 + 1e-3 * torch.randn(E0.shape, generator=g, dtype=torch.float64).to(device),
               F0 + 1e-2 * torch.randn(F0.shape, generator=g, dtype=torch.float64).to(device),
               S0 + 6.2415e-4 * torch.randn(S0.shape, generator=g, dtype=torch.float64).to(device))

        def step_on(b):
            for v in params.values():
                v.grad = None
            L = weighted_loss(*predict(params, eng4, b), tgt)
            L.backward()

        # neighbour tile, threads and atoms per block of the whole step (the
        # forward and the adjoint share the engine's launch settings)
        tuned4 = tune_step(eng4, batch, step_on, candidates=((256, 1), (512, 1), (256, 2), (512, 2)), tiles=tiles4,
                           calls=1, tag="train_step")
        b4 = tuned4["batch"]
        steps = max(2, min(args.steps, 4))
        ms = timed(lambda: step_on(b4), steps, 1)
        eng4.sync_status()
    out["cfg4_train_step"] = {"value": world * batch.nconfig * steps / (ms * 1e-3), "unit": "cfg/s",
                              "configs": batch.nconfig, "atoms": batch.natoms, "nbr_stride": b4.stride,
                              "ms_per_step": ms / steps, "precision": "fp64",
                              "step": "batched forward (E, F, stress) + loss + hand-written adjoint w.r.t. all "
                                      "coefficients", "jax_grad_baseline": "unavailable on this box (no JAX)",
                              "data_diagnostics": diag4,
                              "autotuned": {"n_pad": tuned4["n_pad"], "threads": tuned4["threads"],
                                            "atoms_per_block": tuned4["atoms_per_block"],
                                            "candidates_ms": {k: (v["ms"] if isinstance(v, dict) else v)
                                                              for k, v in tuned4["timings"].items()}}}
    return out


def run_e2e(eng, md, N, args):
    """mtp_compute with pinned host buffers: H2D inputs + kernels + D2H results per step."""
    import torch
    stride = STRIDE
    pin = lambda shape, dt: torch.empty(shape, dtype=dt, pin_memory=True).numpy()
    it = pin((N,), torch.int32)
    rij = pin((N, stride, 3), torch.float64)
    js = pin((N, stride), torch.int32)
    jt = pin((N, stride), torch.int32)
    cnt = pin((N,), torch.int32)
    F = pin((N, 3), torch.float64)
    it[:] = md.types.cpu().numpy()
    md._rebuild()
    md.eng.pack_rij_device(md.x, md.cell, md.js, md.image, md.counts, md.rijs)
    torch.cuda.synchronize()
    rij[:] = md.rijs.cpu().numpy()
    js[:] = md.js.cpu().numpy()
    jt[:] = md.jtypes.cpu().numpy()
    cnt[:] = md.counts.cpu().numpy()
    from mtp_b200._lib import EFLAG, VFLAG, check, lib
    import ctypes
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    e = np.zeros(1)
    vir = np.zeros(6)
    eng.use_own_stream()

    def call():
        code = lib().mtp_compute(eng.handle, N, stride, P(it), P(rij), P(js), P(jt), P(cnt), EFLAG | VFLAG, P(e), P(F),
                                 P(vir), None, None)
        check(code, eng.handle)

    for _ in range(max(1, min(args.warmup, 2))):
        call()
    steps = max(5, min(args.steps, 20))
    t0 = time.perf_counter()
    for _ in range(steps):
        call()
    dt = time.perf_counter() - t0
    h2d = N * 4 + N * stride * (24 + 4 + 4) + N * 4
    d2h = N * 24 + 8 + 48
    return {"value": N * steps / dt, "unit": "atom-steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "steps": steps, "api": "mtp_compute (C ABI, pinned host buffers, synchronous)",
            "note": "force call per MD step as the pair style makes it; integration not included"}


def run_pair_call(args):
    """Latency of one force call of the LAMMPS MD case: level-16 MTP, 2 species
    (cfg1_L16_S2.mtp), bcc a = 2.87 A, 10^3 cells = 2,000 atoms, 50/50 species,
    MAX_ATOMS_PER_NEIGHBOR 60, cutoff 5.0 A.  Host buffers in and out, as the pair
    style calls it: through mtp_compute with page-locked rows (mtp_host_alloc,
    what pair_mtp_b200.cpp packs into) and with pageable numpy arrays, and
    through mtp_execute_potential (the reference bridge's per-atom row pointers,
    built once outside the timed calls), and through mtp_compute_positions
    (page-locked positions of the atoms and their periodic ghosts plus the full
    neighbour list with a 0.3 A skin, rows built on the GPU).  Host wall clock
    per synchronous call."""
    import ctypes
    from mtp_b200 import synth
    from mtp_b200._lib import EFLAG, VFLAG, check, lib
    from mtp_b200.engine import MTPEngine, pinned_empty
    path = os.path.join(ROOT, "tests", "golden", "potentials", "cfg1_L16_S2.mtp")
    s = synth.config1()
    nd = synth.build_neighbors(s, 5.0, n_pad=60)
    N, n = nd.js.shape
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    it = np.ascontiguousarray(nd.itypes, np.int32)
    rij = np.ascontiguousarray(nd.rijs, np.float64)
    js = np.ascontiguousarray(nd.js, np.int32)
    jt = np.ascontiguousarray(nd.jtypes, np.int32)
    cnt = np.ascontiguousarray(nd.counts, np.int32)
    F = np.zeros((N, 3))
    e = np.zeros(1)
    vir = np.zeros(6)
    st = np.zeros(6)
    # positions + ghosts + neighbour list for the device-rows entry point
    gx, gown, glists = synth.ghosts_and_lists(s, 5.3)
    lstride = max(len(c) for c in glists)
    pos_in = {"x": pinned_empty(gx.shape, np.float64), "sp": pinned_empty((len(gx),), np.int32),
              "own": pinned_empty((len(gx),), np.int32), "nb": pinned_empty((N, lstride), np.int32),
              "num": pinned_empty((N,), np.int32)}
    pos_in["x"][...] = gx
    pos_in["sp"][...] = s.types[gown]
    pos_in["own"][...] = gown
    pos_in["nb"][...] = -1
    for i, c in enumerate(glists):
        pos_in["nb"][i, :len(c)] = c
        pos_in["num"][i] = len(c)
    pinned = {}
    for k, a in (("it", it), ("rij", rij), ("js", js), ("jt", jt), ("cnt", cnt), ("F", F), ("e", e), ("vir", vir)):
        pinned[k] = pinned_empty(a.shape, a.dtype)
        pinned[k][...] = a
    Pv = ctypes.c_void_p * N
    pr = Pv(*[rij[i].ctypes.data for i in range(N)])
    pj = Pv(*[js[i].ctypes.data for i in range(N)])
    pt = Pv(*[jt[i].ctypes.data for i in range(N)])
    pf = Pv(*[F[i].ctypes.data for i in range(N)])
    calls = max(20, min(200, 10 * args.steps))
    out = {"workload": "level-16 MTP, 2 species, bcc a=2.87 A 10^3 = 2,000 atoms, 60 slots per row, cutoff 5.0 A",
           "calls": calls, "timer": "host wall clock per synchronous call (H2D + kernels + D2H)"}
    for prec in ("fp64", "mixed"):
        with MTPEngine(path, N, n, cutoff=5.0, precision=prec) as eng:
            h = eng.handle

            def flat():
                check(lib().mtp_compute(h, N, n, P(it), P(rij), P(js), P(jt), P(cnt), EFLAG | VFLAG, P(e), P(F),
                                        P(vir), None, None), h)

            def flat_pinned():
                b = pinned
                check(lib().mtp_compute(h, N, n, P(b["it"]), P(b["rij"]), P(b["js"]), P(b["jt"]), P(b["cnt"]),
                                        EFLAG | VFLAG, P(b["e"]), P(b["F"]), P(b["vir"]), None, None), h)

            def positions():
                b, q = pinned, pos_in
                check(lib().mtp_compute_positions(h, N, len(gx), P(q["x"]), P(q["sp"]), P(q["own"]), lstride,
                                                  P(q["nb"]), P(q["num"]), EFLAG | VFLAG, P(b["e"]), P(b["F"]),
                                                  P(b["vir"]), None, None), h)

            def bridge():
                check(lib().mtp_execute_potential(h, N, int(cnt.sum()), ctypes.cast(pr, ctypes.c_void_p), P(it),
                                                  ctypes.cast(pj, ctypes.c_void_p), P(cnt),
                                                  ctypes.cast(pt, ctypes.c_void_p), float(nd.volume), P(e),
                                                  ctypes.cast(pf, ctypes.c_void_p), P(st)), h)

            for name, fn in (("mtp_compute_pinned", flat_pinned), ("mtp_compute_pageable", flat),
                             ("mtp_execute_potential", bridge), ("mtp_compute_positions", positions)):
                for _ in range(5):
                    fn()
                # buffers of earlier legs are freed now, not by a collection
                # (cudaFreeHost of gigabytes) inside the timed calls
                gc.collect()
                gc.disable()
                st0 = eng.stats()
                t0 = time.perf_counter()
                for _ in range(calls):
                    fn()
                us = (time.perf_counter() - t0) / calls * 1e6
                gc.enable()
                st1 = eng.stats()
                out[f"{prec}_{name}_us"] = us
                out[f"{prec}_{name}_atom_steps_per_s"] = N / (us * 1e-6)
                out[f"{prec}_{name}_graph_replays"] = int(st1["graph_replays"] - st0["graph_replays"])
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--skip-train", action="store_true")
    ap.add_argument("--drift-steps", type=int, default=500,
                    help="NVE drift record length in MD steps (untimed; 1 GPU only; 0: the timed steps only)")
    ap.add_argument("--pair-nve-steps", type=int, default=1000,
                    help="config 1 through the pair style: MD steps of the mini LAMMPS driver (0: skip)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
