#!/usr/bin/env python
"""PM7 SCF solves/s on one B200 (and N replicas on N GPUs).

Workload (default): plain FP64 RHF single point of a 1,002-atom water cluster (334 H2O on a
3.1 A cubic grid, seeded random orientations, +-0.1 A centre jitter, 2,004 basis functions),
synthetic inputs from pm7b200.geometry with seed 0. A step is one complete solve: core
Hamiltonian, SCF to the reference's default tolerances (e_tol 1e-8 eV, p_tol 1e-7), core-core
and post-SCF corrections, charges and dipole.

  value  solves/s from the engine's CUDA events over each solve (device time, inputs resident
         when the first kernel starts)
  e2e    solves/s from the wall clock around the public C-ABI call `pm7_run` with host input
         buffers and host result buffers (host<->device copies inside)

One JSON line on rank 0. `--impl reference` times the CPU restatement of the reference's
`run_pm7` (oracle/, C++ with OpenMP + OpenBLAS) on all host cores instead.

Other workloads (`--workload`):
  batch4096  the mixed batch of 4,096 molecules (half alkanes C_nH_2n+2, n ~ U{1..40}, half
             water clusters of 2..64 H2O, 0.02 A jitter, seed 0) through `pm7_run_batch`; a
             step is one complete batch; value = molecules solved per second of wall time
             around the call (host inputs, uploads and results inside); beside it the plain
             single-molecule path on a fixed sample of the same molecules.
  stream     the served stream: molecules of log-uniform size in 3..500 atoms (substituted
             C/S chains with Cl, and water clusters, seed 0) submitted to `pm7_engine` with
             Poisson arrivals at 80% of the engine's measured burst capacity; reports
             solves/s and p50/p99 submit-to-finish latency, and the plain path on a sample.
  dandc640   the divide-and-conquer SCF (`pm7_run_dandc`) of the flat chain C640H1282,
             1,922 atoms, buffer 15 Bohr, cores of 8 atoms; a step is one solve from host
             buffers to host results.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "pm7-rs_b200"))

import numpy as np  # noqa: E402

A0 = 0.529177210903


def workload(name):
    from pm7b200 import geometry as G

    if name == "water334":
        z, x = G.water_cluster(334, seed=0)
        desc = "1002-atom water cluster (334 H2O), 2004 basis functions, RHF FP64"
    elif name == "water1000":
        z, x = G.water_cluster(1000, seed=0)
        desc = "3000-atom water cluster (1000 H2O), 6000 basis functions, RHF FP64"
    elif name == "decane":
        z, x = G.decane(0)
        desc = "n-decane C10H22 (32 atoms, 62 basis functions), RHF FP64"
    else:
        raise SystemExit(f"unknown workload {name}")
    return z, x, desc


def nao_of(z):
    return int(sum(1 if int(v) == 1 else 4 for v in z))


def near_w_doubles(z, x):
    """Sum of npair(u)*npair(v) over atom pairs closer than 7 Angstrom (the stored blocks)."""
    return near_pairs(z, x)[1]


def near_pairs(z, x):
    """(atom pairs closer than 7 Angstrom, their stored two-electron doubles)."""
    npair = np.array([1 if int(v) == 1 else 10 for v in z], dtype=np.int64)
    count, tot = 0, 0
    for i in range(len(z)):
        d = np.linalg.norm(x[i + 1:] - x[i], axis=1) * A0
        near = d < 7.0
        count += int(np.sum(near))
        tot += int(np.sum(npair[i] * npair[i + 1:][near]))
    return count, tot


class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, max, throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device, interval_ms=200):
        self.device = device
        self.interval_ms = interval_ms
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", str(self.interval_ms)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            for name, val in zip(names, r[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text())
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "fallback": True}


def fp64_dgemm_peak(device):
    """FP64 tensor-core peak measured here: best cuBLAS DGEMM (torch.matmul, float64)."""
    import torch

    torch.cuda.set_device(device)
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        a @ b
        e.record()
        torch.cuda.synchronize()
        best = max(best, 2.0 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def read_traffic(kernel):
    """Per-launch DRAM bytes of `kernel` from a committed ncu summary, scaled to the bench size."""
    p = ROOT / "profiles" / "traffic.txt"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        parts = line.split()
        if len(parts) >= 2 and parts[0] == kernel:
            try:
                return float(parts[1])
            except ValueError:
                return None
    return None


def cpu_sample_full(z, x):
    """One full oracle solve on all host cores: (seconds, iterations)."""
    from oracle import harness

    harness.set_threads(os.cpu_count() or 1)
    t = time.perf_counter()
    r = harness.run(z, x, want_matrices=0)
    return time.perf_counter() - t, r["iterations"]


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def allreduce_max(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist

    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def bench_config(args, desc, z, world):
    """The `config` both arms print for the single-molecule workloads (identical dicts)."""
    nao = nao_of(z)
    return {"workload": args.workload, "description": desc, "seed": 0, "n_atoms": len(z), "nao": nao,
            "parallelism": f"replicas{world}",
            "l2": f"inputs larger than L2 (H, F, P and DIIS history are {8 * nao * nao / 1e6:.0f} MB each at nao={nao})"}


def run_reference(args, world, rank):
    """CPU restatement of the reference (oracle/) on the host cores; rank 0 only.

    Every step, warm-up included, is one complete `run_pm7` solve of the workload (core
    Hamiltonian, SCF to the default tolerances, core-core, corrections, charges, dipole) on
    all host cores: OpenMP over pairs, atoms and rows as the reference's rayon pool, and the
    OpenBLAS bundled with numpy for the eigensolver."""
    if rank != 0:
        return
    from oracle import harness

    z, x, desc = workload(args.workload)
    cores = os.cpu_count() or 1
    harness.set_threads(cores)
    for _ in range(args.warmup):
        harness.run(z, x, want_matrices=0)
    times, r = [], None
    for _ in range(args.steps):
        t = time.perf_counter()
        r = harness.run(z, x, want_matrices=0)
        times.append(time.perf_counter() - t)
    solve_s = sum(times) / len(times)
    value = 1.0 / solve_s
    sample = (f"{args.steps} complete solves of the {desc} ({r['iterations']} SCF iterations each), "
              f"{min(times):.2f}-{max(times):.2f} s per solve")
    line = {
        "impl": "reference", "metric": "PM7 SCF solves/s (RHF single point)", "value": value, "unit": "solves/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": solve_s * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": bench_config(args, desc, z, world),
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "result": {"heat_of_formation_kcal": r["heat_of_formation_kcal"], "total_ev": r["total_ev"],
                   "scf_iterations": r["iterations"]},
    }
    print(json.dumps(line), flush=True)


def run_b200(args, world, rank, local):
    from pm7b200 import api

    if api.device_count() < 1:
        raise SystemExit("no CUDA device visible: the engine has no CPU fallback")
    z, x, desc = workload(args.workload)
    n_atoms, nao = len(z), nao_of(z)
    opts = dict(device=local, want_matrices=0)
    if args.precision == "mixed":
        # the mixed-precision solve is the timed one (fp32 tcgen05 cycles, fp64 refinement)
        opts["precision"] = 1
        desc = desc.replace("RHF FP64", "RHF mixed precision")
        args.no_mixed = True
    for _ in range(args.warmup):
        api.run_pm7(z, x, **opts)
    peaks = measured_peaks()
    dgemm = fp64_dgemm_peak(local) if rank == 0 and not args.no_fp64_peak else None
    barrier(world)
    sampler = ClockSampler(local)
    sampler.start()
    launches0 = api.launch_count()
    dev_ms = 0.0
    results = []
    lat = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ts = time.perf_counter()
        r = api.run_pm7(z, x, **opts)
        lat.append((time.perf_counter() - ts) * 1e3)
        dev_ms += r["device_ms"]
        results.append(r)
    wall = time.perf_counter() - t0
    launches = api.launch_count() - launches0

    def stage_pass(**extra):
        # per-stage CUDA-event breakdown on a separate, untimed pass: its event bookkeeping
        # stays out of the timed loops
        api.profile_enable(True)
        for _ in range(args.steps):
            api.run_pm7(z, x, **opts, **extra)
        p = api.profile_read()
        api.profile_enable(False)
        return p

    prof = stage_pass()
    # the same solve in mixed precision: fp32 purification cycles on tcgen05, fp64 refinement
    mixed = None
    if not args.no_mixed:
        api.run_pm7(z, x, precision=1, **opts)
        mdev, mres = 0.0, []
        tm0 = time.perf_counter()
        for _ in range(args.steps):
            q = api.run_pm7(z, x, precision=1, **opts)
            mdev += q["device_ms"]
            mres.append(q)
        mwall = time.perf_counter() - tm0
        mprof = stage_pass(precision=1)
        mixed = {"value": args.steps / (mdev * 1e-3), "e2e": args.steps / mwall, "unit": "solves/s",
                 "iterations": mres[-1]["iterations"], "fp32_iterations": mres[-1]["fp32_iterations"],
                 "dhf_err_vs_fp64_kcal": abs(mres[-1]["heat_of_formation_kcal"] - results[-1]["heat_of_formation_kcal"]),
                 "max_charge_err_vs_fp64": float(np.max(np.abs(mres[-1]["charges"] - results[-1]["charges"]))),
                 "stages": {k: {"ms_total": round(v[0], 3), "calls": v[1]} for k, v in mprof.items()}}
        tf_ms, tf_calls = mprof.get("sp2_square_tf32", (0.0, 0))
        if tf_calls:
            ld = ((nao + 31) // 32) * 32
            t = (nao + 127) // 128
            flops = 3 * (t * (t + 1) // 2) * 128 * 128 * 2.0 * ld  # issued: 3 MMA products per lower tile
            alg = 3.0 * float(nao) ** 3                             # algorithmic: 3 symmetric products
            ach = alg / (tf_ms / tf_calls * 1e-3) / 1e12
            peak_tf32 = peaks.get("bf16_tflops", 1590.0) / 2.0
            mixed["roofline"] = {"kernel": "k_square_tf32x3 (tcgen05.mma kind::tf32, TMA, TMEM)", "bound": "tensor",
                                 "achieved": ach, "peak": peak_tf32, "unit": "TFLOP/s", "frac": ach / peak_tf32,
                                 "issued_tflops": flops / (tf_ms / tf_calls * 1e-3) / 1e12,
                                 "ms_avg": tf_ms / tf_calls, "launches": tf_calls,
                                 "peak_source": "half the measured bf16 dense rate in MEASURED_PEAKS.json (TF32 runs at half the bf16 rate)"}
    # the nuclear gradient of the same solve through pm7_gradient (closed_form_gradient: the SCF
    # and the gradient of its total energy), wall clock with host buffers; the device split of
    # the gradient stages from one more, untimed call with stage events
    grad = None
    if not args.no_gradient:
        api.closed_form_gradient(z, x, **opts)
        gw, go = [], None
        for _ in range(args.steps):
            t = time.perf_counter()
            go = api.closed_form_gradient(z, x, **opts)
            gw.append(time.perf_counter() - t)
        api.profile_enable(True)
        api.closed_form_gradient(z, x, **opts)
        gp = api.profile_read()
        api.profile_enable(False)
        gpair, gcorr = gp.get("gradient_pairs", (0.0, 0))[0], gp.get("gradient_corrections", (0.0, 0))[0]
        grad = {"value": args.steps / sum(gw), "unit": "SCF+gradient/s (pm7_gradient, host buffers)",
                "gradient_device_ms": gpair + gcorr, "pairs_ms": gpair, "corrections_ms": gcorr,
                "pair_stencil_energies": len(z) * (len(z) - 1) // 2 * 12,
                "max_gradient_ev_bohr": go["max_gradient"],
                "net_force_ev_bohr": float(np.max(np.abs(go["gradient"].sum(axis=0))))}
    clocks = sampler.stop()
    barrier(world)
    dev_s = allreduce_max(dev_ms * 1e-3, world)
    wall = allreduce_max(wall, world)
    if rank != 0:
        return
    total = args.steps * world
    value = total / dev_s
    e2e = total / wall
    r0 = results[-1]
    # dominant kernels of ours and their roofline: the FP64 DMMA GEMMs (k_gemm_sym, k_gemm_tn), timed per
    # launch with CUDA events on the engine's stream
    stages = {k: {"ms_total": round(v[0], 3), "calls": v[1], "ms_avg": round(v[0] / max(v[1], 1), 4)}
              for k, v in prof.items()}
    roofline = None
    i8_ms, i8_calls = prof.get("sp2_square_i8", (0.0, 0))
    sq_ms, sq_calls = prof.get("sp2_square_gemm", (0.0, 0))
    cm_ms, cm_calls = prof.get("commutator_gemm", (0.0, 0))
    gemm_ms = sq_ms + cm_ms
    if sq_calls or cm_calls:
        flops = sq_calls * float(nao) ** 3 + cm_calls * 2.0 * float(nao) ** 3  # algorithmic
        launches_g = sq_calls + cm_calls
        achieved = flops / (gemm_ms * 1e-3) / 1e12
        sq_traffic, cm_traffic = read_traffic("sp2_square_gemm"), read_traffic("commutator_gemm")
        traffic = None
        if sq_traffic is not None and cm_traffic is not None:
            traffic = (sq_calls * sq_traffic + cm_calls * cm_traffic) / launches_g
        label = ("k_gemm_sym (SP2 squares) + k_gemm_tn (F.P)" if sq_calls else "k_gemm_tn (F.P)") + \
            ", FP64 DMMA mma.sync.m16n8k8"
        roofline = {"kernel": label, "bound": "tensor", "achieved": achieved,
                    "peak": dgemm, "unit": "TFLOP/s", "frac": (achieved / dgemm) if dgemm else None,
                    "traffic": traffic, "launches": launches_g, "ms_avg": gemm_ms / launches_g,
                    "algorithmic_per_launch": f"{flops / launches_g:.4g} flop (SP2 square nao^3, commutator 2 nao^3)",
                    "peak_source": "FP64 cuBLAS DGEMM 8192^3 measured in this run (MEASURED_PEAKS.json has no FP64 entry)"}
    if i8_calls:
        # the FP64-accuracy squarings on the integer tensor cores: issued int8 work per launch
        # (36 digit-pair products over the 128 x 64 lower tiles, K padded to 32) against twice
        # the measured bf16 dense rate (kind::i8 runs at exactly twice kind::f16 per SM), and
        # the fp64-equivalent rate (nao^3 per symmetric squaring) against the measured DGEMM
        tm, tn = (nao + 127) // 128, (nao + 63) // 64
        tiles = sum(min(2 * r + 2, tn) for r in range(tm))
        kpad = ((nao + 31) // 32) * 32
        ops = 36.0 * 2.0 * 128 * 64 * kpad * tiles
        ms_avg = i8_ms / i8_calls
        achieved_tops = ops / (ms_avg * 1e-3) / 1e12
        peak_i8 = 2.0 * peaks.get("bf16_tflops", 1590.0)
        fp64_eq = float(nao) ** 3 / (ms_avg * 1e-3) / 1e12
        prev = roofline
        roofline = {"kernel": "k_sp2_step_i8 (SP2 squares, tcgen05.mma kind::i8 on int8 digit planes, TMA, TMEM; "
                              "fp64 accuracy by the Ozaki scheme)", "bound": "tensor", "achieved": achieved_tops,
                    "peak": peak_i8, "unit": "TOP/s", "frac": achieved_tops / peak_i8,
                    "traffic": read_traffic("sp2_square_i8"), "launches": i8_calls, "ms_avg": ms_avg,
                    "algorithmic_per_launch": f"{ops:.4g} int8 ops issued ({float(nao) ** 3:.4g} fp64-equivalent flop)",
                    "fp64_equivalent_tflops": fp64_eq, "fp64_equivalent_frac_of_dgemm": (fp64_eq / dgemm) if dgemm else None,
                    "peak_source": "twice the measured bf16 dense rate in MEASURED_PEAKS.json"}
        if prev is not None:
            roofline["commutator_dmma"] = prev
    # pair integrals: the build stage computes every pair's overlap/resonance and core-core
    # terms and the multipole two-electron blocks of the pairs inside 7 Angstrom
    pair_rate = None
    b_ms, b_calls = prof.get("build", (0.0, 0))
    if b_calls:
        n_near, w_near = near_pairs(z, x)
        n_all = len(z) * (len(z) - 1) // 2
        per = b_ms / b_calls * 1e-3
        pair_rate = {"pairs_all": n_all, "pairs_near": n_near, "w_doubles_near": w_near, "build_ms": per * 1e3,
                     "pairs_per_s": n_all / per, "near_pairs_per_s": n_near / per,
                     "note": "build stage (k_pairs_all + k_near_integrals + k_hcore_diag) per solve"}
    fock_ms, fock_calls = prof.get("fock", (0.0, 0))
    fock_roof = None
    if fock_calls:
        w_near = near_w_doubles(z, x)
        nbytes = 8.0 * (w_near + 3.0 * nao * nao)
        achieved_gbs = nbytes / (fock_ms / fock_calls * 1e-3) / 1e9
        fock_roof = {"kernel": "fock (k_fock_far + k_fock_near + k_fock_atom)", "bound": "hbm",
                     "achieved": achieved_gbs, "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                     "frac": achieved_gbs / peaks.get("hbm_gbs", 6650.0), "traffic": read_traffic("fock"),
                     "algorithmic_per_launch": f"{nbytes:.4g} B", "peak_source": "MEASURED_PEAKS.json hbm_gbs"}
    # whole-solve roofline: iterations x (Fock bytes / HBM + dense flops / FP64 peak), the
    # dense flops per iteration being an eigensolve (10/3 n^3), the density (n^2 n_occ) and the
    # commutator (2 n^3); the pair integrals (the build stage, ~0.3% of a solve) are not counted
    whole = None
    if dgemm and fock_calls:
        n_occ = int(r0["n_occ"])
        its = r0["iterations"]
        fock_b = 8.0 * (near_w_doubles(z, x) + 3.0 * nao * nao)
        dense = 10.0 / 3.0 * nao ** 3 + float(nao) ** 2 * n_occ + 2.0 * nao ** 3
        t_roof = its * (fock_b / (peaks.get("hbm_gbs", 6650.0) * 1e9) + dense / (dgemm * 1e12))
        t_meas = dev_s / args.steps
        whole = {"roofline_ms": t_roof * 1e3, "measured_ms": t_meas * 1e3, "frac": t_roof / t_meas,
                 "iterations": its, "dense_flops_per_iteration": dense, "fock_bytes_per_iteration": fock_b,
                 "note": "roofline time of the solve over its measured device time; pair integrals not counted"}
    extras = None
    if world == 1 and not args.no_extras and args.workload == "water334" and args.precision == "fp64":
        extras = default_extras(args, local)
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        t_cpu, it_cpu = cpu_sample_full(z, x)
        cpu = {"value": 1.0 / t_cpu, "unit": "solves/s", "cores": os.cpu_count(), "kind": "port",
               "sample": f"one complete oracle solve of the same {desc} ({it_cpu} iterations, {t_cpu:.1f} s)"}
    h2d = n_atoms * (1 + 24)
    d2h = 8 * n_atoms + 8 * nao + 8 * 30
    line = {
        "metric": "PM7 SCF solves/s (RHF single point)", "value": value, "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_s * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "data": "synthetic",
        "dtype": "f64" if args.precision == "fp64" else "f32 (tcgen05 3xTF32) + f64 refinement",
        "config": bench_config(args, desc, z, world),
        "e2e": {"value": e2e, "unit": "solves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                       "device_p50": float(np.percentile([q["device_ms"] for q in results], 50))},
        "roofline": roofline,
        "roofline_fock": fock_roof,
        "pair_integrals": pair_rate,
        "autotune": api.autotune_report(),
        "mixed_precision": mixed,
        "whole_solve_roofline": whole,
        "served_and_batched": extras,
        "gradient": grad,
        "stages": stages,
        "clocks": clocks,
        "cpu_baseline": cpu,
        "result": {"heat_of_formation_kcal": r0["heat_of_formation_kcal"], "total_ev": r0["total_ev"],
                   "scf_iterations": r0["iterations"]},
    }
    print(json.dumps(line), flush=True)


def default_extras(args, local):
    """The served stream (FP64 and mixed precision) and the 4,096-molecule batch, one pass
    each, for the default line: what the served/batched engine sustains against the plain
    path on the same requests."""
    sub = argparse.Namespace(**vars(args))
    sub.steps, sub.warmup, sub.no_gradient, sub.no_cpu_baseline = 1, 1, True, True
    out = {}
    for prec in ("fp64", "mixed"):
        sub.precision = prec
        ln = run_stream_bench(sub, 1, 0, local, oracle_check=True)
        out[f"stream_{prec}"] = {
            "solves_per_s": ln["value"], "latency_ms": ln["latency_ms"], "requests": ln["config"]["requests"],
            "rate_per_s": ln["config"]["rate_per_s"], "capacity_per_s": ln["config"]["capacity_per_s"],
            "plain_fp64_solves_per_s": ln["plain_path"]["value"],
            "served_over_plain": ln["plain_path"]["served_over_plain"],
            "sustained_solves_per_s": ln["sustained"]["value"],
            "sustained_over_plain": ln["plain_path"]["sustained_over_plain"],
            "capacity_over_plain": ln["plain_path"]["capacity_over_plain"],
            "max_dhf_diff_vs_plain_kcal": ln["plain_path"]["max_dhf_diff_kcal"],
            "oracle_check": ln.get("oracle_check"), "failed": ln["config"]["failed"], "clocks": ln["clocks"]}
    for prec in ("fp64", "mixed"):
        sub.precision = prec
        ln = run_batch_bench(sub, 1, 0, local)
        out[f"batch4096_{prec}"] = {
            "solves_per_s": ln["value"], "wall_s": ln["ms_per_step"] / 1e3,
            "plain_fp64_solves_per_s": ln["plain_path"]["value"],
            "batched_over_plain": ln["plain_path"]["batched_over_plain"],
            "max_dhf_diff_vs_plain_kcal": ln["plain_path"]["max_dhf_diff_kcal"],
            "failed": ln["config"]["failed_rank0"], "clocks": ln["clocks"]}
    return out


def _percentiles(v):
    return {"p50": float(np.percentile(v, 50)), "p99": float(np.percentile(v, 99)), "max": float(np.max(v))}


def _plain_sample(api, mols, idx, device):
    """The plain single-molecule path on a sample: (solves/s, results by index)."""
    out = {}
    t = time.perf_counter()
    for i in idx:
        z, x = mols[i]
        out[i] = api.run_pm7(z, x, device=device, want_matrices=0)
    return len(idx) / (time.perf_counter() - t), out


def _oracle_sample(mols, idx):
    from oracle import harness

    harness.set_threads(os.cpu_count() or 1)
    t = time.perf_counter()
    res = {}
    for i in idx:
        res[i] = harness.run(*mols[i], want_matrices=0)
    return len(idx) / (time.perf_counter() - t), res


def run_batch_bench(args, world, rank, local):
    """Configuration: 4,096 molecules of uneven size in one batched device run per GPU.

    With N ranks the batch is 4,096 x N molecules of one seeded draw, split by
    `pm7_batch_partition` (longest processing time by estimated cost); each rank
    solves its share on its own GPU, no collective on the solve path."""
    from pm7b200 import api, shard
    from pm7b200 import geometry as G

    every = G.batch(4096 * world, seed=0)
    mols = [every[i] for i in shard.shard_of(every, rank, world)]
    opts = dict(device=local, want_matrices=0, precision=1 if args.precision == "mixed" else 0)
    for _ in range(args.warmup):  # full batches: the grow-only device and pinned buffers reach size
        api.run_batch(mols, **opts)
    barrier(world)
    sampler = ClockSampler(local, interval_ms=500)  # multi-second timed region; driver queries stall CUDA calls
    sampler.start()
    launches0 = api.launch_count()
    walls = []
    res = None
    for _ in range(args.steps):
        t = time.perf_counter()
        res = api.run_batch(mols, **opts)
        walls.append(time.perf_counter() - t)
    launches = api.launch_count() - launches0
    clocks = sampler.stop()
    barrier(world)
    wall = allreduce_max(sum(walls), world)
    # stage split from one more, untimed batch (stage events synchronise, so they stay out of the timing)
    api.profile_enable(True)
    api.run_batch(mols, **opts)
    prof = api.profile_read()
    api.profile_enable(False)
    # the same batch with every molecule's nuclear gradient (pm7_run_batch_gradient), one pass
    grad = None
    if not args.no_gradient:
        t = time.perf_counter()
        gres = api.run_batch_gradient(mols, **opts)
        gw = allreduce_max(time.perf_counter() - t, world)
        grad = {"value": len(every) / gw, "unit": "SCF+gradient/s (pm7_run_batch_gradient, host buffers)",
                "wall_s": gw, "failed_rank0": sum(1 for r in gres if isinstance(r, Exception))}
    if rank != 0:
        return
    failed = sum(1 for r in res if isinstance(r, Exception))
    value = len(every) * args.steps / wall
    rng = np.random.default_rng(7)
    idx = sorted(rng.choice(len(mols), size=48, replace=False).tolist())
    plain, plain_res = _plain_sample(api, mols, idx, local)  # plain FP64 path
    dhf = max(abs(res[i]["heat_of_formation_kcal"] - plain_res[i]["heat_of_formation_kcal"]) for i in idx)
    cpu = None
    if not args.no_cpu_baseline:
        cidx = idx[:12]
        cpu_rate, cres = _oracle_sample(mols, cidx)
        dhf_oracle = max(abs(res[i]["heat_of_formation_kcal"] - cres[i]["heat_of_formation_kcal"]) for i in cidx)
        cpu = {"value": cpu_rate, "unit": "solves/s", "cores": os.cpu_count(), "kind": "port",
               "sample": f"12 molecules of the batch solved one by one by the oracle (max |dHf| vs batch "
                         f"{dhf_oracle:.2e} kcal/mol)"}
    natoms = [len(z) for z, _ in mols]
    line = {
        "metric": "PM7 SCF solves/s (batched RHF single points)", "value": value, "unit": "solves/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": wall * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "data": "synthetic",
        "dtype": "f64" if args.precision == "fp64" else "f32 (tcgen05 3xTF32) + f64 refinement",
        "config": {"workload": "batch4096", "molecules": len(every), "molecules_rank0": len(mols), "seed": 0,
                   "atoms_min": min(natoms), "atoms_max": max(natoms), "atoms_mean": float(np.mean(natoms)),
                   "failed_rank0": failed, "parallelism": f"lpt-shard{world}",
                   "l2": "each step streams the whole batch (GBs of per-molecule state) through HBM"},
        "e2e": {"value": value, "unit": "solves/s", "note": "wall clock around pm7_run_batch with host buffers"},
        "plain_path": {"value": plain, "unit": "solves/s", "sample": "48 molecules of the batch through pm7_run",
                       "batched_over_plain": value / plain, "max_dhf_diff_kcal": dhf},
        "gpu_launches": launches, "clocks": clocks, "cpu_baseline": cpu, "autotune": api.autotune_report(),
        "stages": {k: {"ms_total": round(v[0], 3), "calls": v[1]} for k, v in prof.items()},
        "stages_note": "one extra untimed batch with stage events",
        "gradient": grad,
    }
    return line


def run_stream_bench(args, world, rank, local, oracle_check=False):
    """Configuration: a served stream with Poisson arrivals at ~80% of capacity."""
    from pm7b200 import api
    from pm7b200 import geometry as G

    count = args.stream_count
    mols = G.stream(count, seed=rank)
    prec = 1 if args.precision == "mixed" else 0
    with api.Engine(device=local) as eng:
        # capacity: the whole stream submitted at once (the engine's saturated throughput on
        # these molecules), timed after untimed warm-up passes (first use of the engine:
        # buffers and memory pools sized for the full stream, launch shapes of its batch sizes)
        burst = mols[: min(count, 120)]
        for _ in range(max(1, args.warmup - 1)):
            for k in [eng.submit(z, x, want_matrices=0, precision=prec) for z, x in burst]:
                eng.poll(k, wait=True)
        for _ in range(2):  # the engine's throughput on a full stream settles on its third pass
            for k in [eng.submit(z, x, want_matrices=0, precision=prec) for z, x in mols]:
                eng.poll(k, wait=True)
        t = time.perf_counter()
        tk = [eng.submit(z, x, want_matrices=0, precision=prec) for z, x in mols]
        for k in tk:
            eng.poll(k, wait=True)
        capacity = len(mols) / (time.perf_counter() - t)
        rate = 0.8 * capacity
        rng = np.random.default_rng(11)
        gaps = rng.exponential(1.0 / rate, size=count)
        barrier(world)
        sampler = ClockSampler(local, interval_ms=500)  # multi-second timed region; driver queries stall CUDA calls
        sampler.start()
        launches0 = api.launch_count()
        tickets = [None] * count
        submitted = np.zeros(count)
        t0 = time.perf_counter()
        due = t0
        for i, (z, x) in enumerate(mols):
            due += gaps[i]
            now = time.perf_counter()
            if due > now:
                time.sleep(due - now)
            submitted[i] = time.perf_counter()
            tickets[i] = eng.submit(z, x, want_matrices=0, precision=prec)
        res = [eng.poll(tk, wait=True)[1] for tk in tickets]
        wall = time.perf_counter() - t0
        launches = api.launch_count() - launches0
        clocks = sampler.stop()
        # stage split from one more, untimed burst (stage events synchronise, so they stay out
        # of the timed stream)
        api.profile_enable(True)
        for k in [eng.submit(z, x, want_matrices=0, precision=prec) for z, x in burst]:
            eng.poll(k, wait=True)
        prof = api.profile_read()
        api.profile_enable(False)
    barrier(world)
    wall = allreduce_max(wall, world)
    if rank != 0:
        return
    ok = [r for r in res if not isinstance(r, Exception)]
    lat = [r["latency_ms"] for r in ok]
    value = len(ok) * world / wall
    # sustained rate: completions inside the steady window between the submissions of the
    # 10th and the 90th percentile request (no ramp-up, no drain), per second of that window
    finished = np.array([submitted[i] + r["latency_ms"] * 1e-3 for i, r in enumerate(res)
                         if not isinstance(r, Exception)])
    w0, w1 = submitted[count // 10], submitted[(9 * count) // 10]
    sustained = float(np.sum((finished >= w0) & (finished < w1))) / (w1 - w0) * world
    idx = list(range(0, count, max(1, count // 24)))[:24]
    plain, plain_res = _plain_sample(api, mols, idx, local)
    dhf = max(abs(res[i]["heat_of_formation_kcal"] - plain_res[i]["heat_of_formation_kcal"])
              for i in idx if not isinstance(res[i], Exception))
    natoms = [len(z) for z, _ in mols]
    line = {
        "metric": "PM7 SCF solves/s and p50/p99 latency (served stream)", "value": value, "unit": "solves/s",
        "n_gpus": world, "steps": 1, "warmup": 1, "ms_per_step": wall * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "data": "synthetic",
        "dtype": "f64" if args.precision == "fp64" else "f32 (tcgen05 3xTF32) + f64 refinement",
        "config": {"workload": "stream", "requests": count, "seed": rank, "arrival": "Poisson",
                   "rate_per_s": rate, "capacity_per_s": capacity, "capacity_probe": "all requests submitted at once", "atoms_min": min(natoms),
                   "atoms_max": max(natoms), "failed": count - len(ok), "parallelism": f"replicas{world}"},
        "latency_ms": _percentiles(lat),
        "e2e": {"value": value, "unit": "solves/s", "note": "submit to finish through pm7_engine, host buffers"},
        "plain_path": {"value": plain, "unit": "solves/s", "sample": f"{len(idx)} molecules of the stream via pm7_run",
                       "served_over_plain": value / plain, "sustained_over_plain": sustained / plain,
                       "capacity_over_plain": capacity * world / plain, "max_dhf_diff_kcal": dhf},
        "sustained": {"value": sustained, "unit": "solves/s",
                      "window": "completions between the submissions of the 10th and 90th percentile requests"},
        "gpu_launches": launches, "clocks": clocks,
        "stages": {k: {"ms_total": round(v[0], 3), "calls": v[1]} for k, v in prof.items()},
        "stages_note": f"one more untimed burst of {len(burst)} requests with stage events",
    }
    if oracle_check:
        # the served results against the FP64 oracle on the stream's smaller requests
        small = [i for i in range(count) if len(mols[i][0]) <= 120 and not isinstance(res[i], Exception)][:8]
        _, ores = _oracle_sample(mols, small)
        line["oracle_check"] = {
            "requests": len(small), "max_dhf_err_kcal": max(abs(res[i]["heat_of_formation_kcal"] -
                                                                ores[i]["heat_of_formation_kcal"]) for i in small),
            "max_charge_err": max(float(np.max(np.abs(res[i]["charges"] - ores[i]["charges"]))) for i in small)}
    return line


def run_dandc_bench(args, world, rank, local):
    """Configuration: the divide-and-conquer SCF of the flat chain C640H1282 (1,922 atoms),
    buffer 15 Bohr, cores of 8 atoms, p_tol 1e-7, SCF options e_tol 1e-10 / p_tol 1e-8 /
    max_scf 400: the largest system of pm7-rs's divide-and-conquer scaling series. One molecule
    per rank (replicas); each step is one pm7_run_dandc from host buffers to host results."""
    from pm7b200 import api
    from pm7b200 import geometry as G

    z, x = G.flat_alkane(args.dandc_carbons)
    dc = dict(buffer=15.0, core_size=8, p_tol=1.0e-7, max_scf=400)
    opts = dict(e_tol=1.0e-10, p_tol=1.0e-8, max_scf=400, device=local, want_matrices=0)
    for _ in range(args.warmup):
        r = api.run_dandc(z, x, dandc=dc, gradient=False, **opts)
    barrier(world)
    sampler = ClockSampler(local, interval_ms=500)
    sampler.start()
    launches0 = api.launch_count()
    walls = []
    for _ in range(args.steps):
        t = time.perf_counter()
        r = api.run_dandc(z, x, dandc=dc, gradient=False, **opts)
        walls.append(time.perf_counter() - t)
    launches = api.launch_count() - launches0
    clocks = sampler.stop()
    barrier(world)
    wall = allreduce_max(sum(walls), world)
    t = time.perf_counter()
    rg = api.run_dandc(z, x, dandc=dc, gradient=True, **opts)
    gwall = time.perf_counter() - t
    if rank != 0:
        return
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import harness

        zc, xc = G.flat_alkane(160)
        t = time.perf_counter()
        o = harness.run_dandc(zc, xc, dandc=dc, want_matrices=0, e_tol=1.0e-10, p_tol=1.0e-8, max_scf=400)
        tc = time.perf_counter() - t
        scale = len(z) / len(zc)  # the method is linear in the atom count at a fixed buffer
        cpu = {"value": 1.0 / (tc * scale), "unit": "solves/s", "cores": os.cpu_count(), "kind": "port",
               "sample": f"the oracle's D&C of C160H322 ({len(zc)} atoms, {o['iterations']} iterations, "
                         f"{tc:.1f} s) scaled by the atom ratio {scale:.2f} to the {len(z)}-atom chain"}
    n = len(z)
    line = {
        "metric": "PM7 divide-and-conquer SCF solves/s", "value": world * args.steps / wall, "unit": "solves/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": wall * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "data": "synthetic", "dtype": "f64",
        "config": {"workload": f"dandc{args.dandc_carbons}", "atoms": n, "nao": int(r["nao"]), "buffer_bohr": 15.0, "core_size": 8,
                   "subsystems": r["subsystems"], "largest_subsystem": r["largest_subsystem"],
                   "iterations": r["iterations"], "converged": r["converged"],
                   "stored_density_elements": r["stored_density_elements"], "parallelism": f"replicas{world}",
                   "l2": "the global density (nao^2 doubles) and the per-subsystem buckets exceed L2 together"},
        "e2e": {"value": world * args.steps / wall, "unit": "solves/s",
                "note": "wall clock around pm7_run_dandc with host buffers (partition, build, SCF, results)"},
        "per_iteration_ms": wall * 1e3 / args.steps / max(r["iterations"], 1),
        "gradient": {"wall_s": gwall, "unit": "s per pm7_run_dandc with the gradient",
                     "max_abs_ev_per_bohr": float(np.abs(rg["gradient"]).max())},
        "gpu_launches": launches, "clocks": clocks, "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="water334",
                    choices=["water334", "water1000", "decane", "batch4096", "stream", "dandc640"])
    ap.add_argument("--stream-count", type=int, default=1200)
    ap.add_argument("--dandc-carbons", type=int, default=640, help="dandc640: chain length (small cases for profiles)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="batch4096/stream: fp64, or fp32 tcgen05 purification cycles with fp64 refinement")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64-peak", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision solve of the default workload")
    ap.add_argument("--no-gradient", action="store_true", help="skip the nuclear-gradient figure of the default workload")
    ap.add_argument("--no-extras", action="store_true",
                    help="default workload: skip the served-stream and batch figures added to its line")
    args = ap.parse_args()
    if args.impl == "reference":
        # CPU only: rank 0 runs, the other ranks exit without joining a process group
        run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")))
        return
    # this arm runs the CPU checker (the OpenMP oracle) between GPU measurements: its idle worker
    # threads must sleep rather than spin on the cores the engine's host threads use (set before
    # the first OpenMP library loads; the reference arm keeps the default policy)
    os.environ.setdefault("OMP_WAIT_POLICY", "PASSIVE")
    world, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        elif args.workload == "batch4096":
            line = run_batch_bench(args, world, rank, local)
            if line:
                print(json.dumps(line), flush=True)
        elif args.workload == "stream":
            line = run_stream_bench(args, world, rank, local, oracle_check=not args.no_cpu_baseline)
            if line:
                print(json.dumps(line), flush=True)
        elif args.workload == "dandc640":
            run_dandc_bench(args, world, rank, local)
        else:
            run_b200(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
