#!/usr/bin/env python3
"""Benchmark: seconds per RHF energy + analytic gradient, mixed precision
(FP32 quartets below Q_ab Q_cd max|D| = 1e-3, incremental dP Fock builds)
against the plain FP64 GPU path, on C40H82 / STO-3G (282 basis functions,
all-anti geometry with sigma = 0.02 A seeded jitter); Fock builds per second.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c40h82|c20h42|c100h202|c10h22] [--no-cpu-baseline]
                    [--no-side] [--no-batch]

A step is one energy + gradient from scratch (one-electron integrals, SCF to
|dE| < 1e-10 and DIIS error < 1e-8, gradient) for one molecule.  With N > 1
(torchrun) every rank converges its own molecule (same workload, its own
jitter seed): weak scaling, no collective on the data path; value = the max
over ranks of the per-step time / N.  With --shard every rank holds the same
molecule and evaluates a cost-balanced share of its quartets, J/K and the
gradient all-reduced over NCCL after every build: strong scaling, value =
the max over ranks of the step time.

``value``  device time of the step on a resident system (shell pairs and
           Schwarz factors already on the GPU), CUDA events on the engine's
           stream, between steps an L2 flush (256 MiB write; the working set
           is L2-resident, so the flush is what keeps steps cold).
``e2e``    the same step through the public C-ABI call ``pyfacc_run`` from
           host coordinates: basis parsing, pair construction, host->device
           copies and the device->host read of energy and gradient included.
``roofline``  the dominant kernels, the J/K digestion classes: algorithmic
           FP64 flops of a full FP64 Fock build (and FP32 flops of an all-FP32
           build) on the converged density / the build's CUDA-event time, over
           the FMA peaks measured in the same run.
``cpu_baseline`` / ``--impl reference``  the CPU restatement of the
           reference's path (oracle/; the reference itself cannot be built:
           no Fortran compiler, Libint or LAPACK) on all host cores, timed on
           a bounded uniform sample of the same workload: the one-electron
           matrices in full, every k-th bra shell pair of a Fock build and of
           the gradient, one dense step (eigh + transforms), scaled to one
           energy + gradient with the oracle's own SCF iteration count for
           this molecule (tests/golden/c40h82_sto3g.json).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import tempfile
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "pyfacc-scf_b200")
sys.path.insert(0, PKG)

WORKLOADS = {
    "c40h82": dict(n=40, seed=40, basis="sto-3g", label="C40H82 RHF STO-3G (282 bf)"),
    "c20h42": dict(n=20, seed=1, basis="sto-3g", label="C20H42 RHF STO-3G (142 bf)"),
    "c10h22": dict(n=10, seed=1, basis="sto-3g", label="C10H22 RHF STO-3G (72 bf)"),
    "c100h202": dict(n=100, seed=4, basis="sto-3g", label="C100H202 RHF STO-3G (702 bf)"),
}
# SCF iterations of the oracle (core-Hamiltonian guess + DIIS, the
# reference's start, to dE < 1e-10 and DIIS error < 1e-8); read from the
# oracle fixtures when they hold the count, else these values, measured by
# running the oracle's SCF on the same molecules
ORACLE_SCF_ITERS = {"c20h42": 22, "c10h22": 21, "c40h82": 24}
# DRAM bytes per launch of the dominant J/K class kernel from one ncu capture
# (profiles/jk_kernel_fp64_c40h82.md): the working set is L2-resident
JK_TRAFFIC_BYTES = 4.73e6
JK_TRAFFIC_NOTE = ("dram read + write per launch of jk_kernel<double,1,0,0,0> (the largest class) in a full FP64 "
                   "C40H82 build (ncu, profiles/jk_kernel_fp64_c40h82.md)")


def metric_name(wl):
    return f"s per RHF energy+gradient (mixed precision), {WORKLOADS[wl]['label']}"


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def geometry(wl, rank=0):
    from pyfacc import geometry as G
    w = WORKLOADS[wl]
    return G.alkane(w["n"], seed=w["seed"] + 1000 * rank)


def molecule(wl, rank=0):
    import pyfacc
    sp, xyz = geometry(wl, rank)
    return pyfacc.Molecule(sp, xyz, WORKLOADS[wl]["basis"])


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        # raw samples go to $PYFACC_CLOCKS_DIR (default: the temp directory);
        # the JSON line carries their summary
        out = os.environ.get("PYFACC_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = os.path.join(out, f"clocks_gpu{index}.csv")

    def __enter__(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv",
                                          "-lms", "200"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        try:
            rows = [l.strip().split(", ") for l in open(self.path) if l[0].isdigit()]
        except OSError:
            return None
        if not rows:
            return None
        sm = [float(r[1].split()[0]) for r in rows]
        mx = float(rows[0][2].split()[0])
        loaded = [s for s in sm if s > 0.5 * mx] or sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if len(r) > 5 + k and r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows)}


def device_step(sys_):
    """One energy + gradient on a resident system; engine-stream event time (s)."""
    r = sys_.scf(check=False)
    g = sys_.gradient()
    t = (r.timings_ms["total"] + sys_.result().timings_ms["gradient"]) / 1e3
    return r, g, t


def timed_steps(sys_, steps, flush):
    import torch
    times, iters, builds = [], [], []
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        r, g, t = device_step(sys_)
        times.append(t)
        iters.append(r.n_iter)
        builds.append(r.n_fock_builds)
    return times, iters, builds


def jk_rates(sy, nb=20):
    """Full J/K builds on the system's converged density: builds per second
    (engine-stream CUDA events) and the algorithmic flops of each precision,
    for the FP64 lists, the mixed lists and all quartets in FP32."""
    import torch
    from pyfacc import _native as N
    from pyfacc.distributed import _CudaView
    n = sy.nbf
    ptr = ctypes.c_void_p()
    N.check(N.lib().pyfacc_system_density_dev(sy.handle, ctypes.byref(ptr)), "pyfacc_system_density_dev")
    P = torch.as_tensor(_CudaView(int(ptr.value), n * n), device="cuda").reshape(n, n).clone()
    out = {}
    for name in ("fp64", "mixed", "fp32"):
        for _ in range(3):
            sy.jk(P, precision=name)
        ms, f64, f32 = [], 0.0, 0.0
        for _ in range(nb):
            sy.jk(P, precision=name)
            st = sy.jk_stats()
            ms.append(st["ms"])
            f64, f32 = st["flops_fp64"], st["flops_fp32"]
        t = statistics.mean(ms) * 1e-3
        out[name] = {"builds_per_s": 1.0 / t, "ms_per_build": t * 1e3, "flops_fp64": f64, "flops_fp32": f32,
                     "tflops_fp64": f64 / t / 1e12, "tflops_fp32": f32 / t / 1e12}
    return out, P


def oracle_fixture(wl):
    path = os.path.join(ROOT, "tests", "golden", f"{wl}_sto3g.json")
    try:
        with open(path) as fh:
            return json.load(fh), os.path.relpath(path, ROOT)
    except OSError:
        return None, None


def oracle_iterations(wl):
    d, rel = oracle_fixture(wl)
    if d and "scf_iterations" in d:
        return int(d["scf_iterations"]), f"oracle SCF iterations from {rel}"
    return ORACLE_SCF_ITERS.get(wl, 24), "oracle SCF iterations measured by running oracle.scf on this molecule"


def full_run_note(wl):
    """The oracle's whole SCF + gradient of this molecule, timed once when its
    fixture was generated (on that machine's threads), for comparison with
    the sampled estimate."""
    d, rel = oracle_fixture(wl)
    if not d or "oracle_seconds" not in d:
        return None
    t = d["oracle_seconds"]
    return {"s": t.get("scf", 0.0) + t.get("gradient", 0.0), "threads": d.get("oracle_threads"), "source": rel}


def cpu_sample(wl, P=None, jk_stride=16, grad_stride=128):
    """The oracle (CPU restatement of the reference path, OpenMP on all host
    cores) on a bounded uniform sample of one energy + gradient of the
    workload, scaled to the whole: one-electron matrices in full, one dense
    SCF step (S^-1/2, X^T F X, eigh, density) in full, every jk_stride-th bra
    pair of a Fock build and every grad_stride-th bra / one-electron pair of
    the gradient.  P: a density (the engine's converged one, or None for the
    reference's own core-Hamiltonian guess, rscf.f90:113-114); the oracle's
    work does not depend on it (Schwarz screening only)."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    sp, xyz = geometry(wl, 0)
    mol = O.molecule(sp, xyz, os.path.join(PKG, "data", "basis_set", WORKLOADS[wl]["basis"] + ".txt"))
    n = mol.shells.nbf
    nocc = (mol.nalpha + mol.nbeta + 1) // 2
    t0 = time.perf_counter()
    S, T, V = O.one_electron(mol)
    H = T + V
    t_1e = time.perf_counter() - t0
    t0 = time.perf_counter()
    s, U = np.linalg.eigh(S)
    X = U / np.sqrt(s)
    e, Cp = np.linalg.eigh(X.T @ H @ X)
    C = X @ Cp
    Pg = 2.0 * C[:, :nocc] @ C[:, :nocc].T
    t_dense = time.perf_counter() - t0
    if P is None:
        P = Pg
    t0 = time.perf_counter()
    O.jk_sample(mol, P, jk_stride)
    t_jk = (time.perf_counter() - t0) * jk_stride
    t0 = time.perf_counter()
    O.gradient_sample(mol, P, 0.5 * P, 0.5 * P, P, grad_stride)
    t_grad = (time.perf_counter() - t0) * grad_stride
    iters, src = oracle_iterations(wl)
    value = t_1e + iters * (t_jk + t_dense) + t_grad
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count()))
    return {"value": value, "unit": "s", "cores": threads, "kind": "port",
            "sample": (f"oracle on {threads} threads, {WORKLOADS[wl]['label']}: one-electron S/T/V in full "
                       f"({t_1e:.2f} s), one dense SCF step ({t_dense:.3f} s), every {jk_stride}th bra pair of a "
                       f"Fock build (x{jk_stride} = {t_jk:.1f} s per build), every {grad_stride}th pair of the "
                       f"gradient (x{grad_stride} = {t_grad:.1f} s); value = 1e + {iters} x (build + dense) + "
                       f"gradient, {src}"),
            "parts_s": {"one_electron": t_1e, "fock_build": t_jk, "dense_step": t_dense, "gradient": t_grad},
            "scf_iterations": iters,
            "full_run_when_fixture_was_made": full_run_note(wl)}


def run_ours(args):
    import numpy as np
    import torch
    import pyfacc
    from pyfacc import _native as N

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    wl = args.workload
    shard = args.shard and world > 1
    mol = molecule(wl, 0 if shard else rank)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    if shard:
        # one molecule, its Fock builds and gradient split across the ranks
        # (cost-balanced bra-pair ranges), J/K and gradient all-reduced over
        # NCCL after every build: strong scaling
        from pyfacc.distributed import sharded_system
        s_mixed = sharded_system(mol, precision="mixed", device=local)
        s_fp64 = sharded_system(mol, precision="fp64", device=local)
    else:
        s_mixed = pyfacc.System(mol, precision="mixed", device=local)
        s_fp64 = pyfacc.System(mol, precision="fp64", device=local)
    for _ in range(max(args.warmup, 1)):
        rm, gm, _ = device_step(s_mixed)
        r64, g64, _ = device_step(s_fp64)
    dE = abs(rm.energy - r64.energy)
    dG = float(np.abs(gm - g64).max())

    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = N.lib().pyfacc_launch_count()
    with Clocks(local) as clk:
        t_mx, it_mx, nb_mx = timed_steps(s_mixed, args.steps, flush)
        launches = (N.lib().pyfacc_launch_count() - l0) // max(args.steps, 1)
        t_64, it_64, nb_64 = timed_steps(s_fp64, args.steps, flush)
    torch.cuda.synchronize()
    step_mx = statistics.mean(t_mx)
    step_64 = statistics.mean(t_64)
    if dist:
        t = torch.tensor([step_mx, step_64], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        step_mx, step_64 = t.tolist()
        dist.barrier()

    breakdown = {}
    for name, sy in (("mixed", s_mixed), ("fp64", s_fp64)):
        rr = sy.result()
        breakdown[name] = {k: round(v, 3) for k, v in rr.timings_ms.items()}
        breakdown[name]["scf_iterations"] = rr.n_iter
        breakdown[name]["fock_builds"] = rr.n_fock_builds
        breakdown[name]["quartets"] = rr.quartets

    # Fock builds on the converged density: rates and the J/K roofline
    rates, Pconv = jk_rates(s_fp64)
    rates_by_wl = {WORKLOADS[wl]["label"]: {k: v["builds_per_s"] for k, v in rates.items()}}

    # side measurements on rank 0: the other alkanes, and the batch
    side = {}
    if rank == 0 and not args.no_side:
        for swl in ("c20h42", "c100h202"):
            if swl == wl:
                continue
            res = {}
            for prec in ("fp64", "mixed"):
                sy = pyfacc.System(molecule(swl, 0), precision=prec, device=local)
                for _ in range(2):
                    device_step(sy)
                ts, _, _ = timed_steps(sy, 3, flush)
                r, g, _ = device_step(sy)
                res[prec] = (statistics.mean(ts), r.energy, g)
                if prec == "fp64":
                    rr, _ = jk_rates(sy, nb=10)
                    rates_by_wl[WORKLOADS[swl]["label"]] = {k: v["builds_per_s"] for k, v in rr.items()}
                sy.close()
            side[swl] = {"workload": WORKLOADS[swl]["label"], "fp64_s": res["fp64"][0], "mixed_s": res["mixed"][0],
                         "mixed_speedup_vs_fp64": res["fp64"][0] / res["mixed"][0],
                         "delta_e": abs(res["fp64"][1] - res["mixed"][1]),
                         "max_grad_diff": float(np.abs(res["fp64"][2] - res["mixed"][2]).max()),
                         "timing": "mean of 3 device-timed steps after 2 warm-up steps"}
    batch = None
    if rank == 0 and not args.no_batch:
        batch = batch_measurement(pyfacc, local)

    # e2e through the C ABI with host buffers
    m, keep = mol._struct()
    opt = pyfacc._options(precision="mixed", compute_gradient=1, device=local)
    grad = np.zeros((mol.natoms, 3))
    e2e = []
    for i in range(args.warmup + args.steps):
        res = N.Result()
        res.gradient = grad.ctypes.data_as(N.P_double)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st = N.lib().pyfacc_run(ctypes.byref(m), ctypes.byref(opt), ctypes.byref(res))
        dt = time.perf_counter() - t0
        N.check(st, "pyfacc_run", allow=(N.OK,))
        if i >= args.warmup:
            e2e.append(dt)
    e2e_step = statistics.mean(e2e)
    if dist:
        t = torch.tensor([e2e_step], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_step = t.item()

    peak64 = peak32 = None
    if rank == 0:
        p32 = ctypes.c_double()
        peak64 = N.lib().pyfacc_probe_fp64_gflops(local, ctypes.byref(p32))
        peak32 = p32.value

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_sample(wl, Pconv.cpu().numpy())

    if dist:
        dist.destroy_process_group()
    if rank != 0:
        return
    h2d = mol.natoms * (3 * 8 + 4 + 2) + len(mol.basis) + 1
    d2h = 8 + mol.natoms * 3 * 8
    a64 = rates["fp64"]["tflops_fp64"]
    a32 = rates["fp32"]["tflops_fp32"]
    roof = {
        "kernel": "J/K digestion (jk_kernel<double, class> x 6 classes), full FP64 Fock build on the converged "
                  "density",
        "bound": "fp64",
        "achieved": a64,
        "peak": peak64 / 1e3 if peak64 else None,
        "unit": "TFLOP/s",
        "frac": (a64 / (peak64 / 1e3)) if peak64 else None,
        "traffic": JK_TRAFFIC_BYTES,
        "traffic_note": JK_TRAFFIC_NOTE,
        "peak_source": "measured in this run: FP64 FMA microbenchmark (pyfacc_probe_fp64_gflops); "
                       "MEASURED_PEAKS.json holds no FP64/FP32 CUDA-core figure",
        "algorithmic_flops_per_build": rates["fp64"]["flops_fp64"],
        "ms_per_build": rates["fp64"]["ms_per_build"],
        "fp32": {"kernel": "jk_kernel<float, class> x 6, every quartet in FP32, converged density",
                 "bound": "fp32", "achieved": a32, "peak": peak32 / 1e3 if peak32 else None, "unit": "TFLOP/s",
                 "frac": (a32 / (peak32 / 1e3)) if peak32 else None,
                 "algorithmic_flops_per_build": rates["fp32"]["flops_fp32"],
                 "ms_per_build": rates["fp32"]["ms_per_build"]},
    }
    clk_s = clk.summary()
    out = {
        "metric": metric_name(wl),
        "value": step_mx if shard else step_mx / world,
        "unit": "s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": step_mx * 1e3,
        "higher_is_better": False,
        "scaling": "strong" if shard else "weak",
        "vs_baseline": None,
        "dtype": "f64+f32 (mixed); f64 for the plain path",
        "data": "synthetic, seeded (geometry builder pyfacc.geometry.alkane)",
        "config": {"workload": WORKLOADS[wl]["label"], "precision": "mixed",
                   "schwarz_thresh": 1e-12, "fp32_thresh": 1e-3, "scf": "dE<1e-10, DIIS err<1e-8",
                   "coarse_err": 1e-3, "gradient_fp32_thresh": 1e-1,
                   "mixed_energy": "last incremental mixed build (no FP64 polish build)",
                   "l2": "flushed between steps (256 MiB write)",
                   "parallelism": f"one molecule sharded x{world} (NCCL all-reduce of J/K)" if shard
                   else f"replicas x{world}"},
        "fp64_s_per_step": step_64 if shard else step_64 / world,
        "mixed_speedup_vs_fp64": step_64 / step_mx,
        "delta_e_mixed_vs_fp64": dE,
        "max_grad_diff_mixed_vs_fp64": dG,
        "scf_iterations": {"mixed": it_mx[0], "fp64": it_64[0]},
        "fock_builds_per_step": {"mixed": nb_mx[0], "fp64": nb_64[0]},
        "step_times_s": {"mixed": t_mx, "fp64": t_64},
        "fock_builds_per_s": rates["fp64"]["builds_per_s"],
        "fock_builds_per_s_by_workload": rates_by_wl,
        "breakdown_ms": breakdown,
        "side": side,
        "batch_water256": batch,
        "e2e": {"value": e2e_step if shard else e2e_step / world, "unit": "s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                "api": "pyfacc_run (C ABI, host coordinates in, energy + gradient out)"},
        "gpu_launches": int(launches),
        "roofline": roof,
        "peaks_measured": {"fp64_gflops": peak64, "fp32_gflops": peak32},
        "cpu_baseline": cpu,
        "clocks": clk_s,
    }
    print(json.dumps(out))


def batch_measurement(pyfacc, device):
    """256 water clusters (H2O)n, n ~ U{4..16} (rng seed 3), STO-3G RHF,
    energies + gradients of all molecules in one pyfacc_run_batch call
    (host coordinates in, host energies and gradients out), mixed precision
    and FP64, mean of 3 calls after a warm-up call; a sample of the same
    molecules one by one through pyfacc_run for comparison."""
    import numpy as np
    from pyfacc import geometry as G
    clusters = G.water_clusters(count=256, seed=3)
    mols = [pyfacc.Molecule(sp, xyz, "sto-3g") for sp, xyz in clusters]
    out = {"workload": "256 water clusters (H2O)n, n in [4,16], 28-112 bf, STO-3G RHF, energy+gradient",
           "molecules": len(mols)}
    res = {}
    for prec in ("mixed", "fp64"):
        pyfacc.run_batch(mols, gradient=True, precision=prec, device=device)  # warm-up (task-width tuning)
        ts = []
        for _ in range(3):
            t0 = time.perf_counter()
            r = pyfacc.run_batch(mols, gradient=True, precision=prec, device=device)
            ts.append(time.perf_counter() - t0)
        st = pyfacc.batch_stats()
        res[prec] = r
        tm = statistics.mean(ts)
        out[prec] = {"s_per_batch": tm, "s_per_batch_samples": ts, "ms_per_molecule": tm * 1e3 / len(mols),
                     "molecules_per_s": len(mols) / tm,
                     "converged": int(sum(x.converged for x in r)),
                     "breakdown_ms": {k: round(st[k], 2) for k in ("ms_setup", "ms_one_electron", "ms_scf",
                                                                     "ms_polish", "ms_gradient")},
                     "iterations": int(st["iterations"]), "task_width": st["task_width"],
                     "fock_tflops": st["flops_fock"] / max(st["ms_scf"] + st["ms_polish"], 1e-9) / 1e9}
    out["mixed_speedup_vs_fp64"] = out["fp64"]["s_per_batch"] / out["mixed"]["s_per_batch"]
    out["delta_e_mixed_vs_fp64"] = max(abs(a.energy - b.energy) for a, b in zip(res["mixed"], res["fp64"]))
    out["max_grad_diff_mixed_vs_fp64"] = max(float(np.abs(a.gradient - b.gradient).max())
                                             for a, b in zip(res["mixed"], res["fp64"]))
    sample = mols[:16]
    for m in sample[:2]:
        pyfacc.run(m, gradient=True, precision="mixed", device=device)
    t0 = time.perf_counter()
    for m in sample:
        pyfacc.run(m, gradient=True, precision="mixed", device=device)
    seq = (time.perf_counter() - t0) / len(sample)
    out["one_by_one_ms_per_molecule"] = seq * 1e3
    out["batch_speedup_vs_one_by_one"] = seq / (out["mixed"]["s_per_batch"] / len(mols))
    return out


def run_reference(args):
    """The CPU restatement of the reference path (oracle/) on all host
    cores, with the reference's own start (core-Hamiltonian guess density):
    per step a bounded uniform sample of one energy + gradient of the
    workload (cpu_sample), scaled to the whole.  Under torchrun only rank 0
    runs it."""
    rank, world, local = dist_env()
    if rank != 0:
        return
    wl = args.workload
    for _ in range(args.warmup):
        cpu_sample("c10h22", None, jk_stride=64, grad_stride=512)  # warm-up: small, loads the oracle
    samples = []
    cb = None
    for _ in range(args.steps):
        cb = cpu_sample(wl, None)
        samples.append(cb["value"])
    value = statistics.mean(samples)
    cb["value"] = value
    cb["samples_s"] = samples
    out = {
        "impl": "reference",
        "metric": metric_name(wl),
        "value": value, "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic, seeded", "config": {"workload": WORKLOADS[wl]["label"]},
        "cpu_baseline": cb,
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "CPU restatement of the reference path (oracle/): the reference cannot be built here "
                "(no gfortran/nvfortran, Libint 2.11.1 or LAPACK) and its ERI path is incomplete; "
                "warm-up steps run a small sample (C10H22)",
    }
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c40h82", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-side", action="store_true", help="skip the C20H42 / C100H202 side measurements")
    ap.add_argument("--no-batch", action="store_true", help="skip the 256-water-cluster batch measurement")
    ap.add_argument("--shard", action="store_true",
                    help="with N > 1: one molecule sharded over the ranks (strong scaling) instead of replicas")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        print("note: fewer than 3 warm-up steps", file=sys.stderr)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
