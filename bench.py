#!/usr/bin/env python3
"""Benchmark: seconds per RHF energy + analytic gradient, mixed precision
(FP32 quartets below a Schwarz bound of 1e-5, incremental dP Fock builds)
against the plain FP64 GPU path, on C20H42 / STO-3G (142 basis functions,
all-anti geometry with sigma = 0.02 A seeded jitter); Fock builds per second.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c20h42|c40h82|h2o] [--no-cpu-baseline]

A step is one energy + gradient from scratch (one-electron integrals, SCF to
|dE| < 1e-10 and DIIS error < 1e-8, gradient) for one molecule.  With N > 1
(torchrun) every rank converges its own molecule (same workload, its own
jitter seed): weak scaling, no collective on the data path; value = N / the
max over ranks of the per-step time.

``value``  device time of the step on a resident system (shell pairs and
           Schwarz factors already on the GPU), CUDA events on the engine's
           stream, between steps an L2 flush (256 MiB write).
``e2e``    the same step through the public C-ABI call ``pyfacc_run`` from
           host coordinates: basis parsing, pair construction, host->device
           copies and the device->host read of energy and gradient included.
``--impl reference`` times the CPU restatement of the reference's path (the
           reference itself cannot be built: no Fortran compiler, Libint or
           LAPACK) on all host cores: a bounded sample of Fock builds, scaled
           to one energy + gradient.
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

METRIC = "s per RHF energy+gradient (mixed precision), C20H42/STO-3G"
# SCF iterations of the oracle (core-Hamiltonian guess + DIIS, the
# reference's start) for the workloads, measured in this repository
REF_SCF_ITERS = {"c20h42": 22, "c10h22": 21, "c40h82": 24}

WORKLOADS = {
    "c20h42": dict(n=20, seed=1, basis="sto-3g", label="C20H42 RHF STO-3G (142 bf)"),
    "c40h82": dict(n=40, seed=40, basis="sto-3g", label="C40H82 RHF STO-3G (282 bf)"),
    "c10h22": dict(n=10, seed=1, basis="sto-3g", label="C10H22 RHF STO-3G (72 bf)"),
    "c100h202": dict(n=100, seed=4, basis="sto-3g", label="C100H202 RHF STO-3G (702 bf)"),
}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def molecule(wl, rank=0):
    import pyfacc
    from pyfacc import geometry as G
    w = WORKLOADS[wl]
    sp, xyz = G.alkane(w["n"], seed=w["seed"] + 1000 * rank)
    return pyfacc.Molecule(sp, xyz, w["basis"])


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


def flush_l2(buf):
    buf.zero_()


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
    mol = molecule(args.workload, rank)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def device_step(sys_, grad=True):
        r = sys_.scf(check=False)
        g = sys_.gradient() if grad else None
        return r, g

    common = dict(device=local)
    s_mixed = pyfacc.System(mol, precision="mixed", **common)
    s_fp64 = pyfacc.System(mol, precision="fp64", **common)
    # warm-up (also the accuracy comparison)
    for _ in range(max(args.warmup, 1)):
        rm, gm = device_step(s_mixed)
        r64, g64 = device_step(s_fp64)
    dE = abs(rm.energy - r64.energy)
    dG = float(np.abs(gm - g64).max())

    def timed(sys_, steps):
        times, fock_ms, fock_flops, iters, ev_ms = [], 0.0, 0.0, [], []
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for _ in range(steps):
            flush_l2(flush)
            torch.cuda.synchronize()
            e0.record()
            r, g = device_step(sys_)
            e1.record()
            torch.cuda.synchronize()
            # engine-stream events: SCF (1e .. final diagonalisation) + gradient
            times.append((r.timings_ms["total"] + sys_.result().timings_ms["gradient"]) / 1e3)
            ev_ms.append(e0.elapsed_time(e1))
            fock_ms += r.timings_ms["fock"]
            fock_flops += r.flops["fock"]
            iters.append(r.n_iter)
        return times, fock_ms, fock_flops, iters, ev_ms

    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = N.lib().pyfacc_launch_count()
    with Clocks(local) as clk:
        t_mx, fock_ms_mx, fock_fl_mx, it_mx, ev_mx = timed(s_mixed, args.steps)
        launches = (N.lib().pyfacc_launch_count() - l0) // max(args.steps, 1)
        t_64, fock_ms_64, fock_fl_64, it_64, ev_64 = timed(s_fp64, args.steps)
    torch.cuda.synchronize()
    step_mx = statistics.mean(t_mx)
    step_64 = statistics.mean(t_64)
    if dist:
        t = torch.tensor([step_mx, step_64], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        step_mx, step_64 = t.tolist()
        dist.barrier()

    # Fock builds per second: J/K builds on the converged density (FP64
    # lists, and the FP64 + FP32 lists of mixed mode), mean of 20
    def fock_rates(sy):
        n = sy.nbf
        Pdev = ctypes.c_void_p()
        N.lib().pyfacc_system_density_dev(sy.handle, ctypes.byref(Pdev))
        J = torch.zeros(n, n, dtype=torch.float64, device="cuda")
        K = torch.zeros(n, n, dtype=torch.float64, device="cuda")
        out = {}
        for name, prec in (("fp64", N.PRECISION_FP64), ("mixed", N.PRECISION_MIXED)):
            for _ in range(3):
                N.lib().pyfacc_system_jk(sy.handle, Pdev, 1, Pdev, J.data_ptr(), K.data_ptr(), prec)
            nb = 20
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(nb):
                N.lib().pyfacc_system_jk(sy.handle, Pdev, 1, Pdev, J.data_ptr(), K.data_ptr(), prec)
            torch.cuda.synchronize()
            out[name] = nb / (time.perf_counter() - t0)
        return out

    rates = {WORKLOADS[args.workload]["label"]: fock_rates(s_fp64)}
    fock_s = 1.0 / rates[WORKLOADS[args.workload]["label"]]["fp64"]
    breakdown = {}
    for name, sy in (("mixed", s_mixed), ("fp64", s_fp64)):
        rr = sy.result()
        breakdown[name] = {k: round(v, 3) for k, v in rr.timings_ms.items()}
        breakdown[name]["scf_iterations"] = rr.n_iter
        breakdown[name]["quartets"] = rr.quartets

    # the larger alkane, C40H82 / STO-3G (282 bf), mixed vs FP64, on rank 0 only
    c40 = None
    if rank == 0 and args.workload == "c20h42" and not args.no_c40:
        m40 = molecule("c40h82", 0)
        res40 = {}
        for prec in ("fp64", "mixed"):
            sy = pyfacc.System(m40, precision=prec, device=local)
            for _ in range(2):
                device_step(sy)
            ts = []
            for _ in range(2):
                flush_l2(flush)
                r, g = device_step(sy)
                ts.append((r.timings_ms["total"] + sy.result().timings_ms["gradient"]) / 1e3)
            res40[prec] = (min(ts), r.energy, g)
            if prec == "fp64":
                rates[WORKLOADS["c40h82"]["label"]] = fock_rates(sy)
            sy.close()
        c40 = {"workload": WORKLOADS["c40h82"]["label"], "fp64_s": res40["fp64"][0], "mixed_s": res40["mixed"][0],
               "mixed_speedup_vs_fp64": res40["fp64"][0] / res40["mixed"][0],
               "delta_e": abs(res40["fp64"][1] - res40["mixed"][1]),
               "max_grad_diff": float(np.abs(res40["fp64"][2] - res40["mixed"][2]).max())}

    if rank == 0 and args.workload == "c20h42" and not args.no_c40:
        sy = pyfacc.System(molecule("c100h202", 0), precision="fp64", device=local)
        sy.scf(check=False)
        rates[WORKLOADS["c100h202"]["label"]] = fock_rates(sy)
        sy.close()

    # batch of 256 water clusters (H2O)n, n uniform in [4, 16], rank 0 only:
    # one pyfacc_run_batch call = energies and gradients of all 256 molecules
    batch = None
    if rank == 0 and args.workload == "c20h42" and not args.no_batch:
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
        N.lib().pyfacc_run(ctypes.byref(m), ctypes.byref(opt), ctypes.byref(res))
        dt = time.perf_counter() - t0
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
        cpu = cpu_baseline(args.workload, 0, n_fock_builds=REF_SCF_ITERS.get(args.workload, 22))

    if dist:
        dist.destroy_process_group()
    if rank != 0:
        return
    h2d = mol.natoms * (3 * 8 + 4 + 2) + len(mol.basis) + 1
    d2h = 8 + mol.natoms * 3 * 8
    fock_tflops = fock_fl_64 / (fock_ms_64 * 1e-3) / 1e12 if fock_ms_64 > 0 else None
    roof = {
        "kernel": "J/K digestion (jk_kernel<double, class>), FP64 plain path",
        "bound": "fp64",
        "achieved": fock_tflops,
        "peak": peak64 / 1e3 if peak64 else None,
        "unit": "TFLOP/s",
        "frac": (fock_tflops / (peak64 / 1e3)) if (fock_tflops and peak64) else None,
        "peak_source": "measured in this run: FP64 FMA microbenchmark (pyfacc_probe_fp64_gflops)",
        # DRAM bytes per launch of the dominant class kernel (ps|ss), FP64,
        # from one ncu capture (profiles/jk_kernel_fp64_c20h42.md): the
        # working set is L2-resident, so DRAM traffic is a few MB per launch
        "traffic": 2.06e6,
        "traffic_unit": "bytes per launch (dram read + write), jk_kernel<double,1,0,0,0> at C20H42",
        "algorithmic_flops_per_build": fock_fl_64 / max(1, sum(it_64)),
    }
    clk_s = clk.summary()
    out = {
        "metric": METRIC if args.workload == "c20h42"
        else f"s per RHF energy+gradient (mixed precision), {WORKLOADS[args.workload]['label']}",
        "value": step_mx * 1.0 / world,
        "unit": "s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": step_mx * 1e3,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64+f32 (mixed); f64 for the plain path",
        "data": "synthetic, seeded (geometry builder pyfacc.geometry.alkane)",
        "config": {"workload": WORKLOADS[args.workload]["label"], "precision": "mixed",
                   "schwarz_thresh": 1e-12, "fp32_thresh": 1e-5, "scf": "dE<1e-10, DIIS err<1e-8",
                   "coarse_err": 1e-3, "gradient_fp32_thresh": 1e-3,
                   "mixed_energy": "last incremental mixed build (no FP64 polish build)",
                   "l2": "flushed between steps (256 MiB write)", "parallelism": f"replicas x{world}"},
        "fp64_s_per_step": step_64 / world,
        "mixed_speedup_vs_fp64": step_64 / step_mx,
        "delta_e_mixed_vs_fp64": dE,
        "max_grad_diff_mixed_vs_fp64": dG,
        "scf_iterations": {"mixed": it_mx[0], "fp64": it_64[0]},
        "fock_builds_per_s": 1.0 / fock_s,
        "fock_builds_per_s_by_workload": rates,
        "breakdown_ms": breakdown,
        "c40h82": c40,
        "batch_water256": batch,
        "wall_bracket_ms": {"mixed": statistics.mean(ev_mx), "fp64": statistics.mean(ev_64)},
        "e2e": {"value": e2e_step / world, "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "api": "pyfacc_run (C ABI, host coordinates)"},
        "gpu_launches": None,
        "roofline": roof,
        "peaks_measured": {"fp64_gflops": peak64, "fp32_gflops": peak32},
        "cpu_baseline": cpu,
        "clocks": clk_s,
    }
    out["gpu_launches"] = int(launches)
    print(json.dumps(out))


def batch_measurement(pyfacc, device):
    """256 water clusters (H2O)n, n ~ U{4..16} (rng seed 3), STO-3G RHF,
    energies + gradients of all molecules in one pyfacc_run_batch call
    (host coordinates in, host energies and gradients out), mixed precision
    and FP64; a sample of the same molecules one by one through pyfacc_run
    for comparison."""
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
        for _ in range(2):
            t0 = time.perf_counter()
            r = pyfacc.run_batch(mols, gradient=True, precision=prec, device=device)
            ts.append(time.perf_counter() - t0)
        st = pyfacc.batch_stats()
        res[prec] = r
        out[prec] = {"s_per_batch": min(ts), "ms_per_molecule": min(ts) * 1e3 / len(mols),
                     "molecules_per_s": len(mols) / min(ts),
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


def cpu_baseline(wl, n_iter, n_fock_builds):
    """The oracle's OpenMP J/K (the CPU restatement of the reference path) on
    the same molecule: one full Fock build timed, scaled by the number of
    Fock builds of the GPU run plus 4 build-equivalents for the gradient."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from pyfacc import geometry as G
    w = WORKLOADS[wl]
    sp, xyz = G.alkane(w["n"], seed=w["seed"])
    mol = O.molecule(sp, xyz, os.path.join(PKG, "data", "basis_set", w["basis"] + ".txt"))
    n = mol.shells.nbf
    D = np.eye(n) * 0.5
    t0 = time.perf_counter()
    O.jk(mol, D, thresh=1e-12)
    tb = time.perf_counter() - t0
    builds = n_fock_builds + 4
    return {"value": tb * builds, "unit": "s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"one FP64 J/K build of {w['label']} on {os.cpu_count()} threads ({tb:.2f} s), "
                      f"x ({n_fock_builds} SCF builds of the oracle + 4 for the gradient)"}


def run_reference(args):
    """The CPU restatement of the reference path (oracle/) on all host
    cores: per step one full J/K build of the workload (the hot loop of
    rscf.f90:118-135 done integral-direct), scaled to one energy + gradient
    by the oracle's own SCF iteration count for this molecule (core guess,
    DIIS) plus 4 build-equivalents for the gradient."""
    rank, world, local = dist_env()
    if rank != 0:
        return
    samples = []
    for i in range(args.warmup + args.steps):
        cb = cpu_baseline(args.workload, 0, n_fock_builds=REF_SCF_ITERS.get(args.workload, 22))
        if i >= args.warmup:
            samples.append(cb["value"])
    value = statistics.mean(samples)
    cb["value"] = value
    out = {
        "impl": "reference",
        "metric": METRIC if args.workload == "c20h42" else f"s per RHF energy+gradient, {WORKLOADS[args.workload]['label']}",
        "value": value, "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic, seeded", "config": {"workload": WORKLOADS[args.workload]["label"]},
        "cpu_baseline": cb,
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "CPU restatement of the reference path (oracle/): the reference cannot be built here "
                "(no gfortran/nvfortran, Libint 2.11.1 or LAPACK) and its ERI path is incomplete",
    }
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c20h42", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-c40", action="store_true", help="skip the C40H82 side measurement")
    ap.add_argument("--no-batch", action="store_true", help="skip the 256-water-cluster batch measurement")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
