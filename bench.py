"""Benchmark: batched PM3 single points on B200 (pm3gpu) beside the CPU reference path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl pm3gpu|reference] [--n-mol M]

Workload (one step): 4096 seeded, neutral, closed-shell C/H/N/O/S organics of 5-60 atoms
(uniform size), plain FP64 RHF PM3 with the reference's default options (A-DIIS -> CDIIS,
e_tol 1e-8 eV, p_tol 1e-7, stability search on), every molecule to convergence. The metric is
converged single points per second over the whole job. Under torchrun every rank solves its
own 4096 molecules (seed offset by rank): weak scaling, no data-path collective.

`value`: inputs (atom numbers and coordinates) already resident in HBM, CUDA-event time on the
device. `e2e`: the same through the host C ABI (pm3gpu_batch) from pinned host buffers,
host<->device copies inside the timed region. By default four batches are in flight (four
contexts, each with its own stream and host thread) and the device time spans all K steps; L2 is
flushed (a 512 MiB write) before them and the per-CTA workspaces exceed L2. With `--inflight 1`
each step is timed alone with a flush between steps. The headline (plain) arm uses the built-in
launch choice and the reference's defaults; the tuned arm beside it calibrates the launch choice
on another sample of the same generator and adds the learned guess and mixed precision.
`--impl reference` times the reference algorithm's CPU implementation (the C++ oracle that
restates pm3-rs, linked to SciPy's OpenBLAS) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "pm3-rs_b200"))
A2B = 1.0 / 0.529177210903
# the headline metric: batched converged single points per second, and seconds per SCF of the
# 6000-atom system, tuned modes beside plain FP64, heats of formation within 0.01 kcal/mol
METRIC = "converged SCF/s (batched) & s/SCF @6k atoms: tuned vs plain FP64 GPU, \u0394Hf\u22641e-2"
WORKLOAD = "organics-4096: seeded C/H/N/O/S trees, 5-60 atoms uniform, RHF PM3 FP64, reference default options"
WORKLOAD_D3H4 = ("d3h4-4096: the organics-4096 molecules with method PM3-D3H4 (the SCF plus the D3, H4 and H-H "
                 "corrections on the device), reference default options")


# ------------------------------------------------------------------------- CPU (oracle) side
def _oracle_worker(args):
    mols, opts = args
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    n_conv = 0
    for z, xyz in mols:
        try:
            r = O.single_point(z, xyz, **opts)
            n_conv += int(r["converged"])
        except Exception:
            pass
    return n_conv


def _oracle_hess_worker(mols):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import hessian_ref

    n_ok = 0
    for z, xyz in mols:
        try:
            hessian_ref.numerical_hessian(z, xyz)
            n_ok += 1
        except Exception:
            pass
    return n_ok


def _oracle_opt_worker(mols):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import lbfgs_ref

    n_conv = 0
    for z, xyz in mols:
        try:
            n_conv += int(lbfgs_ref.optimize(z, xyz)["converged"])
        except Exception:
            pass
    return n_conv


def cpu_throughput(mols, cores, steps=1, warmup=0, opts=None):
    """Converged molecules/s of the oracle over `mols` on `cores` spawn workers (one thread each)."""
    import multiprocessing as mp

    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    os.environ["OMP_NUM_THREADS"] = "1"
    ctx = mp.get_context("spawn")
    chunks = [mols[i::cores] for i in range(cores)]
    with ctx.Pool(cores) as pool:
        o = opts or {}
        pool.map(_oracle_worker, [(c[:1], o) for c in chunks])  # start-up outside the timing
        for _ in range(warmup):
            pool.map(_oracle_worker, [(c, o) for c in chunks])
        rates = []
        for _ in range(max(steps, 1)):
            t0 = time.perf_counter()
            n = sum(pool.map(_oracle_worker, [(c, o) for c in chunks]))
            rates.append((n, time.perf_counter() - t0))
    return rates


def molecules(n_mol, seed, workload="organics-4096", only=None):
    from pm3_rs import workloads

    if workload == "radicals-2048":
        mols = workloads.radical_batch(n_mol, 10, 80, seed=seed, only=only)
    else:
        mols = workloads.organic_batch(n_mol, 5, 60, seed=seed, only=only)
    return [(z, xyz * A2B) for z, xyz in mols]


def rank_molecules(n_per_rank, rank, world, workload="organics-4096", seed=1234):
    """This rank's part of ONE batch of n_per_rank x world molecules: the batch is partitioned over
    the ranks by the longest-processing-time rule on a size cost (atoms^3; the atom counts are drawn
    without building the molecules), and each rank builds only its own molecules. Weak scaling."""
    from pm3_rs import sharding, workloads

    n = n_per_rank * world
    if workload == "radicals-2048":
        sizes = np.random.default_rng(seed).integers(10, 81, n)
    else:
        sizes = workloads.organic_batch_sizes(n, 5, 60, seed)
    parts = sharding.partition_costs(sizes.astype(np.float64) ** 3, world)
    return molecules(n, seed, workload, only=parts[rank])


RADICALS = "radicals-2048: seeded C/H/N/O/S organics of 10-80 atoms minus one H (doublets), UHF PM3 FP64 + analytic gradients, reference default options"


def workload_spec(args):
    """(description, oracle options, GPU option overrides, gradients?, default batch size)."""
    if args.workload == "radicals-2048":
        return RADICALS, {"multiplicity": 2, "want_gradient": True}, {"multiplicity": 2}, True, 2048
    if args.workload == "d3h4-4096":
        return WORKLOAD_D3H4, {"variant": 2}, {"variant": 2}, False, 4096
    return WORKLOAD, {}, {}, False, 4096


# --------------------------------------------------------------------------- ranks
def shard_seed(rank, base=1234):
    """Seed of one rank's batch: every rank solves its own molecules (weak scaling; the batch
    shards by molecules, so there is no data-path collective)."""
    return base + 7919 * rank


def reduce_over_ranks(tot, e_tot, conv, e_conv, dist, device):
    """Whole-job numbers: the slowest rank's device times (ms) and the converged counts summed
    over ranks. `dist` is torch.distributed or None for one process."""
    if not dist:
        return tot, e_tot, conv, e_conv
    import torch

    t_max = torch.tensor([tot, e_tot], dtype=torch.float64, device=device)
    c_sum = torch.tensor([float(conv), float(e_conv)], dtype=torch.float64, device=device)
    dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
    dist.all_reduce(c_sum, op=dist.ReduceOp.SUM)
    return float(t_max[0]), float(t_max[1]), int(c_sum[0]), int(c_sum[1])


# --------------------------------------------------------------------------- GPU helpers
def gpu_uuid(dev):
    import torch

    try:
        return str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid):
        self.uuid = uuid
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *exc):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self):
        self.f.flush()
        rows = []
        try:
            for line in open(self.f.name):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                if self.uuid and self.uuid not in parts[0]:
                    continue
                rows.append(parts)
        finally:
            os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        reasons = set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            for k, nm in enumerate(names):
                if r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def fp64_gemm_peak(dev):
    """Measured FP64 dense peak of this GPU: cuBLAS DGEMM 8192^3, best of 3 (TFLOP/s)."""
    import torch

    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    best = 0.0
    for _ in range(3):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = max(best, 2.0 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


PHASES = ["core", "fock", "commutator", "diis_solve", "pack", "tridiagonalise", "eigenvalues", "eigenvectors",
          "back_transform", "density", "final", "gradient"]
# DRAM bytes (read + write) of one scf_batch_kernel launch per molecule of this workload, from an
# ncu capture of a 256-molecule batch at the plain arm's launch choice (5.88 GB); the per-CTA
# workspaces of 296 resident CTAs exceed L2, so the SCF matrices stream from HBM. Scaled to a
# launch by the molecules it solves.
DRAM_BYTES_PER_MOLECULE = 5.88e9 / 256


def scf_flops(nao, n_occ, iters):
    """Algorithmic FP64 flops of the dense SCF algebra per molecule: per iteration and spin
    tridiagonalisation 4/3 n^3 + back-transformation 2 n^3 + commutator 2 n^3 + density
    2 n^2 n_occ; `iters` counts iterations times spins."""
    n = nao.astype(np.float64)
    return float(np.sum(iters * ((4.0 / 3.0) * n ** 3 + 2.0 * n ** 3 + 2.0 * n ** 3 + 2.0 * n * n * n_occ)))


WATER_GRID = (13, 13, 12)  # first 2000 of 2028 sites, 3.1 A spacing, +-0.2 A jitter
LARGE_PHASES = ["core", "fock", "diis", "tridiagonalise", "eigenvalues", "eigenvectors", "back_transform",
                "orthonormalise", "density"]


def _oracle_water_iters(args):
    """Oracle SCF of the water cluster cut after `max_scf` iterations (timing only)."""
    nw, max_scf = args
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from pm3_rs import workloads

    z, xyz = workloads.water_cluster(nw, grid=WATER_GRID)
    t = time.perf_counter()
    try:
        O.single_point(z, xyz * A2B, max_scf=max_scf, stability=0)
    except Exception:  # stops unconverged by design
        pass
    return time.perf_counter() - t


def water_cpu_baseline(nw, iters):
    """CPU oracle on all host cores (OpenMP pair loops, threaded OpenBLAS): setup + 1 and setup + 2
    iterations at full size, extrapolated linearly to `iters` iterations."""
    import multiprocessing as mp

    cores = os.cpu_count() or 1
    os.environ["OPENBLAS_NUM_THREADS"] = str(cores)
    os.environ["OMP_NUM_THREADS"] = str(cores)
    ctx = mp.get_context("spawn")
    with ctx.Pool(1) as pool:
        t1 = pool.map(_oracle_water_iters, [(nw, 1)])[0]
        t2 = pool.map(_oracle_water_iters, [(nw, 2)])[0]
    per_iter = max(t2 - t1, 0.0)
    setup = max(t1 - per_iter, 0.0)
    return setup + iters * per_iter, cores, setup, per_iter


def water_main(args, rank):
    """One 6000-atom water cluster (the large single-system workload): seconds per converged SCF."""
    nw = args.waters
    if args.impl == "reference":
        if rank != 0:
            return
        from pm3_rs import workloads

        total, cores, setup, per_iter = water_cpu_baseline(nw, 16)
        line = {"impl": "reference", "metric": METRIC, "value": total, "unit": "s/SCF", "n_gpus": args.gpus,
                "steps": 1, "warmup": 0, "ms_per_step": 1e3 * total, "higher_is_better": False, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": "water-2000: 2000 H2O (6000 atoms, 12000 basis functions), RHF PM3 FP64",
                           "extrapolated": f"setup {setup:.1f} s + 16 x {per_iter:.1f} s per iteration"},
                "cpu_baseline": {"value": total, "unit": "s/SCF", "cores": cores, "kind": "port",
                                 "sample": "setup + 1 and + 2 iterations at full size, extrapolated to 16"},
                "e2e": {"value": total, "unit": "s/SCF", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return
    import ctypes

    import torch

    from pm3_rs import _lib, native, workloads

    if rank != 0:  # one system: replicas only; other ranks idle
        return
    os.environ["PM3GPU_PROFILE"] = "0"
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    z, xyz = workloads.water_cluster(nw, grid=WATER_GRID)
    xyz = np.ascontiguousarray(xyz * A2B)
    n_atoms = len(z)
    offs = np.array([0, n_atoms], dtype=np.int32)
    z = np.ascontiguousarray(z, dtype=np.int32)
    ctx = _lib.Context(0)
    lib = ctx.lib
    stream = torch.cuda.current_stream(dev)
    lib.pm3gpu_set_stream(ctx.ptr, ctypes.c_void_p(stream.cuda_stream))
    opts = native.options()
    mixed = args.precision == "mixed"
    mode = _lib.PRECISION_MIXED if mixed else _lib.PRECISION_FP64
    if lib.pm3gpu_set_precision(ctx.ptr, mode) != 0:
        raise RuntimeError(ctx.last_error())
    res = (_lib.Result * 1)()
    q = np.zeros(n_atoms)
    d_z, d_xyz = torch.from_numpy(z).to(dev), torch.from_numpy(xyz).to(dev)
    pz, pxyz = torch.from_numpy(z).pin_memory(), torch.from_numpy(xyz).pin_memory()
    pq = torch.zeros(n_atoms, dtype=torch.float64).pin_memory()
    I32, D = ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_double)

    def run_device():
        rc = lib.pm3gpu_batch_device_inputs(ctx.ptr, 1, None, ctypes.c_void_p(d_z.data_ptr()),
                                            ctypes.c_void_p(d_xyz.data_ptr()), offs.ctypes.data_as(I32),
                                            z.ctypes.data_as(I32), ctypes.byref(opts), res, q.ctypes.data_as(D), None)
        if rc != 0 or res[0].status != 0:
            raise RuntimeError(ctx.last_error())

    def run_host():
        rc = lib.pm3gpu_batch(ctx.ptr, 1, offs.ctypes.data_as(I32), ctypes.cast(pz.data_ptr(), I32),
                              ctypes.cast(pxyz.data_ptr(), D), ctypes.byref(opts), 0, res,
                              ctypes.cast(pq.data_ptr(), D), None)
        if rc != 0 or res[0].status != 0:
            raise RuntimeError(ctx.last_error())

    def timed(fn, steps):
        out = []
        for _ in range(steps):
            torch.cuda.synchronize(dev)
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            fn()
            e.record(stream)
            torch.cuda.synchronize(dev)
            out.append(s.elapsed_time(e))
        return out

    for _ in range(args.warmup):
        run_device()
    with ClockSampler(gpu_uuid(0)) as clk:
        ms = timed(run_device, args.steps)
    clocks = clk.summary()
    launches = lib.pm3gpu_last_kernel_launches(ctx.ptr)
    iters, hof = res[0].iterations, res[0].heat_of_formation_kcal
    nrow = lib.pm3gpu_last_large_trace(ctx.ptr, None, 0)
    trace = np.zeros((max(nrow, 1), 5))
    lib.pm3gpu_last_large_trace(ctx.ptr, trace.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), nrow)
    trace = trace[:nrow]
    hb, db = ctypes.c_longlong(), ctypes.c_longlong()
    e_ms = timed(run_host, 1)
    lib.pm3gpu_last_transfer_bytes(ctx.ptr, ctypes.byref(hb), ctypes.byref(db))
    # phase breakdown from a separate profiled solve (every phase then waits for the stream)
    os.environ["PM3GPU_PROFILE"] = "1"
    pctx = _lib.Context(0)
    pctx.lib.pm3gpu_set_stream(pctx.ptr, ctypes.c_void_p(stream.cuda_stream))
    pctx.lib.pm3gpu_set_precision(pctx.ptr, mode)
    rc = pctx.lib.pm3gpu_batch_device_inputs(pctx.ptr, 1, None, ctypes.c_void_p(d_z.data_ptr()),
                                             ctypes.c_void_p(d_xyz.data_ptr()), offs.ctypes.data_as(I32),
                                             z.ctypes.data_as(I32), ctypes.byref(opts), res, q.ctypes.data_as(D),
                                             None)
    ph = (ctypes.c_double * 16)()
    k = pctx.lib.pm3gpu_last_large_phase_ms(pctx.ptr, ph, 16)
    phases = {LARGE_PHASES[i]: round(ph[i], 1) for i in range(min(k, len(LARGE_PHASES)))}
    n = 6 * nw
    # dominant phase: the Householder reduction, HBM-bound on its panel GEMVs, which must read the
    # lower triangle of the trailing matrix once per column: sum_i (n-i)^2 / 2 * 8 bytes = 4 n^3 / 3
    tri_bytes = 4.0 * n ** 3 / 3.0
    tri_ms = phases.get("tridiagonalise", 0.0) / max(res[0].iterations, 1)
    peak = None
    try:
        peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]
        peak_src = "MEASURED_PEAKS.json hbm_gbs (of measured)"
    except Exception:
        peak, peak_src = 6650.0, "fallback 6.65 TB/s"
    achieved = tri_bytes / (tri_ms * 1e-3) / 1e9 if tri_ms > 0 else None
    value = statistics.median(ms) * 1e-3
    accuracy = None
    if mixed:  # the mixed result against an FP64 solve of the same cluster, gradients included
        gctx = _lib.Context(0)
        gctx.lib.pm3gpu_set_stream(gctx.ptr, ctypes.c_void_p(stream.cuda_stream))
        out = {}
        for name, m in (("fp64", _lib.PRECISION_FP64), ("mixed", _lib.PRECISION_MIXED)):
            gctx.lib.pm3gpu_set_precision(gctx.ptr, m)
            r, g = _lib.Result(), np.zeros(3 * n_atoms)
            rc = gctx.lib.pm3gpu_gradient(gctx.ptr, n_atoms, z.ctypes.data_as(I32), xyz.ctypes.data_as(D),
                                          ctypes.byref(opts), ctypes.byref(r), q.ctypes.data_as(D),
                                          g.ctypes.data_as(D))
            if rc != 0:
                raise RuntimeError(gctx.last_error())
            out[name] = (r.heat_of_formation_kcal, r.iterations, g * (23.060547830619 * 1.8897261246))  # eV/Bohr -> kcal/mol/A
        accuracy = {"fp64_heat_of_formation_kcal": out["fp64"][0], "fp64_iterations": out["fp64"][1],
                    "delta_hof_kcal": out["mixed"][0] - out["fp64"][0],
                    "max_gradient_error_kcal_per_A": float(np.abs(out["mixed"][2] - out["fp64"][2]).max()),
                    "split_bf16_iterations": int(trace[:, 4].sum()), "fp64_closing_iterations": int(nrow - trace[:, 4].sum())}
    line = {
        "metric": METRIC, "value": value, "unit": "s/SCF", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": statistics.median(ms), "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16x3/f32 + f64" if mixed else "f64", "data": "synthetic",
        "config": {"workload": f"water-{nw}: {nw} H2O ({3 * nw} atoms, {6 * nw} basis functions), RHF PM3 "
                               + ("mixed (split-BF16 density and commutator, FP64 closing iterations)" if mixed
                                  else "FP64") + ", reference default options",
                   "iterations": iters, "heat_of_formation_kcal": hof,
                   "rms_density_change": [float(f"{v:.3g}") for v in trace[:, 2]],
                   "l2": "inputs and matrices (1.15 GB each) far exceed L2", "parallelism": "replicas only"},
        "e2e": {"value": e_ms[0] * 1e-3, "unit": "s/SCF", "h2d_bytes_per_step": hb.value, "d2h_bytes_per_step": db.value},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved and peak else None, "traffic": None,
                     "kernel": "Householder reduction (symv_tiles_kernel + panel kernels + DGEMM trailing updates)",
                     "peak_source": peak_src, "bytes_per_tridiagonalisation": tri_bytes,
                     "ms_per_tridiagonalisation": tri_ms},
        "phases_ms": phases,
        "clocks": clocks,
    }
    if accuracy:
        line["accuracy_vs_fp64"] = accuracy
    if not args.no_cpu_baseline:
        total, cores, setup, per_iter = water_cpu_baseline(nw, iters)
        line["cpu_baseline"] = {"value": total, "unit": "s/SCF", "cores": cores, "kind": "port",
                                "sample": f"setup + 1 and + 2 iterations at full size ({setup:.1f} s setup, "
                                          f"{per_iter:.1f} s per iteration), extrapolated to {iters} iterations"}
    print(json.dumps(line))


def _oracle_water_first_iteration(args):
    """Oracle SCF of the water cluster cut after one iteration: its time, and the comparison with
    the GPU's state after one iteration from the same SAD start (density loaded from `path`)."""
    nw, path, gpu_e, gpu_dp = args
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from pm3_rs import workloads

    z, xyz = workloads.water_cluster(nw, grid=WATER_GRID)
    t = time.perf_counter()
    ref = O.cut_short(z, xyz * A2B, 1)
    t = time.perf_counter() - t
    gpu = np.load(path, mmap_mode="r")
    dmax, fro_g, fro_r = 0.0, 0.0, 0.0
    for r0 in range(0, gpu.shape[0], 1000):  # in row blocks: two 1.15 GB matrices
        g, o = np.asarray(gpu[r0:r0 + 1000]), ref["density"][r0:r0 + 1000]
        dmax = max(dmax, float(np.abs(g - o).max()))
        fro_g += float((g * g).sum())
        fro_r += float((o * o).sum())
    return {"seconds": t, "electronic_ev_oracle": ref["electronic_ev"], "electronic_ev_gpu": gpu_e,
            "abs_delta_electronic_ev": abs(gpu_e - ref["electronic_ev"]),
            "rms_density_change_oracle": ref["last_change"], "rms_density_change_gpu": gpu_dp,
            "max_abs_delta_density": dmax, "frobenius_density_gpu": fro_g ** 0.5, "frobenius_density_oracle": fro_r ** 0.5}


def large_record(args, dev, stream):
    """The 6000-atom half of the metric: one 2000-water cluster (12000 basis functions) on the
    whole-GPU path, FP64 and mixed (split-BF16 tcgen05 products, FP64 closing iterations) seconds per
    SCF, the mixed result's heat-of-formation and gradient error against FP64, parity of the first
    iteration against the CPU oracle at full size, and the CPU oracle's time (setup + 1 and + 2
    iterations at full size, extrapolated; it runs on the host cores while the GPU solves)."""
    import ctypes
    import multiprocessing as mp

    import torch

    from pm3_rs import _lib, native, workloads

    nw = 2000
    z, xyz = workloads.water_cluster(nw, grid=WATER_GRID)
    z = np.ascontiguousarray(z, np.int32)
    x = np.ascontiguousarray(xyz * A2B)
    n_atoms, n = len(z), 6 * nw
    I32, D = ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_double)
    ctx = _lib.Context(0)
    lib = ctx.lib
    lib.pm3gpu_set_stream(ctx.ptr, ctypes.c_void_p(stream.cuda_stream))
    # warm-up and full-size parity: one SCF iteration from the SAD start, with the eigensolver checks
    lib.pm3gpu_set_large_checks(ctx.ptr, 1)
    r1 = _lib.Result()
    q = np.zeros(n_atoms)
    dens = np.zeros((n, n))
    o1 = native.options(max_scf=1, stability=0)
    rc = lib.pm3gpu_single_point(ctx.ptr, n_atoms, z.ctypes.data_as(I32), x.ctypes.data_as(D), ctypes.byref(o1),
                                 ctypes.byref(r1), q.ctypes.data_as(D), dens.ctypes.data_as(D), None)
    if rc != _lib.SCF_NOT_CONVERGED:
        raise RuntimeError(ctx.last_error())
    chk = np.zeros((8, 6))
    nchk = lib.pm3gpu_last_large_checks(ctx.ptr, chk.ctypes.data_as(D), 8)
    lib.pm3gpu_set_large_checks(ctx.ptr, 0)
    tmp = tempfile.mkdtemp(prefix="pm3gpu_water_")
    dpath = os.path.join(tmp, "gpu_iteration1.npy")
    np.save(dpath, dens)
    del dens
    # CPU legs on the host cores (two kept free for the GPU's host thread) while the GPU solves
    cores = os.cpu_count() or 1
    threads = max(1, cores - 2)
    os.environ["OPENBLAS_NUM_THREADS"] = str(threads)
    os.environ["OMP_NUM_THREADS"] = str(threads)
    pool = mp.get_context("spawn").Pool(1)
    first = pool.apply_async(_oracle_water_first_iteration, ((nw, dpath, r1.electronic_ev, r1.last_change),))
    second = pool.apply_async(_oracle_water_iters, ((nw, 2),))
    out = {}
    for name, mode in (("fp64", _lib.PRECISION_FP64), ("mixed", _lib.PRECISION_MIXED)):
        lib.pm3gpu_set_precision(ctx.ptr, mode)
        r, g = _lib.Result(), np.zeros(3 * n_atoms)
        torch.cuda.synchronize(dev)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        rc = lib.pm3gpu_gradient(ctx.ptr, n_atoms, z.ctypes.data_as(I32), x.ctypes.data_as(D),
                                 ctypes.byref(native.options()), ctypes.byref(r), q.ctypes.data_as(D),
                                 g.ctypes.data_as(D))
        e.record(stream)
        torch.cuda.synchronize(dev)
        if rc != 0:
            raise RuntimeError(ctx.last_error())
        t = (ctypes.c_double * 8)()
        lib.pm3gpu_last_timings(ctx.ptr, t, 8)
        nrow = lib.pm3gpu_last_large_trace(ctx.ptr, None, 0)
        tr = np.zeros((max(nrow, 1), 5))
        lib.pm3gpu_last_large_trace(ctx.ptr, tr.ctypes.data_as(D), nrow)
        out[name] = {"s_per_scf": t[3] * 1e-3, "e2e_s_per_call": s.elapsed_time(e) * 1e-3,
                     "iterations": r.iterations, "split_bf16_iterations": int(tr[:nrow, 4].sum()),
                     "heat_of_formation_kcal": r.heat_of_formation_kcal,
                     "gradient_kcal_per_A": g * (23.06054783061903 / 0.529177210903)}
    lib.pm3gpu_set_precision(ctx.ptr, _lib.PRECISION_FP64)
    ctx.close()
    par = first.get()
    t2 = second.get()
    pool.close()
    pool.join()
    os.unlink(dpath)
    os.rmdir(tmp)
    fp, mx = out["fp64"], out["mixed"]
    per_iter = max(t2 - par["seconds"], 0.0)
    setup = max(par["seconds"] - per_iter, 0.0)
    cpu_total = setup + fp["iterations"] * per_iter
    return {
        "workload": "water-2000: 2000 H2O (6000 atoms, 12000 basis functions), RHF PM3, reference default options",
        "fp64": {k: v for k, v in fp.items() if k != "gradient_kcal_per_A"},
        "mixed": {k: v for k, v in mx.items() if k != "gradient_kcal_per_A"},
        "s_per_scf_unit_note": "SCF passes on the device (CUDA events), without the gradient; e2e_s_per_call is the "
                               "whole pm3gpu_gradient call from host buffers (copies, SCF, gradient)",
        "mixed_vs_fp64": {"delta_hof_kcal": mx["heat_of_formation_kcal"] - fp["heat_of_formation_kcal"],
                          "max_gradient_component_error_kcal_per_A": float(np.abs(mx["gradient_kcal_per_A"] -
                                                                                  fp["gradient_kcal_per_A"]).max()),
                          "tuned_over_plain_s_per_scf": fp["s_per_scf"] / mx["s_per_scf"] if mx["s_per_scf"] else None},
        "first_iteration_vs_oracle": {k: v for k, v in par.items() if k != "seconds"},
        "eigensolver_checks_first_iteration": {"orthonormality_defect": float(chk[0, 3]) if nchk else None,
                                               "max_abs_F_C_minus_C_eps_ev": float(chk[0, 4]) if nchk else None,
                                               "newton_schulz_steps": int(chk[0, 5]) if nchk else None},
        "cpu_baseline": {"value": cpu_total, "unit": "s/SCF", "cores": threads, "kind": "port",
                         "sample": f"setup + 1 and + 2 iterations at full size ({setup:.1f} s setup, {per_iter:.1f} s per "
                                   f"iteration), extrapolated to the FP64 run's {fp['iterations']} iterations"},
        "gpu_over_cpu_fp64": cpu_total / fp["s_per_scf"] if fp["s_per_scf"] else None,
    }


def tuned_arm(args, lib, ctx0, make_slots, measure, plain_opts, gpu_opts, plain, n_mol):
    """The tuned form of the same workload, timed exactly like the plain arm: the launch choice from
    the autotuner (calibrated on another sample of the generator), the learned initial density trained
    before timing on the plain SCF's own converged densities of other molecules of the generator, and
    mixed precision where the path has it. Reports its rate, the ratio to the plain arm, how far its
    heats of formation are from the plain ones (same molecules), and the plain single-molecule rate
    (pm3gpu_single_point one molecule at a time) for context."""
    import ctypes

    import torch

    from pm3_rs import _lib, native, workloads

    I32, D, F32 = ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_float)

    def packed(ms):
        o, zz, xx = workloads.pack(ms)
        return np.ascontiguousarray(o, np.int32), np.ascontiguousarray(zz, np.int32), np.ascontiguousarray(xx)

    t0 = time.perf_counter()
    rad = args.workload == "radicals-2048"
    c_off, c_z, c_xyz = packed(molecules(256 if rad else 1024, seed=777, workload=args.workload))
    path = os.path.join(tempfile.mkdtemp(prefix="pm3gpu_tuning_"), f"tuning_{args.workload}.json")
    # the arms run batches in flight: tune for the rate of the bulk of a batch
    if lib.pm3gpu_set_tuning_goal(ctx0.ptr, _lib.TUNE_THROUGHPUT if args.inflight > 1 else _lib.TUNE_BATCH_TIME) != 0:
        raise RuntimeError(ctx0.last_error())
    if lib.pm3gpu_autotune(ctx0.ptr, len(c_off) - 1, c_off.ctypes.data_as(I32), c_z.ctypes.data_as(I32),
                           c_xyz.ctypes.data_as(D), ctypes.byref(plain_opts), path.encode()) != 0:
        raise RuntimeError(ctx0.last_error())
    tuning = json.load(open(path))
    n_train = max(64, args.tuned_train // (4 if rad else 1))
    t_off, t_z, t_xyz = packed(molecules(n_train, seed=9001, workload=args.workload))
    epochs = 6
    losses = np.zeros(epochs, np.float32)
    tctx = _lib.Context(0)
    if lib.pm3gpu_guess_train(tctx.ptr, len(t_off) - 1, t_off.ctypes.data_as(I32), t_z.ctypes.data_as(I32),
                              t_xyz.ctypes.data_as(D), ctypes.byref(plain_opts), epochs, 4096, 1e-3, 7,
                              losses.ctypes.data_as(F32)) != 0:
        raise RuntimeError(tctx.last_error())
    params = np.zeros(_lib.GUESS_PARAMS, np.float32)
    if lib.pm3gpu_guess_get_params(tctx.ptr, params.ctypes.data_as(F32), _lib.GUESS_PARAMS) != 0:
        raise RuntimeError(tctx.last_error())
    tctx.close()
    setup_s = time.perf_counter() - t0

    def setup(c):
        if lib.pm3gpu_load_tuning(c.ptr, path.encode()) != 0 or \
                lib.pm3gpu_guess_set_params(c.ptr, params.ctypes.data_as(F32), _lib.GUESS_PARAMS) != 0 or \
                lib.pm3gpu_set_precision(c.ptr, _lib.PRECISION_MIXED) != 0:
            raise RuntimeError(c.last_error())

    slots = make_slots(args.inflight, setup)
    o = native.options(**gpu_opts)
    o.guess = _lib.GUESS_LEARNED
    r = measure(slots, o)
    for sl in slots:
        sl["ctx"].close()
    both = (plain["status"] == 0) & (r["status"] == 0)
    dhf = np.abs(r["hof"][both] - plain["hof"][both])
    value = r["conv"] / (r["t_dev"] * 1e-3)
    plain_value = plain["conv"] / (plain["t_dev"] * 1e-3)
    # the plain path one molecule at a time (the drop-in run_pm3 call), on the first molecules
    single_n = 128
    sc = _lib.Context(0)
    res, q = _lib.Result(), np.zeros(512)
    conv1 = 0
    mols1 = molecules(args.n_mol, seed=1234, workload=args.workload, only=range(single_n))
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    for zz, xx in mols1:
        zz = np.ascontiguousarray(zz, np.int32)
        xx = np.ascontiguousarray(xx)
        rc = lib.pm3gpu_single_point(sc.ptr, len(zz), zz.ctypes.data_as(I32), xx.ctypes.data_as(D),
                                     ctypes.byref(plain_opts), ctypes.byref(res), q.ctypes.data_as(D), None, None)
        conv1 += int(rc == 0)
    single_rate = conv1 / (time.perf_counter() - t1)
    sc.close()
    return {
        "value": value, "unit": "SCF/s", "e2e": r["e_conv"] / (r["t_host"] * 1e-3),
        "tuned_over_plain": value / plain_value,
        "e2e_tuned_over_plain": (r["e_conv"] / r["t_host"]) / (plain["e_conv"] / plain["t_host"]),
        "max_abs_dhf_kcal_vs_plain": float(dhf.max()) if dhf.size else None,
        "molecules_dhf_above_0.01_kcal": int((dhf > 0.01).sum()),
        "converged_fraction": r["conv"] / (n_mol * args.steps),
        "modes": {"launch": "autotuned (calibration sample: 1024 other molecules of the generator; goal: "
                            + ("throughput, batches in flight)" if args.inflight > 1 else "batch time)"),
                  "guess": f"learned, trained before timing on {len(t_off) - 1} other molecules ({epochs} epochs)",
                  "precision": "mixed (split-BF16 tcgen05 products where the path has them, FP64 closing iterations)"},
        "setup_seconds": setup_s, "train_loss_per_epoch": [float(v) for v in losses], "tuning": tuning.get("batch"),
        "gpu_launches": r["launches"], "clocks": r["clocks"],
        "plain_single_molecule_scf_per_s": single_rate,
        "single_molecule_sample": f"first {single_n} molecules through pm3gpu_single_point one at a time (wall clock)",
        "tuned_over_plain_single_molecule": value / single_rate if single_rate else None,
    }


def basis_size(zs):
    return int(sum(1 if int(v) == 1 else 4 for v in zs))


def guess_main(args, rank):
    """Learned initial density: train on seeded organics (5-60 atoms), then solve held-out organics
    (20-90 atoms, basis within one CTA) from the learned start and from SAD; SCF iterations, time to
    converged results, and how far the learned-start heats of formation are from the SAD ones."""
    import ctypes

    import torch

    from pm3_rs import _lib, native, workloads

    if rank != 0:
        return
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    ctx = _lib.Context(0)
    lib = ctx.lib
    stream = torch.cuda.current_stream(dev)
    lib.pm3gpu_set_stream(ctx.ptr, ctypes.c_void_p(stream.cuda_stream))
    I32, D, F = ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_float)
    train = workloads.organic_batch(args.train, 5, 60, seed=90001)
    offs, z, xyz = workloads.pack(train)
    offs, z, xyz = np.ascontiguousarray(offs), np.ascontiguousarray(z), np.ascontiguousarray(xyz * A2B)
    losses = np.zeros(args.epochs, np.float32)
    opts = native.options()
    t0 = time.perf_counter()
    rc = lib.pm3gpu_guess_train(ctx.ptr, len(train), offs.ctypes.data_as(I32), z.ctypes.data_as(I32),
                                xyz.ctypes.data_as(D), ctypes.byref(opts), args.epochs, 4096, 1e-3, 7,
                                losses.ctypes.data_as(F))
    if rc != 0:
        raise RuntimeError(ctx.last_error())
    train_s = time.perf_counter() - t0
    if args.save_guess:  # the trained parameters, for `--guess-params` of the batched workloads
        params = np.zeros(_lib.GUESS_PARAMS, np.float32)
        if lib.pm3gpu_guess_get_params(ctx.ptr, params.ctypes.data_as(F), _lib.GUESS_PARAMS) != 0:
            raise RuntimeError(ctx.last_error())
        params.tofile(args.save_guess)
    held = [m for m in workloads.organic_batch(args.n_mol or 4096, 20, 90, seed=90002) if basis_size(m[0]) <= 256]
    hoffs, hz, hxyz = workloads.pack(held)
    hoffs, hz, hxyz = np.ascontiguousarray(hoffs), np.ascontiguousarray(hz), np.ascontiguousarray(hxyz * A2B)
    n_mol = len(held)
    res = (_lib.Result * n_mol)()
    q = np.zeros(len(hz))

    def solve(guess):
        o = native.options(guess=guess)
        torch.cuda.synchronize(dev)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        rc = lib.pm3gpu_batch(ctx.ptr, n_mol, hoffs.ctypes.data_as(I32), hz.ctypes.data_as(I32),
                              hxyz.ctypes.data_as(D), ctypes.byref(o), 0, res, q.ctypes.data_as(D), None)
        e.record(stream)
        torch.cuda.synchronize(dev)
        if rc != 0:
            raise RuntimeError(ctx.last_error())
        return (s.elapsed_time(e), np.array([r.iterations for r in res]), np.array([r.status for r in res]),
                np.array([r.heat_of_formation_kcal for r in res]))

    for _ in range(max(args.warmup, 1)):
        solve(1)
        solve(_lib.GUESS_LEARNED)
    sad = [solve(1) for _ in range(max(args.steps, 1))]
    lrn = [solve(_lib.GUESS_LEARNED) for _ in range(max(args.steps, 1))]
    ms_sad = statistics.median([x[0] for x in sad])
    ms_lrn = statistics.median([x[0] for x in lrn])
    it_sad, st_sad, hof_sad = sad[0][1], sad[0][2], sad[0][3]
    it_lrn, st_lrn, hof_lrn = lrn[0][1], lrn[0][2], lrn[0][3]
    both = (st_sad == 0) & (st_lrn == 0)
    dhf = np.abs(hof_lrn[both] - hof_sad[both])
    line = {
        "metric": METRIC, "value": int((st_lrn == 0).sum()) / (ms_lrn * 1e-3), "unit": "SCF/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_lrn, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 SCF, bf16 network", "data": "synthetic",
        "config": {"workload": f"learned-guess: trained on {len(train)} organics (5-60 atoms, seed 90001, "
                               f"{args.epochs} epochs), evaluated on {n_mol} held-out organics (20-90 atoms, "
                               "basis <= 256, seed 90002), RHF PM3 FP64",
                   "train_seconds": train_s, "train_loss_per_epoch": [float(v) for v in losses]},
        "standard_guess": {"scf_per_s": int((st_sad == 0).sum()) / (ms_sad * 1e-3), "ms_per_batch": ms_sad,
                           "mean_iterations": float(it_sad[st_sad == 0].mean())},
        "learned_guess": {"scf_per_s": int((st_lrn == 0).sum()) / (ms_lrn * 1e-3), "ms_per_batch": ms_lrn,
                          "mean_iterations": float(it_lrn[st_lrn == 0].mean()),
                          "converged": int((st_lrn == 0).sum()), "of": n_mol},
        "max_abs_dhf_kcal_vs_standard": float(dhf.max()) if dhf.size else None,
        "molecules_dhf_above_0.01_kcal": int((dhf > 0.01).sum()),
        "time_to_converged_ratio": ms_sad / ms_lrn,
    }
    print(json.dumps(line))


def optimize_main(args, rank, cores):
    """Batched geometry optimisation (pm3gpu_optimize_batch): 256 generated organics of 5-20
    atoms from the generator's geometry (standard bond lengths and angles, not minima), the
    reference's L-BFGS with OptOptions' defaults. A step = one batched optimisation of all of them
    (every round one SCF + gradient launch over the pending geometries); value = converged
    optimisations per second. Inputs and results are host arrays: the call is the public entry,
    so `e2e` is the same measurement. CPU: the restated optimiser over the oracle on a sample."""
    if rank != 0:
        return
    from pm3_rs import native, workloads

    n_mol = args.n_mol or 256
    mols = [(np.asarray(z), np.asarray(xyz) * A2B) for z, xyz in workloads.organic_batch(n_mol, 5, 20, seed=4242)]
    offs, z, xyz = workloads.pack(mols)
    unit = "optimisations/s"
    os.environ["OPENBLAS_NUM_THREADS"] = "1"  # one thread per spawned oracle process
    os.environ["OMP_NUM_THREADS"] = "1"
    if args.impl == "reference":
        sample = mols[:max(cores, 16)]
        import multiprocessing as mp

        with mp.get_context("spawn").Pool(cores) as pool:
            chunks = [sample[i::cores] for i in range(cores)]
            t0 = time.perf_counter()
            n = sum(pool.map(_oracle_opt_worker, chunks))
            el = time.perf_counter() - t0
        v = n / el
        print(json.dumps({"impl": "reference", "metric": "converged geometry optimisations/s (batched)", "value": v,
                          "unit": unit, "n_gpus": args.gpus, "steps": 1, "warmup": 0, "higher_is_better": True,
                          "cpu_baseline": {"value": v, "unit": unit, "cores": cores, "kind": "port",
                                           "sample": f"first {len(sample)} of the {n_mol} molecules"},
                          "e2e": {"value": v, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return
    import torch

    for _ in range(max(args.warmup, 1)):
        native.optimize_batch(offs, z, xyz)
    torch.cuda.synchronize()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        r = native.optimize_batch(offs, z, xyz)
        times.append(time.perf_counter() - t0)
    conv = int(r["converged"].sum())
    t = float(np.median(times))
    value = conv / t
    line = {"metric": "converged geometry optimisations/s (batched)", "value": value, "unit": unit, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"optimize-{n_mol}: generated organics of 5-20 atoms from standard geometry, "
                                   "RHF PM3, reference OptOptions (L-BFGS, gtol 1e-3 eV/Bohr, 200 iterations)",
                       "converged": conv, "mean_iterations": float(np.mean(r["iterations"])),
                       "mean_evaluations": float(np.mean(r["evaluations"])), "timing": "wall clock of the call"},
            "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": None, "d2h_bytes_per_step": None}}
    if not args.no_cpu_baseline:
        sample = mols[:max(cores, 16)]
        import multiprocessing as mp

        with mp.get_context("spawn").Pool(cores) as pool:
            chunks = [sample[i::cores] for i in range(cores)]
            t0 = time.perf_counter()
            n = sum(pool.map(_oracle_opt_worker, chunks))
            el = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": n / el, "unit": unit, "cores": cores, "kind": "port",
                                "sample": f"first {len(sample)} of the {n_mol} molecules, one process per core"}
    print(json.dumps(line))


def hessian_main(args, rank, cores):
    """Batched gradient-difference Hessians (pm3gpu_numerical_hessian_batch, the reference's
    numerical_hessian): 64 generated organics of 5-15 atoms; a step = the Hessians of all of them,
    6N displaced SCF + gradient evaluations per molecule under the reference's tightened SCF, every
    displaced geometry of the step in one batched launch. value = Hessians per second. Inputs and
    results are host arrays through the public entry, so `e2e` is the same measurement. CPU: the
    restated numerical_hessian over the oracle on a sample, one process per core."""
    if rank != 0:
        return
    from pm3_rs import native, workloads

    n_mol = args.n_mol or 64
    mols = [(np.asarray(z), np.asarray(xyz) * A2B) for z, xyz in workloads.organic_batch(n_mol, 5, 15, seed=5151)]
    offs, z, xyz = workloads.pack(mols)
    unit = "Hessians/s"
    metric = "gradient-difference Hessians/s (batched)"
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    os.environ["OMP_NUM_THREADS"] = "1"
    n_grad = int(sum(6 * len(m[0]) for m in mols))

    def cpu(sample):
        import multiprocessing as mp

        with mp.get_context("spawn").Pool(cores) as pool:
            chunks = [sample[i::cores] for i in range(cores)]
            t0 = time.perf_counter()
            n = sum(pool.map(_oracle_hess_worker, chunks))
            return n / (time.perf_counter() - t0)

    sample = mols[:max(cores, 16)]
    if args.impl == "reference":
        v = cpu(sample)
        print(json.dumps({"impl": "reference", "metric": metric, "value": v, "unit": unit, "n_gpus": args.gpus,
                          "steps": 1, "warmup": 0, "higher_is_better": True,
                          "cpu_baseline": {"value": v, "unit": unit, "cores": cores, "kind": "port",
                                           "sample": f"first {len(sample)} of the {n_mol} molecules"},
                          "e2e": {"value": v, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return
    import torch

    for _ in range(max(args.warmup, 1)):
        native.numerical_hessian_batch(offs, z, xyz)
    torch.cuda.synchronize()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        r = native.numerical_hessian_batch(offs, z, xyz)
        times.append(time.perf_counter() - t0)
    ok = int((r["status"] == 0).sum())
    t = float(np.median(times))
    value = ok / t
    line = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"hessian-{n_mol}: generated organics of 5-15 atoms, RHF PM3, central differences "
                                   "of the analytic gradient (step 1e-3 Bohr), SCF tightened to e_tol 1e-12 / "
                                   "p_tol 1e-11", "gradient_evaluations_per_step": n_grad,
                       "timing": "wall clock of the call"},
            "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": None, "d2h_bytes_per_step": None}}
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = {"value": cpu(sample), "unit": unit, "cores": cores, "kind": "port",
                                "sample": f"first {len(sample)} of the {n_mol} molecules, one process per core"}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    # 20 timed steps: with batches in flight the timed region starts and ends drained, and 5 steps
    # leave about a fifth of it in the fill and drain (10.5k against 13.2k SCF/s on organics-4096)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="pm3gpu", choices=["pm3gpu", "reference"])
    ap.add_argument("--n-mol", type=int, default=None, help="molecules per step (default: 4096 organics, 2048 radicals)")
    ap.add_argument("--cpu-sample", type=int, default=1024)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="organics-4096",
                    choices=["organics-4096", "radicals-2048", "water-2000", "learned-guess", "optimize-256",
                             "hessian-64", "d3h4-4096"],
                    help="organics-4096: the batched headline (default); radicals-2048: 2048 doublet radicals "
                         "of 10-80 atoms, UHF + analytic gradients; water-2000: one 6000-atom water cluster "
                         "(12000 basis functions) on the whole-GPU path, seconds per SCF; optimize-256: batched "
                         "L-BFGS; hessian-64: batched gradient-difference Hessians; d3h4-4096: the organics with "
                         "method PM3-D3H4")
    ap.add_argument("--train", type=int, default=20000, help="learned-guess workload: training molecules")
    ap.add_argument("--epochs", type=int, default=6, help="learned-guess workload: training epochs")
    ap.add_argument("--waters", type=int, default=2000,
                    help="water-2000 workload: number of waters (the cluster uses the first sites of a 13 x 13 x 12 grid)")
    ap.add_argument("--inflight", type=int, default=4,
                    help="batched workloads: batches in flight (contexts/streams/host threads); 1 times the batches "
                         "one after another")
    ap.add_argument("--save-guess", default=None,
                    help="learned-guess workload: write the trained parameters (float32) to this file")
    ap.add_argument("--guess-params", default=None,
                    help="batched workloads: start every molecule from the learned density of these parameters "
                         "(float32, as written by --save-guess)")
    ap.add_argument("--no-tuned", dest="tuned", action="store_false",
                    help="batched workloads: skip the tuned arm (autotuned launch choice, learned initial density "
                         "trained before timing, mixed precision where the path has it) reported beside the plain one")
    ap.add_argument("--tuned-train", type=int, default=8192,
                    help="tuned arm: molecules (same generator, another seed) whose converged densities train the "
                         "learned initial density before timing")
    ap.add_argument("--tail-helpers", action="store_true",
                    help="batched workloads: idle CTAs take the beta spin of unaccelerated unrestricted jobs "
                         "(pm3gpu_set_tail_helpers) in every arm")
    ap.add_argument("--no-large", dest="large", action="store_false",
                    help="organics workload: skip the 6000-atom record (2000-water cluster, FP64 and mixed s/SCF, "
                         "first-iteration parity against the CPU oracle, CPU time extrapolated)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="water-2000 workload: FP64 throughout, or split-BF16 density and commutator products "
                         "with FP64 closing iterations (reports the heat-of-formation and gradient error against FP64)")
    ap.add_argument("--phases", action="store_true",
                    help="after the timed steps, run one more (untimed) batch with per-phase SM-cycle counters "
                         "and print the phase shares to stderr")
    args = ap.parse_args()
    if args.phases:
        os.environ["PM3GPU_PROFILE"] = "1"
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    cores = os.cpu_count() or 1

    if args.workload == "water-2000":
        return water_main(args, rank)
    if args.workload == "learned-guess":
        return guess_main(args, rank)
    if args.workload == "optimize-256":
        return optimize_main(args, rank, cores)
    if args.workload == "hessian-64":
        return hessian_main(args, rank, cores)
    desc, oracle_opts, gpu_opts, want_grad, default_n = workload_spec(args)
    if args.n_mol is None:
        args.n_mol = default_n
    if args.impl == "reference":
        if rank != 0:
            return
        mols = molecules(args.n_mol, seed=1234, workload=args.workload, only=range(min(args.cpu_sample, args.n_mol)))
        rates = cpu_throughput(mols, cores, steps=args.steps, warmup=0, opts=oracle_opts)
        n = sum(r[0] for r in rates)
        t = sum(r[1] for r in rates)
        value = n / t
        line = {
            "impl": "reference", "metric": METRIC, "value": value, "unit": "SCF/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / len(rates),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": desc, "molecules_per_step": len(mols), "note": "CPU sample of the workload"},
            "cpu_baseline": {"value": value, "unit": "SCF/s", "cores": cores, "kind": "port",
                             "sample": f"first {len(mols)} of the {args.n_mol} molecules per step, one process per core"},
            "e2e": {"value": value, "unit": "SCF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line))
        return

    import ctypes

    import torch

    from pm3_rs import _lib, native

    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    mols = rank_molecules(args.n_mol, rank, world, workload=args.workload)
    from pm3_rs import workloads

    offs, z, xyz = workloads.pack(mols)
    n_mol, n_atoms = len(mols), len(z)
    I32 = ctypes.POINTER(ctypes.c_int32)
    D = ctypes.POINTER(ctypes.c_double)
    F32 = ctypes.POINTER(ctypes.c_float)
    stream = torch.cuda.current_stream(dev)
    d_z = torch.from_numpy(z).to(dev)
    d_xyz = torch.from_numpy(np.ascontiguousarray(xyz)).to(dev)
    d_off = torch.from_numpy(offs).to(dev)
    h_z = np.ascontiguousarray(z)
    h_off = np.ascontiguousarray(offs)
    pz = torch.from_numpy(z).pin_memory()
    pxyz = torch.from_numpy(np.ascontiguousarray(xyz)).pin_memory()
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    peak = fp64_gemm_peak(dev)
    xfer = [0, 0]
    lib = _lib.load()

    def make_slots(n, setup=None):
        """`n` batches in flight: contexts, each with its own stream, result buffers and host thread
        (ctypes releases the GIL inside the library call)."""
        out = []
        for _ in range(max(1, n)):
            c = _lib.Context(local)
            if args.tail_helpers and lib.pm3gpu_set_tail_helpers(c.ptr, 1) != 0:
                raise RuntimeError(c.last_error())
            if setup:
                setup(c)
            st = torch.cuda.Stream(dev)
            lib.pm3gpu_set_stream(c.ptr, ctypes.c_void_p(st.cuda_stream))
            out.append({"ctx": c, "stream": st, "results": (_lib.Result * n_mol)(), "charges": np.zeros(n_atoms),
                        "grads": np.zeros((n_atoms, 3)) if want_grad else None,
                        "pq": torch.zeros(n_atoms, dtype=torch.float64).pin_memory(),
                        "pgr": torch.zeros(3 * n_atoms, dtype=torch.float64).pin_memory() if want_grad else None})
        return out

    def run_slot(sl, host, o):
        c, res = sl["ctx"], sl["results"]
        if host:
            rc = lib.pm3gpu_batch(c.ptr, n_mol, h_off.ctypes.data_as(I32), ctypes.cast(pz.data_ptr(), I32),
                                  ctypes.cast(pxyz.data_ptr(), D), ctypes.byref(o), 0, res,
                                  ctypes.cast(sl["pq"].data_ptr(), D),
                                  ctypes.cast(sl["pgr"].data_ptr(), D) if want_grad else None)
        else:
            rc = lib.pm3gpu_batch_device_inputs(c.ptr, n_mol, ctypes.c_void_p(d_off.data_ptr()),
                                                ctypes.c_void_p(d_z.data_ptr()), ctypes.c_void_p(d_xyz.data_ptr()),
                                                h_off.ctypes.data_as(I32), h_z.ctypes.data_as(I32), ctypes.byref(o),
                                                res, sl["charges"].ctypes.data_as(D),
                                                sl["grads"].ctypes.data_as(D) if want_grad else None)
        if rc != 0:
            raise RuntimeError(c.last_error())

    def timed_inflight(slots, o, host, steps, stagger=0.0):
        """K steps over the slots (each step one full pass over the batch); slot k submits its first
        batch k * stagger seconds after the timed region opens, then back to back, so that one batch's
        bulk fills the SMs the previous batch's last jobs leave idle. Device time (CUDA events) spans
        all K steps."""
        import threading

        flush.fill_(1.0)
        torch.cuda.synchronize(dev)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        for sl in slots:
            sl["stream"].wait_event(s)
        acc = [[0, 0, 0.0, 0.0] for _ in slots]  # converged, launches, flops, kernel ms
        errs = []

        def worker(k):
            sl = slots[k]
            try:
                if stagger > 0.0:
                    time.sleep(k * stagger)
                for _ in range(k, steps, len(slots)):
                    run_slot(sl, host, o)
                    res = np.ctypeslib.as_array(sl["results"])  # a view: no per-molecule Python work
                    ok = res["status"] == 0
                    acc[k][0] += int(ok.sum())
                    acc[k][1] += lib.pm3gpu_last_kernel_launches(sl["ctx"].ptr)
                    its = res["iterations"][ok] * (1.0 + res["unrestricted"][ok])
                    acc[k][2] += scf_flops(res["nao"][ok], res["n_occ"][ok], its)
                    t = (ctypes.c_double * 8)()
                    lib.pm3gpu_last_timings(sl["ctx"].ptr, t, 8)
                    acc[k][3] += t[5]
                    hb, db = ctypes.c_longlong(), ctypes.c_longlong()
                    lib.pm3gpu_last_transfer_bytes(sl["ctx"].ptr, ctypes.byref(hb), ctypes.byref(db))
                    xfer[0], xfer[1] = hb.value, db.value
            except Exception as ex:  # surfaced after the join
                errs.append(ex)

        threads = [threading.Thread(target=worker, args=(k,)) for k in range(len(slots))]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        if errs:
            raise errs[0]
        for sl in slots:
            ev = torch.cuda.Event()
            ev.record(sl["stream"])
            stream.wait_event(ev)
        e.record(stream)
        torch.cuda.synchronize(dev)
        return (s.elapsed_time(e), sum(a[0] for a in acc), sum(a[1] for a in acc), sum(a[2] for a in acc),
                sum(a[3] for a in acc))

    def measure(slots, o):
        """Warm-up (W steps), then K device-resident steps (clocks sampled) and K host-API steps."""
        timed_inflight(slots, o, False, max(args.warmup, len(slots)))
        t0 = time.perf_counter()
        run_slot(slots[0], False, o)  # one batch alone: the submission interval of the slots
        stagger = (time.perf_counter() - t0) / len(slots) if len(slots) > 1 else 0.0
        if dist:
            dist.barrier()
        torch.cuda.synchronize(dev)
        with ClockSampler(gpu_uuid(local)) as clk:
            t_dev, conv, launches, flops, kern_ms = timed_inflight(slots, o, False, args.steps, stagger)
        clocks = clk.summary()
        hof = np.ctypeslib.as_array(slots[0]["results"])["heat_of_formation_kcal"].copy()
        st = np.ctypeslib.as_array(slots[0]["results"])["status"].copy()
        timed_inflight(slots, o, True, len(slots))
        if dist:
            dist.barrier()
        t_host, e_conv, _, _, _ = timed_inflight(slots, o, True, args.steps, stagger)
        return {"t_dev": t_dev, "conv": conv, "launches": launches, "flops": flops, "kern_ms": kern_ms,
                "t_host": t_host, "e_conv": e_conv, "clocks": clocks, "stagger": stagger, "hof": hof, "status": st,
                "h2d": xfer[0], "d2h": xfer[1]}

    # ------------------------------------------------------------ plain arm: the headline value
    opts = native.options(**gpu_opts)
    guess_params = None
    if args.guess_params:  # learned initial density (the standard-guess pass stays as backup)
        guess_params = np.fromfile(args.guess_params, dtype=np.float32)
        opts.guess = _lib.GUESS_LEARNED

    def plain_setup(c):
        if guess_params is not None and lib.pm3gpu_guess_set_params(
                c.ptr, guess_params.ctypes.data_as(F32), len(guess_params)) != 0:
            raise RuntimeError(c.last_error())

    plain_slots = make_slots(args.inflight, plain_setup)
    plain = measure(plain_slots, opts)

    # ------------------------------------------------------------ tuned arm (one GPU only)
    tuned = None
    if world == 1 and args.tuned:
        tuned = tuned_arm(args, lib, plain_slots[0]["ctx"], make_slots, measure, opts, gpu_opts, plain, n_mol)
    for sl in plain_slots:
        sl["ctx"].close()

    tot, e_tot, conv, e_conv = reduce_over_ranks(plain["t_dev"], plain["t_host"], plain["conv"], plain["e_conv"], dist,
                                                 dev)
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    value = conv / (tot * 1e-3)
    e2e = e_conv / (e_tot * 1e-3)
    kern_ms = plain["t_dev"] if len(plain_slots) > 1 else plain["kern_ms"]
    achieved = plain["flops"] / (kern_ms * 1e-3) / 1e12 if kern_ms > 0 else None
    line = {
        "metric": METRIC, "value": value, "unit": "SCF/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": tot / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": desc, "arm": "plain FP64: reference default options and guess, built-in launch choice",
                   "molecules_per_step_per_gpu": n_mol, "parallelism": f"dp{world}",
                   "sharding": ("one batch of molecules x ranks split by the longest-processing-time rule on atoms^3"
                                if world > 1 else "one GPU"),
                   "l2": "flushed before the timed steps (512 MiB write); per-CTA workspaces (> 126 MB) exceed L2",
                   "batches_in_flight": max(1, args.inflight),
                   "guess": f"learned ({args.guess_params})" if guess_params is not None else "reference default (SAD)",
                   "submission": (f"slot k submits its first batch k x {1e3 * plain['stagger']:.0f} ms into the timed "
                                  "region (one batch time / slots), then back to back")
                   if args.inflight > 1 else "one batch at a time",
                   "converged_fraction": conv / (n_mol * args.steps * world),
                   "tail_helpers": bool(args.tail_helpers)},
        "e2e": {"value": e2e, "unit": "SCF/s", "h2d_bytes_per_step": plain["h2d"], "d2h_bytes_per_step": plain["d2h"]},
        "gpu_launches": plain["launches"],
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": (achieved / peak) if achieved else None,
                     "traffic": DRAM_BYTES_PER_MOLECULE * n_mol,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one scf_batch_kernel launch "
                                       "over 256 molecules of this workload at the same launch choice, scaled by "
                                       "molecules per launch",
                     "kernel": "scf_batch_kernel", "peak_source": "FP64 cuBLAS DGEMM 8192^3 measured in this run",
                     "flops_per_step": plain["flops"] / args.steps, "kernel_ms_per_step": kern_ms / args.steps},
        "clocks": plain["clocks"],
    }
    if tuned:
        line["tuned"] = tuned
    if args.phases:
        os.environ["PM3GPU_PROFILE"] = "1"
        pc = _lib.Context(local)
        lib.pm3gpu_set_stream(pc.ptr, ctypes.c_void_p(stream.cuda_stream))
        sl = {"ctx": pc, "results": (_lib.Result * n_mol)(), "charges": np.zeros(n_atoms),
              "grads": np.zeros((n_atoms, 3)) if want_grad else None}
        run_slot(sl, False, opts)
        cyc = (ctypes.c_double * 16)()
        k = lib.pm3gpu_last_phase_cycles(pc.ptr, cyc, 16)
        tot_c = sum(cyc[i] for i in range(k)) or 1.0
        print(json.dumps({"phase_share": {PHASES[i]: round(cyc[i] / tot_c, 4) for i in range(min(k, len(PHASES)))},
                          "cta_cycles": tot_c}), file=sys.stderr)
        pc.close()
    if world == 1 and not args.no_cpu_baseline:
        sample = mols[: args.cpu_sample]
        r = cpu_throughput(sample, os.cpu_count() or 1, steps=1, opts=oracle_opts)
        line["cpu_baseline"] = {"value": r[0][0] / r[0][1], "unit": "SCF/s", "cores": os.cpu_count(),
                                "kind": "port",
                                "sample": f"first {len(sample)} of the {n_mol} molecules, one oracle process per core"}
    if world == 1 and args.large and args.workload == "organics-4096":
        line["large_6k"] = large_record(args, dev, stream)
    print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
