"""Small, self-contained cases of single kernels, sized for an ncu capture (a few GB on the device).

    python pm3-rs_b200/profile_cases.py split-gemm [--n 4096] [--reps 1]
        the tcgen05 split-BF16 product C = A B^T of random n x n FP64 operands (pm3gpu_split_gemm)
    python pm3-rs_b200/profile_cases.py water [--waters 1000] [--iters 2]
        one whole-GPU solve of a water cluster cut after `iters` SCF iterations: one launch of
        core_pairs_kernel (pair integrals, H_core, pair table) and a few of fock_pairs_kernel
    python pm3-rs_b200/profile_cases.py dgemm [--n 4096] [--reps 1]
        the FP64 DMMA GEMM C = A B (n x n, column-major) of the whole-GPU path (pm3gpu_dgemm)
    python pm3-rs_b200/profile_cases.py mlp [--mols 512]
        learned-guess inference on `mols` organics with a random model (pm3gpu_guess_predict):
        three launches of the tcgen05 layer kernel over all atom and pair rows
    python pm3-rs_b200/profile_cases.py corrections [--mols 4096] [--reps 1]
        the PM3-D3H4 corrections alone on `mols` organics (pm3gpu_corrections_batch): the D3
        coordination-number, pair, chain and sum kernels, then the H4 / H-H kernel, per repetition

Each case prints what it ran and exits 0 on success. The profiles/ summaries name the exact command.
"""
import argparse
import ctypes
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from pm3_rs import _lib, native, workloads  # noqa: E402

A2B = 1.0 / 0.529177210903
D = ctypes.POINTER(ctypes.c_double)


def split_gemm(n, reps):
    ctx = _lib.Context(0)
    rng = np.random.default_rng(0)
    a, b = rng.standard_normal((n, n)), rng.standard_normal((n, n))
    out = np.zeros((n, n), np.float32)
    for _ in range(reps):
        t = time.perf_counter()
        rc = ctx.lib.pm3gpu_split_gemm(ctx.ptr, n, n, n, a.ctypes.data_as(D), n, b.ctypes.data_as(D), n,
                                       out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
        if rc != 0:
            raise RuntimeError(ctx.last_error())
        print(f"split-gemm n={n}: {1e3 * (time.perf_counter() - t):.1f} ms per call (host copies included)")
    ref = a[:128] @ b.T
    print(f"relative error of the first 128 rows: {np.abs(out[:128] - ref).max() / np.abs(ref).max():.2e}")


def water(waters, iters):
    side = int(np.ceil(waters ** (1.0 / 3.0)))
    z, xyz = workloads.water_cluster(waters, grid=(side, side, side))
    z = np.ascontiguousarray(z, np.int32)
    x = np.ascontiguousarray(xyz * A2B)
    ctx = _lib.Context(0)
    res, q = _lib.Result(), np.zeros(len(z))
    o = native.options(max_scf=iters, stability=0)
    rc = ctx.lib.pm3gpu_single_point(ctx.ptr, len(z), z.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                     x.ctypes.data_as(D), ctypes.byref(o), ctypes.byref(res), q.ctypes.data_as(D),
                                     None, None)
    if rc not in (_lib.OK, _lib.SCF_NOT_CONVERGED):  # cut short by design
        raise RuntimeError(ctx.last_error())
    print(f"water-{waters}: n = {res.nao}, {res.iterations} iterations, E_elec {res.electronic_ev:.6f} eV")


def dgemm(n, reps):
    ctx = _lib.Context(0)
    rng = np.random.default_rng(0)
    a, b = np.asfortranarray(rng.standard_normal((n, n))), np.asfortranarray(rng.standard_normal((n, n)))
    c = np.zeros((n, n), order="F")
    for _ in range(reps):
        t = time.perf_counter()
        rc = ctx.lib.pm3gpu_dgemm(ctx.ptr, 0, 0, n, n, n, 1.0, a.ctypes.data_as(D), n, b.ctypes.data_as(D), n, 0.0,
                                  c.ctypes.data_as(D), n)
        if rc != 0:
            raise RuntimeError(ctx.last_error())
        print(f"dgemm n={n}: {1e3 * (time.perf_counter() - t):.1f} ms per call (host copies included)")
    ref = a[:64] @ b
    print(f"max relative error of the first 64 rows: {np.abs(c[:64] - ref).max() / np.abs(ref).max():.2e}")


def mlp(mols):
    ctx = _lib.Context(0)
    rng = np.random.default_rng(3)
    n_par = 64 * 256 + 256 + 2 * (256 * 256 + 256) + 256 * 8 + 8
    params = (rng.standard_normal(n_par) * 0.05).astype(np.float32)
    F32 = ctypes.POINTER(ctypes.c_float)
    if ctx.lib.pm3gpu_guess_set_params(ctx.ptr, params.ctypes.data_as(F32), n_par) != 0:
        raise RuntimeError(ctx.last_error())
    offs, z, xyz = workloads.pack(workloads.organic_batch(mols, 5, 60, seed=5))
    offs = np.ascontiguousarray(offs, np.int32)
    z = np.ascontiguousarray(z, np.int32)
    x = np.ascontiguousarray(xyz * A2B)
    I32 = ctypes.POINTER(ctypes.c_int32)
    t = time.perf_counter()
    rc = ctx.lib.pm3gpu_guess_predict(ctx.ptr, len(offs) - 1, offs.ctypes.data_as(I32), z.ctypes.data_as(I32),
                                      x.ctypes.data_as(D), None, None)
    if rc != 0:
        raise RuntimeError(ctx.last_error())
    print(f"mlp: {mols} molecules in {1e3 * (time.perf_counter() - t):.1f} ms (features, three layer launches)")


def corrections(mols, reps):
    offs, z, xyz = workloads.pack(workloads.organic_batch(mols, 5, 60, seed=1234))
    x = xyz * A2B
    t = time.perf_counter()
    for _ in range(reps):
        r = native.corrections_batch(offs, z, x, "pm3-d3h4")
    ms = 1e3 * (time.perf_counter() - t) / reps
    print(f"corrections: {mols} molecules, {len(z)} atoms, PM3-D3H4 in {ms:.2f} ms per call (host copies included); "
          f"mean D3 {r['d3_ev'].mean():.4f} eV, H4 {r['h4_ev'].mean():.4f} eV")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["split-gemm", "water", "dgemm", "mlp", "corrections"])
    ap.add_argument("--n", type=int, default=4096)
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--waters", type=int, default=1000)
    ap.add_argument("--iters", type=int, default=2)
    ap.add_argument("--mols", type=int, default=512)
    a = ap.parse_args()
    if a.case == "split-gemm":
        split_gemm(a.n, a.reps)
    elif a.case == "dgemm":
        dgemm(a.n, a.reps)
    elif a.case == "mlp":
        mlp(a.mols)
    elif a.case == "corrections":
        corrections(a.mols, a.reps)
    else:
        water(a.waters, a.iters)


if __name__ == "__main__":
    main()
