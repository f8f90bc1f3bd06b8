"""Small, self-contained cases of single kernels, sized for an ncu capture (a few GB on the device).

    python pm3-rs_b200/profile_cases.py split-gemm [--n 4096] [--reps 1]
        the tcgen05 split-BF16 product C = A B^T of random n x n FP64 operands (pm3gpu_split_gemm)
    python pm3-rs_b200/profile_cases.py water [--waters 1000] [--iters 2]
        one whole-GPU solve of a water cluster cut after `iters` SCF iterations: one launch of
        core_pairs_kernel (pair integrals, H_core, pair table) and a few of fock_pairs_kernel

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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["split-gemm", "water"])
    ap.add_argument("--n", type=int, default=4096)
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--waters", type=int, default=1000)
    ap.add_argument("--iters", type=int, default=2)
    a = ap.parse_args()
    if a.case == "split-gemm":
        split_gemm(a.n, a.reps)
    else:
        water(a.waters, a.iters)


if __name__ == "__main__":
    main()
