"""Spreading one batch of independent molecules over several GPUs (no reference counterpart: pm3-rs
runs one process with rayon over its CPU cores, src/scf.rs:442-448).

Molecules do not interact, so the batch shards by molecules with no data-path collective: each
device solves its part in its own persistent launch and the host gathers the results back into
the caller's order. Parts are balanced by the SCF's cost model, basis size cubed (the dense
eigensolve, commutator and density dominate an iteration), with the longest-processing-time rule:
molecules sorted by cost, largest first, each to the part with the least cost so far.
"""
from __future__ import annotations

import heapq
import threading

import numpy as np

from . import _lib


def basis_sizes(offsets, z) -> np.ndarray:
    """Basis functions of every molecule: 1 per hydrogen (and helium), 4 per other s/p element."""
    z = np.asarray(z)
    per_atom = np.where(z <= 2, 1, 4)
    csum = np.concatenate([[0], np.cumsum(per_atom)])
    offsets = np.asarray(offsets)
    return csum[offsets[1:]] - csum[offsets[:-1]]


def partition(offsets, z, n_parts: int):
    """Molecule indices of each of `n_parts` parts (each ascending), balancing sum(nao^3)."""
    return partition_costs(basis_sizes(offsets, z).astype(np.float64) ** 3, n_parts)


def partition_costs(cost, n_parts: int):
    """The longest-processing-time partition of molecules with the given costs."""
    if n_parts < 1:
        raise ValueError("n_parts must be >= 1")
    cost = np.asarray(cost, dtype=np.float64)
    order = np.argsort(-cost, kind="stable")
    heap = [(0.0, p) for p in range(n_parts)]
    parts = [[] for _ in range(n_parts)]
    for m in order:
        load, p = heapq.heappop(heap)
        parts[p].append(int(m))
        heapq.heappush(heap, (load + cost[m], p))
    return [np.array(sorted(p), dtype=np.int64) for p in parts]


def part_loads(offsets, z, parts):
    """sum(nao^3) of every part."""
    cost = basis_sizes(offsets, z).astype(np.float64) ** 3
    return np.array([cost[p].sum() for p in parts])


def gather_part(offsets, z, xyz, idx):
    """(offsets, z, xyz) of the molecules `idx` of a batch, in that order, and each molecule's atom
    range in the full batch."""
    offsets = np.asarray(offsets)
    lo, hi = offsets[idx], offsets[idx + 1]
    atoms = np.concatenate([np.arange(a, b) for a, b in zip(lo, hi)]) if len(idx) else np.zeros(0, np.int64)
    sub_off = np.zeros(len(idx) + 1, dtype=np.int32)
    sub_off[1:] = np.cumsum(hi - lo)
    return sub_off, np.ascontiguousarray(np.asarray(z)[atoms], np.int32), \
        np.ascontiguousarray(np.asarray(xyz).reshape(-1, 3)[atoms]), atoms


def batch_on_devices(offsets, z, xyz_bohr, opts=None, devices=(0,), want_gradient=False, contexts=None):
    """pm3gpu_batch over several devices: partition, one host thread and one context per device
    (each its own persistent launch), results gathered in the caller's molecule order. Returns the
    BatchResult of the whole batch and the parts used."""
    from . import native

    devices = list(devices)
    n_mol = len(offsets) - 1
    parts = partition(offsets, z, len(devices))
    ctxs = contexts or [_lib.default_context(d) for d in devices]
    out = [None] * len(devices)
    errs = []

    def work(k):
        try:
            so, sz, sx, atoms = gather_part(offsets, z, xyz_bohr, parts[k])
            out[k] = (native.batch(so, sz, sx, opts, want_gradient=want_gradient, context=ctxs[k]), atoms)
        except Exception as ex:  # surfaced after the join
            errs.append(ex)

    threads = [threading.Thread(target=work, args=(k,)) for k in range(len(devices))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    if errs:
        raise errs[0]
    results = (_lib.Result * max(n_mol, 1))()
    charges = np.zeros(len(z))
    grads = np.zeros((len(z), 3)) if want_gradient else None
    for k, (res, atoms) in enumerate(out):
        for j, m in enumerate(parts[k]):
            results[m] = res.raw[j]
        charges[atoms] = res.charges
        if want_gradient:
            grads[atoms] = res.gradients
    return native.BatchResult(list(results)[:n_mol], charges, grads, np.asarray(offsets)), parts
