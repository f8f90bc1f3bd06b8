"""The multi-process bench path on CPU: two gloo ranks (127.0.0.1).

Under torchrun the ranks split ONE batch of molecules (n per rank x ranks) by the
longest-processing-time partition (weak scaling, no data-path collective): every molecule lands on
exactly one rank and the ranks' cost shares are balanced. The whole-job line takes the slowest
rank's device time and the sum of the converged counts. The reference arm runs on rank 0 only; the
other ranks exit without work.
"""
import importlib.util
import os
import socket
import subprocess
import sys

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        bench = _bench()
        from pm3_rs import workloads

        mols = bench.rank_molecules(16, rank, world)
        # the same molecules as the one global batch builds, identified by their coordinates
        full = bench.molecules(16 * world, 1234)
        mine = [next(i for i, (_, fx) in enumerate(full) if np.array_equal(fx, x)) for _, x in mols]
        cost = float(sum(float(len(zz)) ** 3 for zz, _ in mols))
        digests = [None] * world
        dist.all_gather_object(digests, (sorted(mine), cost))
        # rank-dependent device times and counts: the job line takes the max and the sum
        tot, e_tot, conv, e_conv = bench.reduce_over_ranks(100.0 + 10 * rank, 50.0 - rank, 7 + rank, 5 + rank, dist,
                                                           "cpu")
        out.put((rank, digests, tot, e_tot, conv, e_conv))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, digests, tot, e_tot, conv, e_conv in got:
        (a, ca), (b, cb) = digests
        assert sorted(a + b) == list(range(32)) and not set(a) & set(b)  # one batch, split
        assert abs(ca - cb) <= 60.0 ** 3  # within one largest molecule's cost
        assert (tot, e_tot, conv, e_conv) == (110.0, 50.0, 15, 11)


def test_reference_arm_idles_on_other_ranks():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
