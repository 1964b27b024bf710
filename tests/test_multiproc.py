"""The N > 1 path of bench.py (replicas: every rank solves its own system, no
collective on the data path, job time = max over ranks), run as world-size-2
gloo ranks on CPU with the oracle standing in for the GPU solve."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, outdir):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import time
    from datetime import timedelta

    import torch.distributed as dist

    import bench
    from oracle import oracle as O
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    bench.set_size(10)
    A, b, xs = bench.make_problem(seed=bench.replica_seed(rank))
    r, i, v = A.arrays()
    M = O.Mat.from_csr(r, i, v)
    Z, W = O.sdainv(M)
    t0 = time.perf_counter()
    res = O.f3r_solve(M, W, Z, b, O.params(tol=1e-10, c=8))
    mine = time.perf_counter() - t0 + 0.05 * rank   # make the ranks' times differ
    tmax = bench.max_over_ranks(mine, world)
    np.savez(os.path.join(outdir, f"r{rank}.npz"), b=b, x=res["x"], xs=xs, solved=res["solved"], mine=mine,
             tmax=tmax)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_replicas(tmp_path):
    world = 2
    mp.start_processes(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    r0, r1 = (np.load(tmp_path / f"r{k}.npz") for k in range(world))
    assert bool(r0["solved"]) and bool(r1["solved"])
    assert not np.array_equal(r0["b"], r1["b"])  # different systems per rank
    for r in (r0, r1):
        assert np.linalg.norm(r["x"] - r["xs"]) / np.linalg.norm(r["xs"]) < 1e-7
    assert float(r0["tmax"]) == float(r1["tmax"]) == max(float(r0["mine"]), float(r1["mine"]))
