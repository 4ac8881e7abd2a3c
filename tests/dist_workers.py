"""Rank bodies of the multi-process tests (gloo on CPU, world size 2)."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def init(rank, world, port):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    return dist


def quadratic_problem(rank):
    """Rank-local least squares 0.5 |A_r w - y_r|^2 (different data per rank)."""
    rng = np.random.default_rng(100 + rank)
    A = rng.standard_normal((20, 8))
    y = rng.standard_normal(20)
    return A, y


def dp_training(rank, world, port, out_dir):
    sys.path.insert(0, ROOT)
    dist = init(rank, world, port)
    from parmoon_b200 import learned as PL
    A, y = quadratic_problem(rank)
    w = {"w": np.zeros(8, dtype=np.float32)}

    def grad_fn(it):
        r = A @ w["w"] - y
        return 0.5 * float(r @ r), (A.T @ r).astype(np.float32)

    def apply_fn(g):
        w["w"] = (w["w"] - 0.01 * g).astype(np.float32)

    hist = PL.train_data_parallel(grad_fn, apply_fn, 25, dist)
    m = PL.allreduce_mean(np.full(3, rank + 1.0, dtype=np.float32), dist)
    import bench
    mx = bench.max_over_ranks(0.5 + rank, dist)
    np.savez(os.path.join(out_dir, f"rank{rank}.npz"), w=w["w"], hist=np.array(hist), mean=m, mx=mx)
    dist.barrier()
    dist.destroy_process_group()
