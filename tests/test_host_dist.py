"""Host logic of the multi-process paths on CPU (gloo, world size 2): the
gradient average of data-parallel training of the learned smoother (on a toy
quadratic and on the stencil network's own gradient, from the oracle), the
identical updates it leads to on every rank, the max-over-ranks timing of
bench.py, and the subdomains of the domain-decomposed solve.  No GPU."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import dist_workers as W


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_data_parallel_training_and_rank_max(tmp_path):
    world = 2
    mp.start_processes(W.dp_training, args=(world, free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    r = [np.load(os.path.join(tmp_path, f"rank{k}.npz")) for k in range(world)]
    # every rank holds the same weights after training
    assert np.array_equal(r[0]["w"], r[1]["w"])
    # ... equal to one process that applies the mean of the ranks' gradients
    probs = [W.quadratic_problem(k) for k in range(world)]
    w = np.zeros(8, dtype=np.float32)
    losses = []
    for _ in range(25):
        gs, ls = [], []
        for A, y in probs:
            res = A @ w - y
            ls.append(0.5 * float(res @ res))
            gs.append((A.T @ res).astype(np.float32))
        g = np.mean(np.stack(gs), axis=0).astype(np.float32)
        losses.append(np.mean(ls))
        w = (w - 0.01 * g).astype(np.float32)
    assert np.allclose(r[0]["w"], w, rtol=1e-5, atol=1e-6)
    assert np.allclose(r[0]["hist"], losses, rtol=1e-5)
    assert losses[-1] < losses[0]
    assert np.allclose(r[0]["mean"], 1.5) and np.allclose(r[1]["mean"], 1.5)
    assert float(r[0]["mx"]) == 1.5 and float(r[1]["mx"]) == 1.5


@pytest.mark.parametrize("elem,n,nl", [(2, 8, 3), (1, 16, 3), (12, 8, 2)])
def test_subdomains_partition_and_halo(tmp_path, elem, n, nl):
    """Domain decomposition host logic (parmoon_b200.dd, gloo, 2 ranks): the
    owned dofs of the ranks partition the global dofs, the halo exchange fills
    every ghost row with its owner's value, and the pattern of every owned
    active row built from the subdomain's cells equals the global row
    (TSquareStructure3D on the subdomain holds all couplings of its owned
    rows, so its assembly of those rows is complete)."""
    world = 2
    mp.start_processes(W.dd_partition, args=(world, free_port(), str(tmp_path), elem, n, nl), nprocs=world,
                       join=True, start_method="spawn")
    r = [np.load(os.path.join(tmp_path, f"dd{k}.npz")) for k in range(world)]
    owned = np.concatenate([x["glob"][:int(x["n_owned"])] for x in r])
    N = r[0]["ref"].size
    assert np.array_equal(np.sort(owned), np.arange(N))
    for x in r:
        assert np.array_equal(x["x"], x["ref"][x["glob"]])  # ghosts filled from their owners
        assert int(x["bad_rows"]) == 0


def test_data_parallel_stencil_network_gradient(tmp_path):
    """Two ranks, each with its own problem, train the stencil network on the
    averaged gradient: both end with the same weights, equal to one process
    that applies the mean of the two ranks' gradients."""
    from oracle import learned_oracle as LO
    from parmoon_b200 import learned as PL
    world = 2
    mp.start_processes(W.dp_learned, args=(world, free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    r = [np.load(os.path.join(tmp_path, f"learned{k}.npz")) for k in range(world)]
    assert np.array_equal(r[0]["w"], r[1]["w"])
    probs = [W.learned_problem(100 + k) for k in range(world)]
    w = PL.init_weights(0).astype(np.float32)
    for _ in range(3):
        gs = []
        for m, rp, kc, A, e, rr in probs:
            _, g = LO.loss_and_grad(LO.bf16_round(w), 4, rp, kc, A, m["active_bound"], m["dof_lat"], e, rr)
            gs.append(g.astype(np.float32))
        w = (w - 0.05 * np.mean(np.stack(gs), axis=0).astype(np.float32)).astype(np.float32)
    assert np.allclose(r[0]["w"], w, rtol=1e-5, atol=1e-7)
