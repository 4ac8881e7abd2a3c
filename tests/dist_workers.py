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


def dd_partition(rank, world, port, out_dir, elem, n, nl):
    """Subdomain of this rank (parmoon_b200.dd): halo exchange of a global
    vector through gloo, and the owned rows of the subdomain pattern mapped
    back to global numbering."""
    sys.path.insert(0, ROOT)
    dist = init(rank, world, port)
    import parmoon_b200 as P
    from parmoon_b200 import dd
    glob, loc = dd.local_hierarchy(elem, n, nl, world, rank)
    F, G = loc[-1], glob[-1]
    g = np.random.default_rng(3).standard_normal(G["N"])
    x = np.full(F["N"], np.nan)
    x[:F["n_owned"]] = g[F["glob"][:F["n_owned"]]]
    dd.exchange_host(dist, F, x)
    # owned active rows: the subdomain's pattern (host builder on the local cells) against the global one
    nloc = F["elem_dof"].size // F["cells"].size
    rp, kc = P.struct_csr_of(F["elem_dof"], nloc, F["N"], F["active_bound"])
    bad_rows = 0
    for r in range(F["active_bound"]):
        mine = np.sort(F["glob"][kc[rp[r]:rp[r + 1]]])
        gr = F["glob"][r]
        ref = G["kcol"][G["rowptr"][gr]:G["rowptr"][gr + 1]]
        bad_rows += int(not np.array_equal(mine, ref))
    np.savez(os.path.join(out_dir, f"dd{rank}.npz"), x=x, glob=F["glob"], n_owned=F["n_owned"], ref=g,
             bad_rows=bad_rows, owned_all=np.concatenate([L["glob"][:L["n_owned"]] for L in loc[-1:]]))
    dist.barrier()
    dist.destroy_process_group()


def dd_solve(rank, world, port, out_dir, elem, n, nl, prec):
    """One rank of the domain-decomposed solve (pmg_solve_dd) on its subdomain,
    the transport gloo through host copies; every rank runs on the same device
    (the exchange and the sums happen on the host between launches, no kernel
    waits for another rank)."""
    sys.path.insert(0, ROOT)
    dist = init(rank, world, port)
    import parmoon_b200 as P
    from parmoon_b200 import dd
    glob, loc = dd.local_hierarchy(elem, n, nl, world, rank)
    h = P.Handle(nl, P.default_params(precision=prec, lin_red=1e-12, lin_maxit=400))
    h.set_coefficients(P.coeff(kind=P.COEF_CONST, eps=1e-3, b=(1.0, 0.5, 0.25), f=1.0))
    dd.load_subdomain(h, loc, dirichlet=lambda x, y, z: (np.abs(x) < 1e-12).astype(float))
    h.assemble(-1, P.FORM_SUPG, copy_out=False)
    comm = dd.TorchComm(dist, loc[-1])
    c = comm.struct(P.lib())
    h.set_halo(comm.send_idx, comm.recv_idx, comm.send_buf.data_ptr(), comm.recv_buf.data_ptr())
    _, st, rc = h.solve_dd(c, raise_on_error=False)
    x = h.get_solution()
    F = loc[-1]
    no = F["n_owned"]
    np.savez(os.path.join(out_dir, f"dds{rank}.npz"), x=x[:no], glob=F["glob"][:no], rc=rc, its=st.iterations,
             rel=st.rel_res)
    h.close()
    dist.barrier()
    dist.destroy_process_group()
