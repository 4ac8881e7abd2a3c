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


def learned_problem(seed):
    """A 3^3-cell Q1 SUPG problem with a curl-field convection and one (e, r) pair (oracle only)."""
    from oracle import cd3d as O
    m = O.struct_mesh(O.Q1, 3)
    rp, kc = O.csr(m["elem_dof"], 8, m["N"], m["active_bound"])
    rng = np.random.default_rng(seed)
    modes = np.zeros((2, 8))
    modes[:, 0:3] = [[1, 0, 1], [0, 1, 1]]
    modes[:, 3] = [0.7, -0.4]
    modes[:, 4] = rng.uniform(0, 6, 2)
    modes[:, 5:8] = rng.normal(size=(2, 3))
    A, _ = O.assemble(O.Q1, m["elem_dof"], m["cell_vert"], m["N"], m["active_bound"], rp, kc, O.FORM_SUPG,
                      O.make_coeff(kind=O.COEF_CURL_FOURIER, eps=1e-3, b=(3.0, 0, 0), f=1.0, modes=modes), quad=2,
                      dir_values=np.zeros(m["N"] - m["active_bound"]))
    N, Na = m["N"], m["active_bound"]
    e = rng.standard_normal(N)
    e[Na:] = 0
    Ad = np.zeros((N, N))
    Ad[np.repeat(np.arange(N), np.diff(rp)), kc] = A
    return m, rp, kc, A, e, Ad @ e


def dp_learned(rank, world, port, out_dir):
    """Data-parallel training of the stencil network with the oracle's gradient
    (BF16 forward rounding included): each rank its own problem, the gradients
    averaged over the ranks by train_data_parallel, the same plain update on
    every rank."""
    sys.path.insert(0, ROOT)
    dist = init(rank, world, port)
    from parmoon_b200 import learned as PL
    from oracle import learned_oracle as LO
    m, rp, kc, A, e, r = learned_problem(100 + rank)
    state = {"w": PL.init_weights(0).astype(np.float32)}

    def grad_fn(it):
        loss, g = LO.loss_and_grad(LO.bf16_round(state["w"]), 4, rp, kc, A, m["active_bound"], m["dof_lat"], e, r)
        return loss, g.astype(np.float32)

    def apply_fn(g):
        state["w"] = (state["w"] - 0.05 * g).astype(np.float32)

    hist = PL.train_data_parallel(grad_fn, apply_fn, 3, dist)
    np.savez(os.path.join(out_dir, f"learned{rank}.npz"), w=state["w"], hist=np.array(hist))
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
