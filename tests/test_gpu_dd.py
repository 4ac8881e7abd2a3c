"""The domain-decomposed solve (pmg_solve_dd, parmoon_b200.dd) on two ranks.

This run has one GPU: both ranks run on it as separate processes, the halo
exchange and the sums of the inner products go through gloo on the host
between launches (the library's stream is idle during every callback), so no
kernel of one rank waits for the other.  Each rank owns a z-slab of the unit
cube with one layer of ghost cells; FGMRES runs over the ranks with the
subdomain V-cycles as an overlapping additive Schwarz preconditioner.  The
union of the ranks' owned values must equal the single-domain solution (both
solved to |r| <= 1e-12 |r0|: 1e-9 relative), and the true residual reached
must be below the tolerance."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import dist_workers as W

pytestmark = pytest.mark.gpu


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("elem,n,nl,prec", [(2, 16, 3, 1), (1, 32, 4, 0), (12, 8, 3, 1)])
def test_two_subdomains_solve_like_one(pmg, tmp_path, elem, n, nl, prec):
    world = 2
    mp.start_processes(W.dd_solve, args=(world, free_port(), str(tmp_path), elem, n, nl, prec), nprocs=world,
                       join=True, start_method="spawn")
    r = [np.load(os.path.join(tmp_path, f"dds{k}.npz")) for k in range(world)]
    for x in r:
        assert int(x["rc"]) == 0 and float(x["rel"]) <= 1e-12, (int(x["rc"]), float(x["rel"]))
    assert int(r[0]["its"]) == int(r[1]["its"])  # the ranks stop together
    levels = pmg.struct_hierarchy(elem, n, nl)
    h = pmg.Handle(nl, pmg.default_params(precision=prec, lin_red=1e-12, lin_maxit=400))
    h.set_coefficients(pmg.coeff(kind=pmg.COEF_CONST, eps=1e-3, b=(1.0, 0.5, 0.25), f=1.0))
    pmg.load_hierarchy(h, levels, dirichlet=lambda x, y, z: (np.abs(x) < 1e-12).astype(float))
    h.assemble(-1, pmg.FORM_SUPG, copy_out=False)
    h.solve()
    ref = h.get_solution()
    h.close()
    x = np.empty_like(ref)
    for k in range(world):
        x[r[k]["glob"]] = r[k]["x"]
    assert np.linalg.norm(x - ref) <= 1e-9 * np.linalg.norm(ref)
