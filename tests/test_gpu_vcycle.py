"""One preconditioner application through the C ABI (pmg_vcycle: zero start,
the Dirichlet part of v, one V-cycle -- MultiGridScaIte.C:89-130) against the
oracle's V-cycle, on random input vectors whose Dirichlet part is not zero.
The solve never produces such vectors (its Krylov vectors vanish on the
Dirichlet rows), so this is what checks that the active rows' Dirichlet
columns, which the solve copy of the level matrices keeps apart, are folded
back in; the hierarchies also run their levels of at most 8192 rows as one
cluster launch.

Bars: FP64 V-cycle within 1e-10 relative (max norm) of the oracle -- the two
differ in the order of partial sums and in the coarse solve (inverse of the
active block against dense elimination) -- and its Dirichlet part equal to
v's; FP32 V-cycle within 1e-4 relative (FP32 values and iterates).  Dropping
the finest level's Dirichlet columns moves the oracle's own V-cycle by 2.2e-2
relative on the Q1 Laplace case and by 7.8e-4 on the Q1 SUPG case (16^3, 3
levels), so both bars see that mistake."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("elem,n,nl,form,ck", [(1, 32, 4, 1, dict(kind=1, eps=1.0)),
                                               (1, 32, 4, 2, dict(kind=0, eps=1e-3, b=(1, .5, .25), f=1.0)),
                                               (2, 16, 3, 2, dict(kind=0, eps=1e-6, b=(1, .5, .25), f=1.0))])
@pytest.mark.parametrize("prec,tol", [(0, 1e-10), (1, 1e-4)])
def test_vcycle_matches_oracle(pmg, oracle, elem, n, nl, form, ck, prec, tol):
    import torch
    levels = pmg.struct_hierarchy(elem, n, nl)
    h = pmg.Handle(nl, pmg.default_params(precision=prec))
    h.set_coefficients(pmg.coeff(**ck))
    pmg.load_hierarchy(h, levels, dirichlet=lambda x, y, z: np.sin(3 * x) + y * z)
    h.assemble(-1, form, copy_out=False)
    olev = []
    for l, L in enumerate(levels):
        d = dict(N=L["N"], Na=L["active_bound"], rp=L["rowptr"], kc=L["kcol"], a=h.get_matrix(l),
                 colors=L["colors"], n_colors=L["n_colors"])
        if l > 0:
            d["P"] = L["P"]
        olev.append(d)
    F = levels[-1]
    rng = np.random.default_rng(7)
    for call in range(2):
        v = rng.standard_normal(F["N"])
        vd = torch.tensor(v, dtype=torch.float64, device="cuda")
        zd = torch.empty_like(vd)
        h.vcycle(vd.data_ptr(), zd.data_ptr())
        torch.cuda.synchronize()
        z = zd.cpu().numpy()
        zo = oracle.mg_apply(olev, v, coarse_direct=True)
        err = float(np.max(np.abs(z - zo)) / np.max(np.abs(zo)))
        assert err < tol, (call, err)
        if prec == 0:
            assert np.array_equal(z[F["active_bound"]:], v[F["active_bound"]:])
    h.close()
