"""The smoother variants of TMultiGrid3D::Smooth (src/FE/MultiGrid3D.C:117-446)
and the step-length control of TMultiGrid3D::Cycle (:517-523, :655-663,
TMGLevel3D::StepLengthControl, src/FE/MGLevel3D.C:908-961) through the C ABI:

  * one V-cycle (pmg_vcycle) with damped Jacobi (MGLevel3D.C:469-560), SOR
    (:280-361) or SSOR, with and without step-length control, against the
    oracle's V-cycle with the same smoother in the same (colour) row order;
  * the FGMRES solve with each of them reaches |r| <= 1e-10 |r0| in the FP64
    true residual.

Bars as for the SSOR V-cycle (tests/test_gpu_vcycle.py): FP64 within 1e-10
relative (max norm) of the oracle, FP32 within 1e-4."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

VARIANTS = [  # (smoother, omega, slc_all, slc_fine)
    (1, 0.8, 0, 0),
    (2, 1.0, 0, 0),
    (2, 0.9, 0, 1),
    (3, 1.0, 1, 0),
    (1, 0.7, 1, 0),
]


def _setup(pmg, elem, n, nl, prec, smoother, omega, slc_all, slc_fine):
    levels = pmg.struct_hierarchy(elem, n, nl)
    prm = pmg.default_params(precision=prec, smoother=smoother, smooth_omega=omega, slc_all=slc_all,
                             slc_fine=slc_fine)
    h = pmg.Handle(nl, prm)
    h.set_coefficients(pmg.coeff(kind=0, eps=1e-3, b=(1, .5, .25), f=1.0))
    pmg.load_hierarchy(h, levels, dirichlet=lambda x, y, z: np.sin(3 * x) + y * z)
    h.assemble(-1, pmg.FORM_SUPG, copy_out=False)
    return h, levels


@pytest.mark.parametrize("smoother,omega,slc_all,slc_fine", VARIANTS)
@pytest.mark.parametrize("prec,tol", [(0, 1e-10), (1, 1e-4)])
@pytest.mark.parametrize("elem,n,nl", [(1, 32, 4), (2, 16, 3)])
def test_vcycle_variant_matches_oracle(pmg, oracle, elem, n, nl, prec, tol, smoother, omega, slc_all, slc_fine):
    import torch
    h, levels = _setup(pmg, elem, n, nl, prec, smoother, omega, slc_all, slc_fine)
    olev = []
    for l, L in enumerate(levels):
        d = dict(N=L["N"], Na=L["active_bound"], rp=L["rowptr"], kc=L["kcol"], a=h.get_matrix(l),
                 colors=L["colors"], n_colors=L["n_colors"])
        if l > 0:
            d["P"] = L["P"]
        olev.append(d)
    F = levels[-1]
    rng = np.random.default_rng(5)
    for call in range(2):
        v = rng.standard_normal(F["N"])
        vd = torch.tensor(v, dtype=torch.float64, device="cuda")
        zd = torch.empty_like(vd)
        h.vcycle(vd.data_ptr(), zd.data_ptr())
        torch.cuda.synchronize()
        z = zd.cpu().numpy()
        zo = oracle.mg_apply(olev, v, coarse_direct=True, omega=omega, smoother=smoother, slc_all=bool(slc_all),
                             slc_fine=bool(slc_fine))
        err = float(np.max(np.abs(z - zo)) / np.max(np.abs(zo)))
        assert err < tol, (call, err)
    h.close()


@pytest.mark.parametrize("smoother,omega,slc_all,slc_fine", VARIANTS)
def test_solve_with_variant_converges(pmg, oracle, smoother, omega, slc_all, slc_fine):
    h, levels = _setup(pmg, 2, 16, 3, 1, smoother, omega, slc_all, slc_fine)
    _, st, rc = h.solve()
    assert rc == 0 and st.rel_res <= 1e-10, (rc, st.rel_res)
    assert st.smoother_used == smoother
    F = levels[-1]
    x = h.get_solution()
    A, b = h.get_matrix(2), h.get_rhs(2)
    r = b - oracle.spmv(F["rowptr"], F["kcol"], A, x)
    assert np.linalg.norm(r) <= 1.05e-10 * st.res0
    h.close()


def test_unbuilt_smoother_codes_are_rejected(pmg):
    """Codes the reference has but this library does not build (ILU = 4, the
    MPI reorderings 5-7) and invalid counts come back as PMG_ERR_ARG, from
    pmg_create and from pmg_set_params."""
    import ctypes
    for kw in (dict(smoother=4), dict(smoother=0), dict(coarse_smoother=4), dict(pre_smooth=-1),
               dict(slc_all=2), dict(smooth_omega=0.0), dict(precision=3)):
        p = pmg.default_params(**kw)
        hh = ctypes.c_void_p()
        assert pmg.lib().pmg_create(ctypes.byref(hh), 2, ctypes.byref(p)) == pmg.ERR_ARG, kw
        h = pmg.Handle(2)
        with pytest.raises(pmg.PmgError) as e:
            h.set_params(p)
        assert e.value.code == pmg.ERR_ARG
        h.close()


@pytest.mark.parametrize("coarse", [1, 2, 3])
@pytest.mark.parametrize("prec,tol", [(0, 1e-10), (1, 1e-4)])
def test_iterative_coarse_solve_matches_oracle(pmg, oracle, coarse, prec, tol):
    """The iterative coarsest-level solve (MultiGrid3D.C:262-330: smoothing
    steps until |r| <= coarse_red |r_0| or coarse_maxit steps) with Jacobi,
    SOR or SSOR, inside one V-cycle, against the oracle's."""
    import torch
    levels = pmg.struct_hierarchy(1, 32, 4)
    prm = pmg.default_params(precision=prec, coarse_smoother=coarse, coarse_maxit=25, coarse_red=1e-3,
                             smooth_omega=0.8 if coarse == 1 else 1.0)
    h = pmg.Handle(4, prm)
    h.set_coefficients(pmg.coeff(kind=0, eps=1e-3, b=(1, .5, .25), f=1.0))
    pmg.load_hierarchy(h, levels, dirichlet=lambda x, y, z: np.sin(3 * x) + y * z)
    h.assemble(-1, pmg.FORM_SUPG, copy_out=False)
    olev = []
    for l, L in enumerate(levels):
        d = dict(N=L["N"], Na=L["active_bound"], rp=L["rowptr"], kc=L["kcol"], a=h.get_matrix(l),
                 colors=L["colors"], n_colors=L["n_colors"])
        if l > 0:
            d["P"] = L["P"]
        olev.append(d)
    v = np.random.default_rng(3).standard_normal(levels[-1]["N"])
    vd = torch.tensor(v, dtype=torch.float64, device="cuda")
    zd = torch.empty_like(vd)
    h.vcycle(vd.data_ptr(), zd.data_ptr())
    torch.cuda.synchronize()
    z = zd.cpu().numpy()
    zo = oracle.mg_apply(olev, v, coarse_direct=False, coarse_smoother=coarse, coarse_maxit=25, coarse_red=1e-3,
                         omega=0.8 if coarse == 1 else 1.0)
    err = float(np.max(np.abs(z - zo)) / np.max(np.abs(zo)))
    assert err < tol, err
    h.close()
