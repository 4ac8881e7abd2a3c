"""Known answers from the mathematics (the reference's own verification is by
manufactured solutions, CD3D_ParMooN.C:516-543).

1. The Q1 Laplacian stencil on a uniform cube of cell size h, assembled on the
   device: diagonal 8h/3, face neighbours 0, edge neighbours -h/6, corner
   neighbours -h/12 (Gauss2 integrates the trilinear products exactly).
2. Convergence of the manufactured solution u = sin(pi x) sin(pi y) sin(pi z)
   (-Laplace u = 3 pi^2 u, homogeneous Dirichlet data): the L2 error of the
   device solution falls like h^2 for Q1 and h^3 for Q2, the H1-semi error
   like h and h^2 (ratios between n and 2n cells within 15 % of 4 / 8 and
   2 / 4).  The errors are integrated by the oracle's L2H1Errors restatement."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_q1_laplace_stencil(pmg):
    n = 6
    h_ = 1.0 / n
    levels = pmg.struct_hierarchy(pmg.Q1_HEX, n, 1)
    L = levels[-1]
    h = pmg.Handle(1)
    h.set_coefficients(pmg.coeff(kind=pmg.COEF_CONST, eps=1.0, f=0.0))
    pmg.load_hierarchy(h, levels)
    h.assemble(-1, pmg.FORM_GALERKIN, copy_out=False)
    A = h.get_matrix(0)
    lat, n1 = L["dof_lat"], n + 1
    ijk = np.stack([lat % n1, (lat // n1) % n1, lat // (n1 * n1)], axis=1)
    expect = {0: 8 * h_ / 3, 1: 0.0, 2: -h_ / 6, 3: -h_ / 12}
    checked = 0
    for r in range(L["active_bound"]):
        if np.any(ijk[r] < 2) or np.any(ijk[r] > n - 2):
            continue  # rows whose neighbours are all active
        for p in range(L["rowptr"][r], L["rowptr"][r + 1]):
            k = int(np.sum(np.abs(ijk[L["kcol"][p]] - ijk[r])))
            assert abs(A[p] - expect[k]) <= 1e-14, (r, k, A[p])
        assert L["rowptr"][r + 1] - L["rowptr"][r] == 27
        checked += 1
    assert checked == (n - 3) ** 3
    h.close()


@pytest.mark.parametrize("elem,rates", [("Q1_HEX", (4.0, 2.0)), ("Q2_HEX", (8.0, 4.0))])
def test_manufactured_solution_converges_at_the_element_order(pmg, oracle, elem, rates):
    et = getattr(pmg, elem)
    oe = oracle.Q1 if elem == "Q1_HEX" else oracle.Q2
    errs = []
    for n in (8, 16):
        levels = pmg.struct_hierarchy(et, n, 3)
        h = pmg.Handle(3, pmg.default_params(lin_red=1e-13, lin_maxit=200))
        h.set_coefficients(pmg.coeff(kind=pmg.COEF_SINE_RHS, eps=1.0))
        pmg.load_hierarchy(h, levels)
        h.assemble(-1, pmg.FORM_GALERKIN, copy_out=False)
        _, st, rc = h.solve()
        assert rc == 0
        F = levels[-1]
        errs.append(oracle.errors(oe, F["elem_dof"], F["cell_vert"], h.get_solution(), 3 if elem == "Q1_HEX" else 4, 0))
        h.close()
    l2_ratio, h1_ratio = errs[0][0] / errs[1][0], errs[0][1] / errs[1][1]
    assert abs(l2_ratio / rates[0] - 1) <= 0.15, (errs, l2_ratio)
    assert abs(h1_ratio / rates[1] - 1) <= 0.15, (errs, h1_ratio)
