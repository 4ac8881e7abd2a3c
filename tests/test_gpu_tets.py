"""P2 tetrahedra (the unstructured configuration): hexahedra split into six
Kuhn tetrahedra, interior vertices jittered by up to 0.2 h, lognormal
diffusion from seeded Fourier modes (correlation length 0.1, sigma 1), b = 0,
f = 1.  Assembly against the oracle (1e-12) and the FGMRES + V-cycle solve
against a dense solve of the same system."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [0, 1])
def test_p2_tet_lognormal_solve(pmg, oracle, prec):
    from parmoon_b200.configs import lognormal_modes
    modes = lognormal_modes(11)
    levels = pmg.struct_hierarchy(pmg.P2_TET, 4, 3, jitter=0.2, seed=4)
    F = levels[-1]
    h = pmg.Handle(3, pmg.default_params(precision=prec, lin_red=1e-14, lin_maxit=300, restart=30))
    h.set_coefficients(pmg.coeff(kind=pmg.COEF_LOGNORMAL, eps=1.0, f=1.0, modes=modes))
    pmg.load_hierarchy(h, levels)
    h.assemble(-1, pmg.FORM_GALERKIN, copy_out=False)
    A = h.get_matrix(2)
    b = h.get_rhs(2)
    Ao, bo = oracle.assemble(oracle.P2, F["elem_dof"], F["cell_vert"], F["N"], F["active_bound"], F["rowptr"],
                             F["kcol"], oracle.FORM_GALERKIN,
                             oracle.make_coeff(kind=oracle.COEF_LOGNORMAL, eps=1.0, f=1.0, modes=modes), quad=111,
                             dir_values=np.zeros(F["N"] - F["active_bound"]))
    assert np.max(np.abs(A - Ao)) <= 1e-12 * np.max(np.abs(Ao))
    assert np.max(np.abs(b - bo)) <= 1e-12 * np.max(np.abs(bo))
    _, st, rc = h.solve()
    assert rc == 0 and st.rel_res <= 1e-13
    x = h.get_solution()
    N = F["N"]
    D = np.zeros((N, N))
    D[np.repeat(np.arange(N), np.diff(F["rowptr"])), F["kcol"]] = Ao
    xd = np.linalg.solve(D, bo)
    assert np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-10
    h.close()
