"""Edge cases of the C ABI on the device: malformed patterns and meshes,
calls out of order, a solve that runs out of iterations, a singular coarsest
matrix, non-finite input, a level whose rows are all Dirichlet rows, and a
one-level hierarchy.  Every failure is a status code (the reference exits)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def code_of(fn):
    import parmoon_b200 as P
    with pytest.raises(P.PmgError) as ei:
        fn()
    return ei.value.code


def test_malformed_csr_is_rejected(pmg):
    L = pmg.struct_level(pmg.Q1_HEX, 2)
    rp, kc, na = L["rowptr"], L["kcol"], L["active_bound"]
    h = pmg.Handle(1)
    # columns not ascending in a row
    kc2 = kc.copy()
    kc2[rp[0]], kc2[rp[0] + 1] = kc[rp[0] + 1], kc[rp[0]]
    assert code_of(lambda: h.set_level_csr(0, rp, kc2, na)) == pmg.ERR_ARG
    # column out of range
    kc3 = kc.copy()
    kc3[rp[1] - 1] = L["N"] + 5
    assert code_of(lambda: h.set_level_csr(0, rp, kc3, na)) == pmg.ERR_ARG
    # a row without its diagonal: drop the diagonal entry of row 0
    d = rp[0] + int(np.where(kc[rp[0]:rp[1]] == 0)[0][0])
    kc4 = np.delete(kc, d)
    rp4 = rp.copy()
    rp4[1:] -= 1
    assert code_of(lambda: h.set_level_csr(0, rp4, kc4, na)) == pmg.ERR_ARG
    # mesh before pattern, dof index out of range, unknown element
    h2 = pmg.Handle(1)
    assert code_of(lambda: h2.set_level_mesh(0, pmg.Q1_HEX, L["elem_dof"], L["cell_vert"])) == pmg.ERR_STATE
    h2.set_level_csr(0, rp, kc, na)
    ed = L["elem_dof"].copy()
    ed.flat[3] = L["N"]
    assert code_of(lambda: h2.set_level_mesh(0, pmg.Q1_HEX, ed, L["cell_vert"])) == pmg.ERR_ARG
    h.close()
    h2.close()


def test_params_and_inputs_are_checked(pmg):
    levels = pmg.struct_hierarchy(pmg.Q1_HEX, 4, 2)
    h = pmg.Handle(2)
    assert code_of(lambda: h.set_params(pmg.default_params(restart=61))) == pmg.ERR_ARG
    assert code_of(lambda: h.set_params(pmg.default_params(assembly_kernel=3))) == pmg.ERR_ARG
    assert code_of(lambda: h.set_params(pmg.default_params(assembly_scatter=3))) == pmg.ERR_ARG
    pmg.load_hierarchy(h, levels)
    F = levels[-1]
    bad = np.zeros(F["N"] - F["active_bound"])
    bad[0] = np.inf
    assert code_of(lambda: h.set_dirichlet_values(1, bad)) == pmg.ERR_NONFINITE
    assert code_of(lambda: h.set_coefficients(pmg.coeff(kind=99))) == pmg.ERR_ARG
    h.close()


def test_iteration_limit_returns_the_iterate(pmg):
    levels = pmg.struct_hierarchy(pmg.Q2_HEX, 8, 2)
    h = pmg.Handle(2, pmg.default_params(lin_maxit=2, lin_red=1e-14))
    h.set_coefficients(pmg.coeff(kind=pmg.COEF_CONST, eps=1e-3, b=(1.0, 0.5, 0.25), f=1.0))
    pmg.load_hierarchy(h, levels)
    h.assemble(-1, pmg.FORM_SUPG, copy_out=False)
    _, st, rc = h.solve(raise_on_error=False)
    assert rc == pmg.ERR_NOT_CONVERGED
    assert st.iterations == 2 and 0 < st.rel_res < 1
    x = h.get_solution()
    assert np.all(np.isfinite(x))
    h.close()


def test_singular_coarsest_matrix(pmg):
    levels = pmg.struct_hierarchy(pmg.Q1_HEX, 4, 2)
    h = pmg.Handle(2)
    pmg.load_hierarchy(h, levels)
    h.assemble(-1, pmg.FORM_GALERKIN, copy_out=False)
    A0 = h.get_matrix(0)
    L0 = levels[0]
    rows = np.repeat(np.arange(L0["N"]), np.diff(L0["rowptr"]))
    A0[rows < L0["active_bound"]] = 0.0  # active block of the coarsest level zero
    h.set_matrix(0, A0)
    _, st, rc = h.solve(raise_on_error=False)
    assert rc == pmg.ERR_SINGULAR
    h.close()


def test_all_dirichlet_coarsest_level_and_one_level_hierarchy(pmg):
    # Q1 on one cell: every dof is a Dirichlet dof, the coarse solve is x = f
    levels = pmg.struct_hierarchy(pmg.Q1_HEX, 2, 2)
    assert levels[0]["active_bound"] == 0
    h = pmg.Handle(2)
    h.set_coefficients(pmg.coeff(kind=pmg.COEF_SINE_RHS, eps=1.0))
    pmg.load_hierarchy(h, levels, dirichlet=lambda x, y, z: x + y)
    h.assemble(-1, pmg.FORM_GALERKIN, copy_out=False)
    _, st, rc = h.solve()
    assert rc == 0 and st.rel_res <= 1e-10
    h.close()
    # one level: the V-cycle is the dense coarse solve, FGMRES converges at once
    one = pmg.struct_hierarchy(pmg.Q2_HEX, 2, 1)
    h1 = pmg.Handle(1)
    h1.set_coefficients(pmg.coeff(kind=pmg.COEF_CONST, eps=1.0, f=1.0))
    pmg.load_hierarchy(h1, one)
    h1.assemble(-1, pmg.FORM_GALERKIN, copy_out=False)
    _, st, rc = h1.solve()
    assert rc == 0 and st.iterations <= 2 and st.rel_res <= 1e-10
    h1.close()


def test_peak_probes_report_positive_throughput(pmg):
    """pmg_measure_peaks (the denominators of the DMMA and BF16 rooflines) runs
    its three probes and reports finite, positive TFLOP/s."""
    fma, dmma, hmma = pmg.measure_peaks()
    assert all(np.isfinite(v) and v > 1.0 for v in (fma, dmma, hmma)), (fma, dmma, hmma)


def test_non_parallelepiped_hexahedra_are_rejected(pmg):
    """The kernels map hexahedra affinely; a cell whose vertices do not form a
    parallelepiped (it would need HexaTrilinear) is an unsupported mesh, not a
    silently wrong matrix."""
    levels = pmg.struct_hierarchy(pmg.Q1_HEX, 2, 1)
    L = levels[-1]
    h = pmg.Handle(1)
    h.set_level_csr(0, L["rowptr"], L["kcol"], L["active_bound"])
    cv = L["cell_vert"].copy().reshape(-1, 8, 3)
    cv[0, 6] += 0.05  # move the far corner of cell 0
    with pytest.raises(pmg.PmgError) as e:
        h.set_level_mesh(0, pmg.Q1_HEX, L["elem_dof"], cv.ravel(), brick=True)
    assert e.value.code == pmg.ERR_UNSUPPORTED
    h.set_level_mesh(0, pmg.Q1_HEX, L["elem_dof"], L["cell_vert"], brick=True)  # the unchanged mesh is fine
    h.close()
