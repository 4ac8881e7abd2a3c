"""The assembly kernels agree.  For coefficients constant in space the
library assembles A = |det J| sum_ab D_ab S_ab from reference matrices, on the
FP64 tensor cores (assembly_kernel = 0, automatic) or on the FP64 CUDA cores
(assembly_kernel = 2); for pure diffusion with a varying eps on Q1 / P1 / P2
the tensor-core kernel contracts per-point coefficients with a reference
table; the per-quadrature-point kernel (assembly_kernel = 1) sums over the
points.  Same matrices and rhs up to rounding order: 1e-13 relative to the
largest entry of the row."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("elem,form,kind,jitter,linear", [
    ("Q2_HEX", "SUPG", "CONST", 0.0, 1), ("Q2_HEX", "SUPG", "CONST", 0.0, 0), ("Q1_HEX", "SUPG", "SINE_RHS", 0.0, 1),
    ("Q1_HEX", "MASS_SUPG", "CONST", 0.0, 1), ("P2_TET", "SUPG", "CONST", 0.2, 1), ("P1_TET", "GALERKIN", "AMC", 0.2, 1),
    ("Q2_HEX", "MASS", "AMC", 0.0, 1), ("P2_TET", "STIFF_SUPG", "CONST", 0.2, 1), ("Q1_HEX", "GALERKIN", "CONST", 0.0, 0),
    ("P2_TET", "GALERKIN", "LOGNORMAL", 0.2, 1), ("Q1_HEX", "GALERKIN", "LOGNORMAL", 0.0, 1),
    ("P1_TET", "SUPG", "LOGNORMAL", 0.2, 0), ("Q1_HEX", "GALERKIN", "LOGNORMAL", 0.0, 0),
    ("NQ1_HEX", "SUPG", "CONST", 0.0, 1), ("NQ1_HEX", "SUPG", "CONST", 0.0, 0), ("NQ1_HEX", "GALERKIN", "SINE_RHS", 0.0, 0)])
def test_reference_matrix_kernel_equals_point_kernel(pmg, elem, form, kind, jitter, linear):
    from parmoon_b200.configs import lognormal_modes
    et = getattr(pmg, elem)
    fm = getattr(pmg, "FORM_" + form)
    levels = pmg.struct_hierarchy(et, 4, 2, jitter=jitter, seed=7)
    if kind == "LOGNORMAL":  # pure diffusion: b = 0, c = 0
        ck = pmg.coeff(kind=pmg.COEF_LOGNORMAL, eps=1e-2, f=2.0, modes=lognormal_modes(3))
    else:
        ck = pmg.coeff(kind=getattr(pmg, "COEF_" + kind), eps=1e-3, b=(1.0, -0.5, 0.25), c=0.3, f=2.0, t=0.4)
    out = []
    for path in (0, 1, 2):
        h = pmg.Handle(2, pmg.default_params(assembly_kernel=path, problem_linear=linear))
        h.set_coefficients(ck)
        pmg.load_hierarchy(h, levels, dirichlet=lambda x, y, z: x + 2 * y - z)
        h.assemble(-1, fm, copy_out=False)
        out.append([(h.get_matrix(l, 1 if form.startswith("MASS") else 0), h.get_rhs(l)) for l in range(2)])
        h.close()
    for l, L in enumerate(levels):
        A1, r1 = out[1][l]
        rows = np.repeat(np.arange(L["N"]), np.diff(L["rowptr"]))
        rowmax = np.maximum.reduceat(np.abs(A1), L["rowptr"][:-1])[rows]
        for path in (0, 2):
            A0, r0 = out[path][l]
            assert np.max(np.abs(A0 - A1) / rowmax) <= 1e-13, path
            assert np.max(np.abs(r0 - r1)) <= 1e-13 * max(1.0, np.max(np.abs(r1))), path


@pytest.mark.parametrize("elem,form,kind", [("P2_TET", "GALERKIN", "LOGNORMAL"), ("P2_TET", "SUPG", "CONST"),
                                            ("P1_TET", "SUPG", "LOGNORMAL"), ("P1_TET", "GALERKIN", "CONST")])
def test_five_point_tet_rule_matches_oracle(pmg, elem, form, kind):
    """quad_rule = PMG_QUAD_KEAST5, the 5-point degree-3 rule the P2 lognormal
    workload names, on every kernel path against the oracle's assembly with the
    same rule (1e-12 of the row's largest entry)."""
    from oracle import cd3d as O
    from parmoon_b200.configs import lognormal_modes
    et = getattr(pmg, elem)
    fm = getattr(pmg, "FORM_" + form)
    levels = pmg.struct_hierarchy(et, 4, 2, jitter=0.2, seed=11)
    if kind == "LOGNORMAL":
        kw = dict(kind=pmg.COEF_LOGNORMAL, eps=1e-2, f=2.0, modes=lognormal_modes(5))
    else:
        kw = dict(kind=pmg.COEF_CONST, eps=1e-3, b=(1.0, -0.5, 0.25), c=0.3, f=2.0)
    F = levels[-1]
    dv = F["dof_xyz"][F["active_bound"]:] @ np.array([1.0, 2.0, -1.0])
    ok = {"kind": kw["kind"], "eps": kw["eps"], "b": kw.get("b", (0, 0, 0)), "c": kw.get("c", 0.0), "f": kw["f"],
          "modes": kw.get("modes")}
    Ao, ro = O.assemble(getattr(O, elem[:2]), F["elem_dof"], F["cell_vert"], F["N"], F["active_bound"],
                        F["rowptr"], F["kcol"], getattr(O, "FORM_" + form), O.make_coeff(**ok), quad=105,
                        dir_values=dv)
    rows = np.repeat(np.arange(F["N"]), np.diff(F["rowptr"]))
    rowmax = np.maximum.reduceat(np.abs(Ao), F["rowptr"][:-1])[rows]
    for path in (0, 1, 2):
        h = pmg.Handle(2, pmg.default_params(assembly_kernel=path, quad_rule=pmg.QUAD_KEAST5))
        h.set_coefficients(pmg.coeff(**kw))
        pmg.load_hierarchy(h, levels, dirichlet=lambda x, y, z: x + 2 * y - z)
        h.assemble(-1, fm, copy_out=False)
        A, r = h.get_matrix(1), h.get_rhs(1)
        h.close()
        assert np.max(np.abs(A - Ao) / rowmax) <= 1e-12, path
        assert np.max(np.abs(r - ro)) <= 1e-12 * max(1.0, np.max(np.abs(ro))), path


def test_quad_rule_must_fit_the_element(pmg):
    levels = pmg.struct_hierarchy(pmg.Q1_HEX, 2, 1)
    h = pmg.Handle(1, pmg.default_params(quad_rule=pmg.QUAD_KEAST5))
    pmg.load_hierarchy(h, levels)
    with pytest.raises(pmg.PmgError) as e:
        h.assemble(-1, pmg.FORM_GALERKIN, copy_out=False)
    assert e.value.code == pmg.ERR_UNSUPPORTED
    h.close()


@pytest.mark.parametrize("elem,form,kind,jitter,kernel", [
    ("Q2_HEX", "SUPG", "CONST", 0.0, 0), ("Q1_HEX", "SUPG", "ROTATING", 0.0, 0), ("Q1_HEX", "MASS_SUPG", "ROTATING", 0.0, 0),
    ("P2_TET", "GALERKIN", "LOGNORMAL", 0.2, 0), ("P1_TET", "SUPG", "CONST", 0.2, 0), ("NQ1_HEX", "SUPG", "CONST", 0.0, 0),
    ("Q2_HEX", "SUPG", "SINE_RHS", 0.0, 1), ("P2_TET", "SUPG", "CURL_FOURIER", 0.2, 1)])
def test_row_gather_equals_colour_scatter(pmg, elem, form, kind, jitter, kernel):
    """assembly_scatter = 2 (local matrices, then every CSR row summed from its
    cells' rows in colour order) gives the same matrix and rhs, bit for bit,
    as assembly_scatter = 1 (each colour's cells adding into the matrix), on
    the tensor-core, per-point and diffusion paths, Dirichlet rows included,
    and on every level."""
    from parmoon_b200.configs import lognormal_modes, curl_modes
    et = getattr(pmg, elem)
    fm = getattr(pmg, "FORM_" + form)
    levels = pmg.struct_hierarchy(et, 8, 3, jitter=jitter, seed=5)
    if kind == "LOGNORMAL":
        ck = pmg.coeff(kind=pmg.COEF_LOGNORMAL, eps=1e-2, f=2.0, modes=lognormal_modes(4))
    elif kind == "CURL_FOURIER":
        m, scale = curl_modes(2)
        ck = pmg.coeff(kind=pmg.COEF_CURL_FOURIER, eps=1e-3, b=(scale, 0, 0), f=1.0, modes=m)
    else:
        ck = pmg.coeff(kind=getattr(pmg, "COEF_" + kind), eps=1e-3, b=(1.0, -0.5, 0.25), c=0.3, f=2.0, t=0.4)
    out = []
    for scatter in (1, 2):
        h = pmg.Handle(3, pmg.default_params(assembly_kernel=kernel, assembly_scatter=scatter))
        h.set_coefficients(ck)
        pmg.load_hierarchy(h, levels, dirichlet=lambda x, y, z: x + 2 * y - z)
        h.assemble(-1, fm, copy_out=False)
        h.assemble(-1, fm, copy_out=False)  # a second assembly overwrites every entry
        out.append([(h.get_matrix(l, 1 if form.startswith("MASS") else 0), h.get_rhs(l)) for l in range(3)])
        h.close()
    for l in range(3):
        assert np.array_equal(out[0][l][0], out[1][l][0]), l
        assert np.array_equal(out[0][l][1], out[1][l][1]), l
