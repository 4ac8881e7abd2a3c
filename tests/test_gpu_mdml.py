"""The non-conforming multilevel method (SC_MG_TYPE_SCALAR = 1) on the device:
N_Q1 levels under the conforming finest level, as CD3D_ParMooN.C:258-313 builds
them.  Against the compiled reference's dumps: every level's matrix and rhs
(1e-12 of the row's largest entry, all three assembly kernels) and the solution
of the FGMRES + V-cycle on the reference's own hierarchy (1e-10 relative L2,
both solved to |r| <= 1e-14 |r0|).  On a structured 32^3 hierarchy the
multilevel preconditioner solves the same finest system as the conforming GMG,
so the two solutions agree."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

CASES = [("mdml_q1_laplace", 1, dict(kind=1, eps=1.0)),
         ("mdml_q1_supg", 2, dict(kind=0, eps=1e-3, b=(1, .5, .25), f=1.0)),
         ("mdml_q2_supg", 2, dict(kind=0, eps=1e-6, b=(1, .5, .25), f=1.0))]


def levels_of(g):
    return sum(1 for k in g.files if k.endswith("_rowptr"))


def elem_of(pmg, g, l):
    return {6: pmg.NQ1_HEX, 8: pmg.Q1_HEX, 27: pmg.Q2_HEX}[int(g[f"L{l}_n_loc"])]


def load_reference_hierarchy(pmg, g, h):
    nl = levels_of(g)
    for l in range(nl):
        q = f"L{l}_"
        Na = int(g[q + "active_bound"])
        h.set_level_csr(l, g[q + "rowptr"], g[q + "kcol"], Na)
        h.set_level_mesh(l, elem_of(pmg, g, l), g[q + "elem_dof"], g[q + "cell_vert"], brick=True)
        h.set_dirichlet_values(l, g[q + "rhs"][Na:])
        if l > 0:
            p = f"L{l-1}_"
            rp, col, val = pmg.cell_prolongation(elem_of(pmg, g, l - 1), g[p + "elem_dof"], g[p + "cell_vert"],
                                                 int(g[p + "N"]), elem_of(pmg, g, l), g[q + "elem_dof"],
                                                 g[q + "cell_vert"], g[q + "parent"], int(g[q + "N"]))
            h.set_transfer(l, rp, col, val, int(g[p + "N"]))


def poly_of(g):
    return 2 if "order=2" in list(g["params"]) else 1


@pytest.mark.parametrize("name,form,ck", CASES)
@pytest.mark.parametrize("path", [0, 1, 2])
def test_assembly_of_every_level_matches_reference(pmg, name, form, ck, path):
    g = golden(name)
    nl = levels_of(g)
    h = pmg.Handle(nl, pmg.default_params(assembly_kernel=path, poly_degree=poly_of(g)))
    h.set_coefficients(pmg.coeff(**ck))
    load_reference_hierarchy(pmg, g, h)
    for l in range(nl):
        q = f"L{l}_"
        e, r = h.assemble(l, form)
        ref, rp = g[q + "entries"], g[q + "rowptr"]
        rowmax = np.maximum.reduceat(np.abs(ref), rp[:-1])[np.repeat(np.arange(rp.size - 1), np.diff(rp))]
        assert np.max(np.abs(e - ref) / rowmax) <= 1e-12, (l, path)
        assert np.max(np.abs(r - g[q + "rhs"])) <= 1e-12 * max(1.0, np.max(np.abs(g[q + "rhs"]))), (l, path)
    h.close()


@pytest.mark.parametrize("name,form,ck", CASES)
@pytest.mark.parametrize("prec", [0, 1])
def test_solve_on_reference_hierarchy_matches_reference(pmg, name, form, ck, prec):
    g = golden(name)
    nl = levels_of(g)
    h = pmg.Handle(nl, pmg.default_params(lin_red=1e-14, lin_maxit=300, restart=30, precision=prec,
                                          poly_degree=poly_of(g)))
    h.set_coefficients(pmg.coeff(**ck))
    load_reference_hierarchy(pmg, g, h)
    h.assemble(-1, form, copy_out=False)
    _, st, rc = h.solve()
    assert rc == 0
    x, ref = h.get_solution(), g["solution"]
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 1e-10, (st.iterations, st.rel_res)
    h.close()


@pytest.mark.parametrize("elem,n,geo", [("Q1_HEX", 32, 4), ("Q2_HEX", 16, 3)])
def test_structured_mdml_solves_the_conforming_system(pmg, elem, n, geo):
    et = getattr(pmg, elem)
    ck = pmg.coeff(kind=pmg.COEF_CONST, eps=1e-3, b=(1.0, 0.5, 0.25), f=1.0)
    prm = dict(lin_red=1e-13, lin_maxit=400, restart=30, precision=pmg.PREC_FP32)
    sols, its = [], []
    for levels in (pmg.mdml_hierarchy(et, n, geo), pmg.struct_hierarchy(et, n, geo)):
        h = pmg.Handle(len(levels), pmg.default_params(**prm))
        h.set_coefficients(ck)
        pmg.load_hierarchy(h, levels, dirichlet=lambda x, y, z: (x < 1e-12).astype(float))
        h.assemble(-1, pmg.FORM_SUPG, copy_out=False)
        _, st, rc = h.solve()
        assert rc == 0 and st.rel_res <= 1e-13
        sols.append(h.get_solution())
        its.append(st.iterations)
        h.close()
    assert np.linalg.norm(sols[0] - sols[1]) / np.linalg.norm(sols[1]) < 1e-10, its
