"""Level set-up on the device (csrc/setup_gpu.cu).

  * pmg_build_level_csr builds the CSR pattern of TSquareStructure3D + Sort
    (src/FE/SquareStructure3D.C:58-527, SquareStructure.C:91-110) from the
    element -> dof map: bit-equal to the reference's own patterns (golden
    fixtures of the compiled reference, hexahedra and tetrahedra, every level)
    and to the host builder on larger structured meshes;
  * pmg_build_transfer builds the nested prolongation (GetProlongationMatrix3D
    + Prolongate, FEDatabase3D.C:1656-1815, MGComponents3D.C:208-488):
    applied to the reference's probe vectors it reproduces the reference's
    Prolongate / DefectRestriction (1e-13), and it equals the host builder;
  * a hierarchy set up entirely on the device solves to the same solution as
    the host-built one."""
import numpy as np
import pytest

from conftest import golden
from test_host_side import locate_cells

pytestmark = pytest.mark.gpu


def n_levels(g):
    return sum(1 for k in g.files if k.endswith("_rowptr"))


@pytest.mark.parametrize("name", ["q1_laplace", "q2_supg", "p1tet_laplace", "p2tet_supg"])
def test_device_csr_equals_reference_structure(pmg, name):
    g = golden(name)
    nl = n_levels(g)
    h = pmg.Handle(nl)
    for l in range(nl):
        p = f"L{l}_"
        N, Na, nloc = int(g[p + "N"]), int(g[p + "active_bound"]), int(g[p + "n_loc"])
        nnz = h.build_level_csr(l, g[p + "elem_dof"], nloc, N, Na)
        rp, kc = h.get_level_csr(l)
        assert nnz == g[p + "kcol"].size
        assert np.array_equal(rp, g[p + "rowptr"]) and np.array_equal(kc, g[p + "kcol"])
    h.close()


@pytest.mark.parametrize("elem,n", [(2, 32), (1, 64), (12, 16), (11, 24)])
def test_device_csr_equals_host_builder(pmg, elem, n):
    L = pmg.struct_level(elem, n)
    nloc = {1: 8, 2: 27, 11: 4, 12: 10}[elem]
    h = pmg.Handle(1)
    h.build_level_csr(0, L["elem_dof"], nloc, L["N"], L["active_bound"])
    rp, kc = h.get_level_csr(0)
    assert np.array_equal(rp, L["rowptr"]) and np.array_equal(kc, L["kcol"])
    h.close()


@pytest.mark.parametrize("name,elem", [("q1_laplace", 1), ("q2_supg", 2), ("p1tet_laplace", 11), ("p2tet_supg", 12)])
def test_device_transfer_matches_reference_prolongate(pmg, name, elem):
    g = golden(name)
    nl = n_levels(g)
    h = pmg.Handle(nl)
    for l in range(nl):
        p = f"L{l}_"
        h.set_level_csr(l, g[p + "rowptr"], g[p + "kcol"], int(g[p + "active_bound"]))
        h.set_level_mesh(l, elem, g[p + "elem_dof"], g[p + "cell_vert"], brick=elem in (1, 2))
    for l in range(1, nl):
        c, f = f"L{l-1}_", f"L{l}_"
        xyz = g[f + "dof_xyz"].reshape(-1, 3)
        owner = locate_cells(elem, g[c + "cell_vert"], xyz)
        h.build_transfer(l, xyz, owner)
        rp, col, val = h.get_transfer(l)
        hrp, hcol, hval = pmg.nested_prolongation(elem, g[c + "elem_dof"], g[c + "cell_vert"], int(g[c + "N"]), xyz,
                                                  owner)
        assert np.array_equal(rp, hrp) and np.array_equal(col, hcol) and np.max(np.abs(val - hval)) < 1e-14
        ci = g[f"T{l}_coarse_in"]
        pf = np.add.reduceat(val * ci[col], rp[:-1]) if col.size else np.zeros(xyz.shape[0])
        assert np.max(np.abs(pf - g[f"T{l}_prolongated"])) < 1e-13
        d = g[f"T{l}_fine_in"]
        r = np.zeros(ci.size)
        np.add.at(r, col, val * np.repeat(d, np.diff(rp)))
        assert np.max(np.abs(r - g[f"T{l}_restricted"])) < 1e-13
    h.close()


@pytest.mark.parametrize("elem,n,nl", [(2, 16, 3), (12, 8, 3)])
def test_device_built_hierarchy_solves_like_host_built(pmg, elem, n, nl):
    levels = pmg.struct_hierarchy(elem, n, nl)
    ck = pmg.coeff(kind=pmg.COEF_CONST, eps=1e-3, b=(1.0, 0.5, 0.25), f=1.0)
    dirichlet = lambda x, y, z: (np.abs(x) < 1e-12).astype(float)
    # host-built reference
    h0 = pmg.Handle(nl, pmg.default_params(lin_red=1e-13))
    h0.set_coefficients(ck)
    pmg.load_hierarchy(h0, levels, dirichlet=dirichlet)
    h0.assemble(-1, pmg.FORM_SUPG, copy_out=False)
    _, st0, _ = h0.solve()
    x0 = h0.get_solution()
    h0.close()
    # device-built patterns and transfers
    nloc = {1: 8, 2: 27, 11: 4, 12: 10}[elem]
    h = pmg.Handle(nl, pmg.default_params(lin_red=1e-13))
    h.set_coefficients(ck)
    for l, L in enumerate(levels):
        h.build_level_csr(l, L["elem_dof"], nloc, L["N"], L["active_bound"])
        h.set_level_mesh(l, elem, L["elem_dof"], L["cell_vert"], brick=elem in (1, 2))
        h.set_row_colors(l, L["colors"], L["n_colors"])
        Na = L["active_bound"]
        xyz = L["dof_xyz"].reshape(-1, 3)
        h.set_dirichlet_values(l, dirichlet(*xyz[Na:].T))
        if l > 0:
            owner = locate_cells(elem, levels[l - 1]["cell_vert"], xyz)
            h.build_transfer(l, xyz, owner)
    h.assemble(-1, pmg.FORM_SUPG, copy_out=False)
    _, st, rc = h.solve()
    assert rc == 0 and abs(st.iterations - st0.iterations) <= 1
    x = h.get_solution()
    assert np.linalg.norm(x - x0) <= 1e-10 * np.linalg.norm(x0)
    h.close()
