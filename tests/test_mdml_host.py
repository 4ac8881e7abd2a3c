"""The non-conforming multilevel hierarchy (SC_MG_TYPE_SCALAR = 1) on the host:
the N_Q1 element of the oracle and the library's transfer builder against the
reference's own assembly, Prolongate and DefectRestriction (golden dumps of
the compiled reference: N_Q1 on the 2^3, 4^3, 8^3 meshes plus the conforming
space on the 8^3 mesh), and the library's structured N_Q1 levels against the
oracle's.  No GPU."""
import numpy as np
import pytest
import scipy.sparse as sp

import parmoon_b200 as P
from conftest import golden
from oracle import cd3d as O

CASES = [("mdml_q1_laplace", O.FORM_GALERKIN, dict(kind=1, eps=1.0)),
         ("mdml_q1_supg", O.FORM_SUPG, dict(kind=0, eps=1e-3, b=(1, .5, .25), f=1.0)),
         ("mdml_q2_supg", O.FORM_SUPG, dict(kind=0, eps=1e-6, b=(1, .5, .25), f=1.0))]
ELEM = {6: (O.NQ1, P.NQ1_HEX), 8: (O.Q1, P.Q1_HEX), 27: (O.Q2, P.Q2_HEX)}


def levels_of(g):
    return sum(1 for k in g.files if k.endswith("_rowptr"))


def transfer_args(g, l, lib):
    k = 1 if lib else 0
    ce, fe = ELEM[int(g[f"L{l-1}_n_loc"])][k], ELEM[int(g[f"L{l}_n_loc"])][k]
    return (ce, g[f"L{l-1}_elem_dof"], g[f"L{l-1}_cell_vert"], int(g[f"L{l-1}_N"]), fe, g[f"L{l}_elem_dof"],
            g[f"L{l}_cell_vert"], g[f"L{l}_parent"], int(g[f"L{l}_N"]))


@pytest.mark.parametrize("name,form,ck", CASES)
def test_oracle_nq1_assembly_matches_reference(oracle, name, form, ck):
    """The oracle's N_Q1 (and conforming top level) matrices and rhs equal the
    reference's Assemble3D on its meshes (point-value N_Q1 basis, Gauss3)."""
    g = golden(name)
    # the SUPG delta's polynomial degree is one global value (INTERNAL_POLYNOMIAL_DEGREE
    # = ANSATZ_ORDER of the finest space), the N_Q1 levels included
    poly = 2 if "order=2" in list(g["params"]) else 1
    for l in range(levels_of(g)):
        q = f"L{l}_"
        N, Na = int(g[q + "N"]), int(g[q + "active_bound"])
        e = ELEM[int(g[q + "n_loc"])][0]
        A, r = O.assemble(e, g[q + "elem_dof"], g[q + "cell_vert"], N, Na, g[q + "rowptr"], g[q + "kcol"], form,
                          O.make_coeff(**ck), poly=poly, dir_values=g[q + "rhs"][Na:])
        rp = g[q + "rowptr"]
        rowmax = np.maximum.reduceat(np.abs(g[q + "entries"]), rp[:-1])[np.repeat(np.arange(N), np.diff(rp))]
        assert np.max(np.abs(A - g[q + "entries"]) / rowmax) <= 1e-12, l
        assert np.max(np.abs(r - g[q + "rhs"])) <= 1e-12 * max(1.0, np.max(np.abs(g[q + "rhs"]))), l


@pytest.mark.parametrize("name", [c[0] for c in CASES])
def test_transfers_match_reference_prolongate(oracle, name):
    """Prolongate / DefectRestriction of the reference (N_Q1 -> N_Q1 between
    meshes, averaged over the fine cells of a face; N_Q1 -> conforming on one
    mesh, averaged over the cells of a vertex): the oracle's operational
    restatement and the library's CSR operator (pmg_cell_prolongation, whose
    transpose is the restriction) both agree with the reference's probes."""
    g = golden(name)
    for l in range(1, levels_of(g)):
        cin, fin = g[f"T{l}_coarse_in"], g[f"T{l}_fine_in"]
        pro, res = g[f"T{l}_prolongated"], g[f"T{l}_restricted"]
        args = transfer_args(g, l, lib=False)
        assert np.max(np.abs(O.cell_transfer(0, *args, cin) - pro)) <= 1e-14
        assert np.max(np.abs(O.cell_transfer(1, *args, fin) - res)) <= 1e-14
        rp, col, val = P.cell_prolongation(*transfer_args(g, l, lib=True))
        Pm = sp.csr_matrix((val, col, rp), shape=(pro.size, cin.size))
        assert np.max(np.abs(Pm @ cin - pro)) <= 1e-14
        assert np.max(np.abs(Pm.T @ fin - res)) <= 1e-14


def test_structured_nq1_levels_match_oracle_and_reference_sizes(oracle):
    """The library's structured N_Q1 builder equals the oracle's (numbering,
    positions, element map), and the hierarchy has the reference's sizes:
    3 n^2 (n+1) faces, and the nnz of its TSquareStructure3D."""
    for n in (2, 4, 8):
        L = P.struct_level(P.NQ1_HEX, n)
        m = O.struct_mesh(O.NQ1, n)
        assert np.array_equal(L["elem_dof"], m["elem_dof"])
        assert np.array_equal(L["dof_xyz"].ravel(), m["dof_xyz"])
        assert np.array_equal(L["cell_vert"], m["cell_vert"])
        assert L["active_bound"] == m["active_bound"] == 3 * n * n * (n - 1)
    g = golden("mdml_q1_laplace")
    lv = P.mdml_hierarchy(P.Q1_HEX, 8, 3)
    for l, L in enumerate(lv):
        assert L["N"] == int(g[f"L{l}_N"]) and L["active_bound"] == int(g[f"L{l}_active_bound"])
        assert int(L["rowptr"][-1]) == g[f"L{l}_kcol"].size


def test_structured_transfers_match_oracle(oracle):
    """pmg_cell_prolongation on the structured hierarchy equals the oracle's
    operational Prolongate / DefectRestriction (random probes)."""
    lv = P.mdml_hierarchy(P.Q2_HEX, 8, 3)
    rng = np.random.default_rng(0)
    for l in range(1, len(lv)):
        C, F = lv[l - 1], lv[l]
        same = l == len(lv) - 1
        par = np.arange(F["n_cells"], dtype=np.int32) if same else P.struct_parents(F["n"])
        ce = O.NQ1
        fe = O.NQ1 if F["elem"] == P.NQ1_HEX else O.Q2
        args = (ce, C["elem_dof"], C["cell_vert"], C["N"], fe, F["elem_dof"], F["cell_vert"], par, F["N"])
        rp, col, val = F["P"]
        Pm = sp.csr_matrix((val, col, rp), shape=(F["N"], C["N"]))
        c, f = rng.standard_normal(C["N"]), rng.standard_normal(F["N"])
        assert np.max(np.abs(Pm @ c - O.cell_transfer(0, *args, c))) <= 1e-13
        assert np.max(np.abs(Pm.T @ f - O.cell_transfer(1, *args, f))) <= 1e-13
