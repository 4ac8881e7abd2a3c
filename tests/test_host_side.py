"""Host-side pieces that need no GPU: the C ABI library loads and exports every
declared entry point, and the product's structured set-up (C++ in the
library) agrees with the oracle's restatement and with the reference's own
CSR patterns."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

from conftest import ROOT, golden


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_ ]*?[\s\*]+(pmg_[A-Za-z0-9_]+)\s*\(", text, re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    import parmoon_b200 as P
    lib = P.lib()
    names = declared_functions()
    assert len(names) > 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_default_params_mirror_reference_defaults():
    import parmoon_b200 as P
    p = P.default_params()
    assert p.smoother == 3 and p.pre_smooth == 2 and p.post_smooth == 2  # SSOR(2,2)
    assert p.smooth_omega == 1.0 and p.gmg_damp == 1.0 and p.delta0 == 1.0
    assert p.sdfem_type == 2 and p.div_factor == 1e10


@pytest.mark.parametrize("elem,n", [(1, 4), (2, 3), (11, 3), (12, 2)])
def test_struct_builder_matches_oracle(oracle, elem, n):
    import parmoon_b200 as P
    L = P.struct_level(elem, n)
    O = oracle.struct_mesh(elem, n)
    assert L["N"] == O["N"] and L["active_bound"] == O["active_bound"]
    assert np.array_equal(L["elem_dof"], O["elem_dof"])
    assert np.allclose(L["cell_vert"], O["cell_vert"])
    assert np.allclose(L["dof_xyz"].ravel(), O["dof_xyz"])
    rp, kc = oracle.csr(O["elem_dof"], oracle.nloc_of(elem), O["N"], O["active_bound"])
    assert np.array_equal(L["rowptr"], rp) and np.array_equal(L["kcol"], kc)
    # lattice colouring is a proper colouring of the matrix graph
    c = L["colors"]
    for r in range(L["active_bound"]):
        cols = L["kcol"][L["rowptr"][r]:L["rowptr"][r + 1]]
        cols = cols[(cols != r) & (cols < L["active_bound"])]
        assert not np.any(c[cols] == c[r])


@pytest.mark.parametrize("elem,nc", [(1, 2), (2, 2), (11, 2), (12, 2)])
def test_struct_prolongation_matches_oracle(oracle, elem, nc):
    import parmoon_b200 as P
    C = P.struct_level(elem, nc)
    F = P.struct_level(elem, 2 * nc)
    rp, col, val = P.struct_prolongation(elem, nc, C["dof_lat"], F["dof_lat"])
    orp, ocol, oval = oracle.prolongation(elem, nc, C["dof_lat"], F["dof_lat"])
    assert np.array_equal(rp, orp) and np.array_equal(col, ocol)
    assert np.allclose(val, oval, rtol=0, atol=1e-15)
    # interpolation property: the coarse interpolant of a polynomial of the element's
    # degree prolongates to the fine interpolant (nested Kuhn / tensor refinement)
    deg = 2 if elem in (2, 12) else 1
    f = lambda x: 0.3 + x[:, 0] - 2 * x[:, 1] + 0.5 * x[:, 2] + (deg == 2) * (x[:, 0] * x[:, 1] - x[:, 2] ** 2)
    uc = f(C["dof_xyz"])
    uf = np.array([np.dot(val[rp[i]:rp[i + 1]], uc[col[rp[i]:rp[i + 1]]]) for i in range(F["N"])])
    assert np.max(np.abs(uf - f(F["dof_xyz"]))) < 1e-13


def lattice_index(xyz, n1):
    ijk = np.rint(np.asarray(xyz).reshape(-1, 3) * (n1 - 1)).astype(np.int64)
    return ijk[:, 0] + n1 * (ijk[:, 1] + n1 * ijk[:, 2])


@pytest.mark.parametrize("name,elem,p", [("q1_laplace", 1, 1), ("q2_supg", 2, 2)])
def test_struct_builder_pattern_equals_reference_up_to_numbering(name, elem, p):
    """Same sparsity graph as TSquareStructure3D once dofs are matched by position."""
    import parmoon_b200 as P
    g = golden(name)
    nl = sum(1 for k in g.files if k.endswith("_rowptr"))
    l = nl - 1
    n = int(round((int(g[f"L{l}_N"]) ** (1 / 3) - 1) / p))
    L = P.struct_level(elem, n)
    assert L["N"] == int(g[f"L{l}_N"]) and L["active_bound"] == int(g[f"L{l}_active_bound"])
    n1 = p * n + 1
    ref_lat = lattice_index(g[f"L{l}_dof_xyz"], n1)
    mine_lat = L["dof_lat"].astype(np.int64)
    # permutation: reference dof -> my dof
    inv = np.empty(n1 ** 3, dtype=np.int64)
    inv[mine_lat] = np.arange(L["N"])
    perm = inv[ref_lat]
    rp, kc = g[f"L{l}_rowptr"], g[f"L{l}_kcol"]
    ref_edges = set(zip(np.repeat(perm, np.diff(rp)).tolist(), perm[kc].tolist()))
    my_edges = set(zip(np.repeat(np.arange(L["N"]), np.diff(L["rowptr"])).tolist(), L["kcol"].tolist()))
    assert ref_edges == my_edges


def locate_cells(elem, cell_vert, pts):
    """Index of a cell of the (affine) mesh containing each point, by inverting every cell's map."""
    v = np.asarray(cell_vert).reshape(-1, 8, 3)
    if elem in (1, 2):
        J = np.stack([(v[:, 1] - v[:, 0]) / 2, (v[:, 3] - v[:, 0]) / 2, (v[:, 4] - v[:, 0]) / 2], axis=2)
        x0 = (v[:, 1] + v[:, 3] + v[:, 4] - v[:, 0]) / 2
    else:
        J = np.stack([v[:, 1] - v[:, 0], v[:, 2] - v[:, 0], v[:, 3] - v[:, 0]], axis=2)
        x0 = v[:, 0]
    Ji = np.linalg.inv(J)
    ref = np.einsum("cij,pcj->pci", Ji, pts[:, None, :] - x0[None])  # [points, cells, 3]
    tol = 1e-10
    if elem in (1, 2):
        inside = np.all(np.abs(ref) <= 1 + tol, axis=2)
    else:
        inside = np.all(ref >= -tol, axis=2) & (ref.sum(axis=2) <= 1 + tol)
    assert inside.any(axis=1).all()
    return inside.argmax(axis=1).astype(np.int32)


@pytest.mark.parametrize("name,elem", [("q1_laplace", 1), ("q2_supg", 2), ("p1tet_laplace", 11), ("p2tet_supg", 12)])
def test_nested_prolongation_matches_reference_prolongate(name, elem):
    """Prolongate and DefectRestriction of the reference (MGComponents3D.C:208-488, 732-1014)
    on its own refined meshes, tetrahedra included, equal P and P^T from pmg_nested_prolongation."""
    import parmoon_b200 as P
    g = golden(name)
    nl = sum(1 for k in g.files if k.endswith("_rowptr"))
    for l in range(1, nl):
        c, f = f"L{l-1}_", f"L{l}_"
        xyz = g[f + "dof_xyz"].reshape(-1, 3)
        owner = locate_cells(elem, g[c + "cell_vert"], xyz)
        rp, col, val = P.nested_prolongation(elem, g[c + "elem_dof"], g[c + "cell_vert"], int(g[c + "N"]), xyz, owner)
        ci = g[f"T{l}_coarse_in"]
        pf = np.array([np.dot(val[rp[i]:rp[i + 1]], ci[col[rp[i]:rp[i + 1]]]) for i in range(xyz.shape[0])])
        assert np.max(np.abs(pf - g[f"T{l}_prolongated"])) < 1e-13
        d = g[f"T{l}_fine_in"]
        r = np.zeros(ci.size)
        np.add.at(r, col, val * np.repeat(d, np.diff(rp)))
        assert np.max(np.abs(r - g[f"T{l}_restricted"])) < 1e-13


def test_nested_prolongation_equals_lattice_interpolation():
    """On the structured hierarchy the nested builder reproduces pmg_struct_prolongation."""
    import parmoon_b200 as P
    for elem in (1, 2, 11, 12):
        C, F = P.struct_level(elem, 2), P.struct_level(elem, 4)
        owner = locate_cells(elem, C["cell_vert"], F["dof_xyz"])
        rp, col, val = P.nested_prolongation(elem, C["elem_dof"], C["cell_vert"], C["N"], F["dof_xyz"], owner)
        srp, scol, sval = P.struct_prolongation(elem, 2, C["dof_lat"], F["dof_lat"])
        assert np.array_equal(rp, srp) and np.array_equal(col, scol)
        assert np.max(np.abs(val - sval)) < 1e-14


def test_create_rejects_bad_level_counts():
    """pmg_create checks its arguments before it looks for a device."""
    import ctypes
    import parmoon_b200 as P
    h = ctypes.c_void_p()
    p = P.default_params()
    for n in (0, -1, 17):
        assert P.lib().pmg_create(ctypes.byref(h), n, ctypes.byref(p)) == P.ERR_ARG


def test_output_arrays_are_checked_and_used_in_place():
    """The binding's caller-provided outputs (get_rhs/get_solution out=, solve
    inplace=True: page-locked host buffers) are used as given, and anything
    the C ABI could not write into directly is rejected before any call."""
    import parmoon_b200 as P
    a = np.zeros(10)
    assert P._out_f64(a, 10) is a
    assert P._out_f64(None, 7).shape == (7,)
    for bad in (np.zeros(9), np.zeros(10, dtype=np.float32), np.zeros(20)[::2], [0.0] * 10):
        with pytest.raises(ValueError):
            P._out_f64(bad, 10)


def test_params_mirror_matches_the_library():
    """The ctypes Params mirror has the library's sizeof(pmg_params): a field
    added on one side only (pmg_default_params writes the whole struct) shows
    up here rather than as a corrupted stack."""
    import ctypes
    import parmoon_b200 as P
    assert P.lib().pmg_params_size() == ctypes.sizeof(P.Params)


def test_host_builders_reject_bad_input():
    """The host set-up helpers (no GPU) return status codes for bad input:
    unknown elements, empty meshes, dofs or parents out of range, a jittered
    N_Q1 mesh, and the N_Q1 space where only the cell-averaged transfer
    applies."""
    import parmoon_b200 as P
    lib = P.lib()
    i = ctypes.c_int
    nc, N, nl = i(), i(), i()
    assert lib.pmg_struct_sizes(99, 4, ctypes.byref(nc), ctypes.byref(N), ctypes.byref(nl)) == P.ERR_ARG
    assert lib.pmg_struct_sizes(P.Q1_HEX, 0, ctypes.byref(nc), ctypes.byref(N), ctypes.byref(nl)) == P.ERR_ARG
    with pytest.raises(P.PmgError) as e:
        P.struct_level(P.NQ1_HEX, 2, jitter=0.1)
    assert e.value.code == P.ERR_UNSUPPORTED
    # a pattern whose cells name a dof beyond the level
    ed = np.array([0, 1, 2, 7], dtype=np.int32)
    rp = np.zeros(5, dtype=np.int32)
    rc = lib.pmg_struct_csr(1, 4, ed.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), 4, 4,
                            rp.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), None)
    assert rc == P.ERR_ARG
    # N_Q1 has no node lattice: the lattice transfer refuses it
    L = P.struct_level(P.NQ1_HEX, 2)
    assert L["colors"] is None
    with pytest.raises(P.PmgError) as e:
        P.struct_prolongation(P.NQ1_HEX, 1, np.zeros(1, dtype=np.int32), np.zeros(1, dtype=np.int32))
    assert e.value.code == P.ERR_UNSUPPORTED
    # a fine cell whose parent is not a coarse cell
    C, F = P.struct_level(P.Q1_HEX, 1), P.struct_level(P.Q1_HEX, 2)
    parents = P.struct_parents(2)
    parents[3] = 5
    with pytest.raises(P.PmgError) as e:
        P.cell_prolongation(P.Q1_HEX, C["elem_dof"], C["cell_vert"], C["N"], P.Q1_HEX, F["elem_dof"],
                            F["cell_vert"], parents, F["N"])
    assert e.value.code == P.ERR_ARG
