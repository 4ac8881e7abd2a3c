"""The oracle (C restatement in oracle/cd3d_oracle.c) against the reference's
own outputs: golden fixtures dumped by the compiled reference
(tests/golden/make_golden.py) and the reference's recorded run log."""
import numpy as np
import pytest

from conftest import golden

# (fixture, element, form, coefficient kwargs, quadrature rule)
ASM_CASES = [
    ("q1_laplace", 1, 1, dict(kind=1, eps=1.0), 2),
    ("q1_supg", 1, 2, dict(kind=0, eps=1e-3, b=(1, .5, .25), f=1.0), 2),
    ("q2_supg", 2, 2, dict(kind=0, eps=1e-6, b=(1, .5, .25), f=1.0), 3),
    ("q2_galerkin", 2, 1, dict(kind=0, eps=1e-2, b=(1, .5, .25), f=1.0), 3),
    ("p2tet_supg", 12, 2, dict(kind=0, eps=1e-3, b=(1, .5, .25), f=1.0), 111),
    ("p1tet_laplace", 11, 1, dict(kind=1, eps=1.0), 104),
]


def n_levels(g):
    return sum(1 for k in g.files if k.endswith("_rowptr"))


def entry_rel_err(e, ref, rowptr):
    """|a-b| / max(|b|, max|row of b|): the entry criterion for cancelling couplings."""
    rowmax = np.maximum.reduceat(np.abs(ref), rowptr[:-1])
    scale = np.maximum(np.abs(ref), np.repeat(rowmax, np.diff(rowptr)))
    return float(np.max(np.abs(e - ref) / scale))


@pytest.mark.parametrize("name,elem,form,ck,quad", ASM_CASES)
def test_oracle_assembly_matches_reference(oracle, name, elem, form, ck, quad):
    g = golden(name)
    for l in range(n_levels(g)):
        p = f"L{l}_"
        N, Na = int(g[p + "N"]), int(g[p + "active_bound"])
        e, r = oracle.assemble(elem, g[p + "elem_dof"], g[p + "cell_vert"], N, Na, g[p + "rowptr"], g[p + "kcol"],
                               form, oracle.make_coeff(**ck), quad=quad, dir_values=g[p + "rhs"][Na:])
        assert entry_rel_err(e, g[p + "entries"], g[p + "rowptr"]) < 1e-12
        assert np.max(np.abs(r - g[p + "rhs"])) <= 1e-12 * max(1.0, np.max(np.abs(g[p + "rhs"])))


def lattice_index(xyz, n1):
    ijk = np.rint(np.asarray(xyz).reshape(-1, 3) * (n1 - 1)).astype(np.int64)
    return (ijk[:, 0] + n1 * (ijk[:, 1] + n1 * ijk[:, 2])).astype(np.int32)


@pytest.mark.parametrize("name,elem,p,n0", [("q1_laplace", 1, 1, 2), ("q2_supg", 2, 2, 2)])
def test_oracle_transfer_matches_reference(oracle, name, elem, p, n0):
    """Prolongate / DefectRestriction of the reference == interpolation P and P^T."""
    g = golden(name)
    for l in range(1, n_levels(g)):
        nc = n0 * 2 ** (l - 1)
        latc = lattice_index(g[f"L{l-1}_dof_xyz"], p * nc + 1)
        latf = lattice_index(g[f"L{l}_dof_xyz"], p * 2 * nc + 1)
        rp, col, val = oracle.prolongation(elem, nc, latc, latf)
        c = g[f"T{l}_coarse_in"]
        assert np.array_equal(oracle.spmv(rp, col, val, c), g[f"T{l}_prolongated"])
        d = g[f"T{l}_fine_in"]
        r = np.zeros(c.size)
        np.add.at(r, col, val * np.repeat(d, np.diff(rp)))
        assert np.max(np.abs(r - g[f"T{l}_restricted"])) < 1e-13


@pytest.mark.parametrize("name,elem", [("q1_laplace", 1), ("q2_galerkin", 2)])
def test_oracle_csr_matches_reference_pattern(oracle, name, elem):
    """The oracle's CSR builder reproduces TSquareStructure3D on the reference's own element->dof map."""
    g = golden(name)
    for l in range(n_levels(g)):
        p = f"L{l}_"
        N, Na = int(g[p + "N"]), int(g[p + "active_bound"])
        nloc = int(g[p + "n_loc"])
        rp, kc = oracle.csr(g[p + "elem_dof"], nloc, N, Na)
        assert np.array_equal(rp, g[p + "rowptr"])
        assert np.array_equal(kc, g[p + "kcol"])


@pytest.mark.parametrize("name", ["q1_laplace", "q1_supg", "q2_supg", "p2tet_supg"])
def test_oracle_solve_matches_reference_solution(oracle, name):
    """FGMRES + GMG (lexicographic SSOR as the reference) reaches the reference's
    solution to 1e-10 relative L2: both solves stop at |r| <= 1e-14 |r0| (the
    reference's run is in the fixture), near the FP64 rounding floor."""
    g = golden(name)
    levels = []
    for l in range(n_levels(g)):
        p = f"L{l}_"
        L = dict(N=int(g[p + "N"]), Na=int(g[p + "active_bound"]), rp=g[p + "rowptr"], kc=g[p + "kcol"],
                 a=g[p + "entries"])
        levels.append(L)
    # the oracle's own hierarchy needs P: use the interpolation on the reference dofs (hexahedra) or
    # a dense direct solve on the finest level (tetrahedra, whose red refinement is not Kuhn-nested)
    fine = levels[-1]
    if name.startswith("p2tet"):
        levels = [fine]
    else:
        elem, p_deg = (2, 2) if name.startswith("q2") else (1, 1)
        for l in range(1, len(levels)):
            nc = 2 ** l  # coarse_steps=1: level 0 has 2 cells per direction
            latc = lattice_index(g[f"L{l-1}_dof_xyz"], p_deg * nc + 1)
            latf = lattice_index(g[f"L{l}_dof_xyz"], p_deg * 2 * nc + 1)
            levels[l]["P"] = oracle.prolongation(elem, nc, latc, latf)
    rhs = g[f"L{n_levels(g)-1}_rhs"]
    sol0 = np.zeros(fine["N"])
    sol0[fine["Na"]:] = rhs[fine["Na"]:]
    sol, it, res, _ = oracle.fgmres_mg(levels, rhs, sol0=sol0, red=1e-14, coarse_direct=True, restart=30)
    assert it > 0
    ref = g["solution"]
    rel = np.linalg.norm(sol - ref) / np.linalg.norm(ref)
    assert rel < 1e-10, rel


def lattice_of(xyz, n1):
    """Lattice index i + n1 (j + n1 k) of points of the unit cube's n1^3 node lattice."""
    ijk = np.rint(np.asarray(xyz).reshape(-1, 3) * (n1 - 1)).astype(np.int64)
    return ijk[:, 0] + n1 * (ijk[:, 1] + n1 * ijk[:, 2])


def test_oracle_solves_c1_to_the_reference_solution(oracle):
    """The C1 configuration exactly (Poisson, Q1, 32^3 cells over 4 levels from
    4^3, Gauss2, sine right-hand side): the oracle's FGMRES + GMG, assembled on
    this library's lattice numbering, against the compiled reference's solution
    (fixture: its own mesh, numbering and solve to |r| <= 1e-14 |r0|), matched
    through the dof positions: 1e-10 relative L2."""
    import parmoon_b200 as P
    g = golden("c1_poisson_q1_32")
    levels = P.struct_hierarchy(1, 32, 4)
    co = oracle.make_coeff(kind=1, eps=1.0)
    olev = []
    for l, L in enumerate(levels):
        a, r = oracle.assemble(1, L["elem_dof"], L["cell_vert"], L["N"], L["active_bound"], L["rowptr"], L["kcol"],
                               1, co)
        d = dict(N=L["N"], Na=L["active_bound"], rp=L["rowptr"], kc=L["kcol"], a=a)
        if l > 0:
            d["P"] = L["P"]
        olev.append(d)
    F = levels[-1]
    sol0 = np.zeros(F["N"])
    sol0[F["active_bound"]:] = r[F["active_bound"]:]
    sol, it, res, _ = oracle.fgmres_mg(olev, r, sol0=sol0, red=1e-14, coarse_direct=True, restart=30)
    assert it > 0
    ours = lattice_of(F["dof_xyz"], 33)
    ref = np.empty(F["N"])
    ref[lattice_of(g["fine_dof_xyz"], 33)] = g["solution"]
    x = np.empty(F["N"])
    x[ours] = sol
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 1e-10


def test_reference_build_reproduces_recorded_log():
    """The compiled reference (amc.h, Q1 16^3, Crank-Nicolson) prints the same L2 errors as the
    reference's recorded ReadIn/tcd3d_GMG.out, to all 7 printed digits, at every step."""
    g = golden("tcd3d_amc")
    log = g["recorded_log"]
    for t, l2 in zip(g["times"], g["l2"]):
        row = np.argmin(np.abs(log[:, 0] - t))
        assert abs(log[row, 0] - t) < 1e-6
        assert abs(float(f"{l2:.6e}") - log[row, 1]) <= 1e-12


def test_oracle_vcycle_is_a_contracting_linear_operator(oracle):
    """The oracle's single V-cycle (the reference for tests/test_gpu_vcycle.py)
    is linear in its input and, on the SPD Q1 Laplace problem (16^3, 3
    levels), reduces the error of A e = v in the energy norm by at least half
    with SSOR(2,2) and the dense coarse solve."""
    import parmoon_b200 as P
    co = oracle.make_coeff(kind=1, eps=1.0)
    levels = P.struct_hierarchy(1, 16, 3)
    olev = []
    for l, L in enumerate(levels):
        a, _ = oracle.assemble(1, L["elem_dof"], L["cell_vert"], L["N"], L["active_bound"], L["rowptr"], L["kcol"],
                               1, co)
        d = dict(N=L["N"], Na=L["active_bound"], rp=L["rowptr"], kc=L["kcol"], a=a, colors=L["colors"],
                 n_colors=L["n_colors"])
        if l > 0:
            d["P"] = L["P"]
        olev.append(d)
    F = olev[-1]
    rng = np.random.default_rng(11)
    u, w = rng.standard_normal(F["N"]), rng.standard_normal(F["N"])
    zu, zw, zs = oracle.mg_apply(olev, u), oracle.mg_apply(olev, w), oracle.mg_apply(olev, 2.0 * u - 3.0 * w)
    assert np.max(np.abs(zs - (2.0 * zu - 3.0 * zw))) <= 1e-12 * np.max(np.abs(zs))
    e = np.zeros(F["N"])
    e[:F["Na"]] = rng.standard_normal(F["Na"])
    v = oracle.spmv(F["rp"], F["kc"], F["a"], e)
    err = e - oracle.mg_apply(olev, v)
    Aa = lambda x: oracle.spmv(F["rp"], F["kc"], F["a"], x)
    assert float(err @ Aa(err)) <= 0.25 * float(e @ Aa(e))


@pytest.mark.parametrize("k", range(5))
def test_oracle_smoother_variants_match_reference(oracle, k):
    """Jacobi (MGLevel3D.C:469-560), SOR (:280-361) and step-length control
    (MultiGrid3D.C:517-523, 655-663; MGLevel3D.C:908-961) in the oracle
    against the compiled reference's FGMRES + GMG on the q1_supg problem
    (3 levels, lexicographic smoothing, iterative SSOR coarse solve), both to
    1e-12: the same iteration count and the same solution to 1e-9 relative."""
    g, v = golden("q1_supg"), golden("q1_supg_smoothers")
    opt = dict(s.split("=") for s in v[f"V{k}_params"])
    levels = []
    for l in range(n_levels(g)):
        p = f"L{l}_"
        levels.append(dict(N=int(g[p + "N"]), Na=int(g[p + "active_bound"]), rp=g[p + "rowptr"], kc=g[p + "kcol"],
                           a=g[p + "entries"]))
    for l in range(1, len(levels)):
        nc = 2 ** l
        latc = lattice_index(g[f"L{l-1}_dof_xyz"], nc + 1)
        latf = lattice_index(g[f"L{l}_dof_xyz"], 2 * nc + 1)
        levels[l]["P"] = oracle.prolongation(1, nc, latc, latf)
    fine = levels[-1]
    rhs = g[f"L{len(levels)-1}_rhs"]
    sol0 = np.zeros(fine["N"])
    sol0[fine["Na"]:] = rhs[fine["Na"]:]
    sol, it, res, _ = oracle.fgmres_mg(levels, rhs, sol0=sol0, red=float(opt["red"]), restart=int(opt["restart"]),
                                       coarse_direct=False, coarse_smoother=3, omega=float(opt["omega"]),
                                       smoother=int(opt["smoother"]), slc_all=opt.get("slc_all") == "1",
                                       slc_fine=opt.get("slc_fine") == "1", reference_restart_rule=True)
    assert it == int(v[f"V{k}_iterations"]), (it, v[f"V{k}_iterations"])
    ref = v[f"V{k}_solution"]
    assert np.linalg.norm(sol - ref) / np.linalg.norm(ref) < 1e-9
