"""GPU parity: libpmg_b200 (through its C ABI) against the oracle and the
reference's golden dumps.

Bars: matrix entries |a-b| <= 1e-12 max(|b|, max|row of b|) and rhs within
1e-12 relative (FP64); SpMV / SSOR / transfers within 1e-12 relative;
solves reach |r|/|r0| <= 1e-10 in FP64 true residual; solutions compared with
a reference or dense solution are solved to |r| <= 1e-14 |r0| and match it
within 1e-10 relative L2."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

ASM_CASES = [
    ("q1_laplace", 1, 1, dict(kind=1, eps=1.0), True),
    ("q1_supg", 1, 2, dict(kind=0, eps=1e-3, b=(1, .5, .25), f=1.0), True),
    ("q2_supg", 2, 2, dict(kind=0, eps=1e-6, b=(1, .5, .25), f=1.0), True),
    ("q2_galerkin", 2, 1, dict(kind=0, eps=1e-2, b=(1, .5, .25), f=1.0), True),
    ("p2tet_supg", 12, 2, dict(kind=0, eps=1e-3, b=(1, .5, .25), f=1.0), False),
    ("p1tet_laplace", 11, 1, dict(kind=1, eps=1.0), False),
]


def n_levels(g):
    return sum(1 for k in g.files if k.endswith("_rowptr"))


def entry_rel_err(e, ref, rowptr):
    rowmax = np.maximum.reduceat(np.abs(ref), rowptr[:-1])
    scale = np.maximum(np.abs(ref), np.repeat(rowmax, np.diff(rowptr)))
    scale[scale == 0] = 1.0
    return float(np.max(np.abs(e - ref) / scale))


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("name,elem,form,ck,brick", ASM_CASES)
def test_assembly_on_reference_mesh_matches_reference(pmg, name, elem, form, ck, brick):
    """Drop-in use: the reference's own element->dof map, vertex coordinates and
    CSR pattern go in; the device fills Entries and rhs like Assemble3D."""
    g = golden(name)
    nl = n_levels(g)
    h = pmg.Handle(nl)
    h.set_coefficients(pmg.coeff(**ck))
    for l in range(nl):
        p = f"L{l}_"
        Na = int(g[p + "active_bound"])
        h.set_level_csr(l, g[p + "rowptr"], g[p + "kcol"], Na)
        h.set_level_mesh(l, elem, g[p + "elem_dof"], g[p + "cell_vert"], brick=brick)
        h.set_dirichlet_values(l, g[p + "rhs"][Na:])
        e, r = h.assemble(l, form)
        assert entry_rel_err(e, g[p + "entries"], g[p + "rowptr"]) < 1e-12
        assert rel(r, g[p + "rhs"]) < 1e-12
    h.close()


STRUCT_CASES = [
    (1, 6, 1, dict(kind=1, eps=1.0), 0.0),
    (1, 6, 2, dict(kind=0, eps=1e-3, b=(1, .5, .25), f=1.0), 0.0),
    (1, 5, 3, dict(kind=0, eps=1.0, f=2.0), 0.0),
    (2, 4, 2, dict(kind=0, eps=1e-6, b=(1, .5, .25), f=1.0), 0.0),
    (2, 4, 1, dict(kind=4, eps=1e-4, f=1.0, t=0.3), 0.0),
    (11, 4, 1, dict(kind=1, eps=1.0), 0.2),
    (12, 3, 2, dict(kind=0, eps=1e-3, b=(1, .5, .25), f=1.0), 0.2),
    (12, 3, 1, "lognormal", 0.2),
    (1, 4, 2, "curl", 0.0),
]


def fourier_modes(seed, n=8, kind="lognormal"):
    rng = np.random.default_rng(seed)
    m = np.zeros((n, 8))
    m[:, 0:3] = rng.integers(-3, 4, size=(n, 3))
    m[:, 3] = rng.normal(size=n) / np.sqrt(n)
    m[:, 4] = rng.uniform(0, 2 * np.pi, n)
    m[:, 5:8] = rng.normal(size=(n, 3))
    return m


@pytest.mark.parametrize("elem,n,form,ck,jitter", STRUCT_CASES)
def test_assembly_structured_matches_oracle(pmg, oracle, elem, n, form, ck, jitter):
    L = pmg.struct_level(elem, n, jitter=jitter, seed=7)
    if ck == "lognormal":
        modes = fourier_modes(3)
        ck_p, ck_o = dict(kind=2, eps=1.0, f=1.0, modes=modes), dict(kind=2, eps=1.0, f=1.0, modes=modes)
    elif ck == "curl":
        modes = fourier_modes(5)
        ck_p = dict(kind=3, eps=1e-3, b=(2.0, 0, 0), f=1.0, modes=modes)
        ck_o = dict(ck_p)
    else:
        ck_p = ck_o = ck
    dv = np.sin(L["dof_xyz"][L["active_bound"]:, 0] + 0.5)
    h = pmg.Handle(1)
    h.set_coefficients(pmg.coeff(**ck_p))
    h.set_level_csr(0, L["rowptr"], L["kcol"], L["active_bound"])
    h.set_level_mesh(0, elem, L["elem_dof"], L["cell_vert"], brick=(elem in (1, 2) and jitter == 0))
    h.set_dirichlet_values(0, dv)
    e, r = h.assemble(0, form)
    quad = {1: 2, 2: 3, 11: 104, 12: 111}[elem]
    eo, ro = oracle.assemble(elem, L["elem_dof"], L["cell_vert"], L["N"], L["active_bound"], L["rowptr"], L["kcol"],
                             form, oracle.make_coeff(**ck_o), quad=quad, dir_values=dv)
    assert entry_rel_err(e, eo, L["rowptr"]) < 1e-12
    assert rel(r, ro) < 1e-12
    h.close()


def make_hierarchy(pmg, elem, n_fine, nl, form, ck, prec=0, dirichlet=None, **prm):
    levels = pmg.struct_hierarchy(elem, n_fine, nl)
    params = pmg.default_params(precision=prec, **prm)
    h = pmg.Handle(nl, params)
    h.set_coefficients(pmg.coeff(**ck))
    pmg.load_hierarchy(h, levels, dirichlet=dirichlet)
    h.assemble(-1, form, copy_out=False)
    return h, levels


def test_kernels_match_oracle(pmg, oracle):
    h, levels = make_hierarchy(pmg, 2, 8, 2, 2, dict(kind=0, eps=1e-3, b=(1, .5, .25), f=1.0))
    F = levels[-1]
    A = h.get_matrix(1)
    rng = np.random.default_rng(0)
    x = rng.standard_normal(F["N"])
    b = rng.standard_normal(F["N"])
    y_ref = oracle.spmv(F["rowptr"], F["kcol"], A, x)
    assert rel(h.matvec(1, x), y_ref) < 1e-12
    r, nrm = h.defect(1, x, b)
    assert rel(r, b - y_ref) < 1e-12 and abs(nrm - np.linalg.norm(b - y_ref)) < 1e-10 * nrm
    # one multicolour SSOR step (forward + backward over the lattice colours)
    xs = h.ssor(1, b, x, 1)
    xo = oracle.ssor(F["rowptr"], F["kcol"], A, b, x, F["active_bound"], colors=F["colors"], n_colors=F["n_colors"])
    assert rel(xs, xo) < 1e-11
    # transfers
    C = levels[0]
    c = rng.standard_normal(C["N"])
    rp, col, val = F["P"]
    assert rel(h.prolongate(1, c), oracle.spmv(rp, col, val, c)) < 1e-13
    rr = np.zeros(C["N"])
    np.add.at(rr, col, val * np.repeat(x, np.diff(rp)))
    assert rel(h.restrict(1, x), rr) < 1e-13
    h.close()


@pytest.mark.parametrize("prec", [0, 1])
def test_solve_q1_laplace(pmg, oracle, prec):
    """C1's method at 16^3: FGMRES + V-cycle SSOR(2,2), 1e-10 in the FP64 true residual."""
    d = lambda x, y, z: np.sin(np.pi * x) * np.sin(np.pi * y) * np.sin(np.pi * z)
    h, levels = make_hierarchy(pmg, 1, 16, 3, 1, dict(kind=1, eps=1.0), prec=prec, dirichlet=d)
    _, st, rc = h.solve()
    assert rc == 0 and st.rel_res <= 1e-10, (rc, st.rel_res)
    x = h.get_solution()
    F = levels[-1]
    A = h.get_matrix(2)
    b = h.get_rhs(2)
    r = b - oracle.spmv(F["rowptr"], F["kcol"], A, x)
    assert np.linalg.norm(r) <= 1.01e-10 * st.res0
    # discretisation check: nodal error of Q1 / Gauss2 at h = 1/16 against the manufactured solution
    ex = d(*F["dof_xyz"].T)
    assert np.max(np.abs(x - ex)) < 1e-2
    h.close()


@pytest.mark.parametrize("prec", [0, 1])
def test_solve_q2_supg_matches_direct(pmg, prec):
    """C2's discretisation at 4^3 cells (Q2, SUPG, eps=1e-6): the iterate agrees with a dense solve."""
    dirichlet = lambda x, y, z: (np.abs(x) < 1e-12).astype(float)
    h, levels = make_hierarchy(pmg, 2, 4, 3, 2, dict(kind=0, eps=1e-6, b=(1, .5, .25), f=1.0), prec=prec,
                               dirichlet=dirichlet)
    h.set_params(pmg.default_params(precision=prec, lin_red=1e-14, lin_maxit=300, restart=30))
    _, st, rc = h.solve()
    assert rc == 0 and st.rel_res <= 1e-13
    x = h.get_solution()
    F = levels[-1]
    A = h.get_matrix(2)
    b = h.get_rhs(2)
    D = np.zeros((F["N"], F["N"]))
    rows = np.repeat(np.arange(F["N"]), np.diff(F["rowptr"]))
    D[rows, F["kcol"]] = A
    xd = np.linalg.solve(D, b)
    assert np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-10
    h.close()


@pytest.mark.parametrize("name,elem,form,ck", [("q1_laplace", 1, 1, dict(kind=1, eps=1.0)),
                                               ("q2_supg", 2, 2, dict(kind=0, eps=1e-6, b=(1, .5, .25), f=1.0))])
@pytest.mark.parametrize("prec", [0, 1])
def test_solve_on_reference_hierarchy_matches_reference_solution(pmg, name, elem, form, ck, prec):
    """Drop-in solve on the reference's own levels (its CSR, numbering, and its
    Prolongate expressed as a CSR P) reproduces the reference's solution to
    1e-10 relative L2: both solve to |r| <= 1e-14 |r0| (FP64 V-cycle, and FP32
    V-cycle inside FP64 FGMRES)."""
    g = golden(name)
    nl = n_levels(g)
    p = 2 if elem == 2 else 1
    h = pmg.Handle(nl, pmg.default_params(lin_red=1e-14, lin_maxit=300, restart=30, precision=prec))
    h.set_coefficients(pmg.coeff(**ck))
    lat = []
    for l in range(nl):
        q = f"L{l}_"
        Na = int(g[q + "active_bound"])
        h.set_level_csr(l, g[q + "rowptr"], g[q + "kcol"], Na)
        h.set_level_mesh(l, elem, g[q + "elem_dof"], g[q + "cell_vert"], brick=True)
        h.set_dirichlet_values(l, g[q + "rhs"][Na:])
        nc = 2 ** (l + 1)
        ijk = np.rint(g[q + "dof_xyz"].reshape(-1, 3) * (p * nc)).astype(np.int64)
        lat.append((ijk[:, 0] + (p * nc + 1) * (ijk[:, 1] + (p * nc + 1) * ijk[:, 2])).astype(np.int32))
        if l > 0:
            rp, col, val = pmg.struct_prolongation(elem, nc // 2, lat[l - 1], lat[l])
            h.set_transfer(l, rp, col, val, int(g[f"L{l-1}_N"]))
    h.assemble(-1, form, copy_out=False)
    _, st, rc = h.solve()
    assert rc == 0
    x = h.get_solution()
    ref = g["solution"]
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 1e-10
    h.close()


def test_errors_are_status_codes(pmg):
    """No exit(): a missing coupling, non-finite coefficients and out-of-order calls return codes."""
    L = pmg.struct_level(1, 3)
    h = pmg.Handle(1)
    # drop one off-diagonal column from an active row -> the slot map finds the hole
    rp, kc = L["rowptr"].copy(), L["kcol"].copy()
    r = 0
    drop = rp[r] + (1 if kc[rp[r]] == r else 0)
    kc2 = np.delete(kc, drop)
    rp2 = rp.copy()
    rp2[r + 1:] -= 1
    h.set_level_csr(0, rp2, kc2, L["active_bound"])
    with pytest.raises(pmg.PmgError) as ei:
        h.set_level_mesh(0, 1, L["elem_dof"], L["cell_vert"], brick=True)
    assert ei.value.code == -6
    with pytest.raises(pmg.PmgError) as ei:
        h.set_coefficients(pmg.coeff(kind=0, eps=float("nan")))
    assert ei.value.code == -7
    h2 = pmg.Handle(1)
    h2.set_level_csr(0, L["rowptr"], L["kcol"], L["active_bound"])
    _, st, rc = h2.solve(raise_on_error=False)
    assert rc == -3
    h.close()
    h2.close()
