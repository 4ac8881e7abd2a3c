"""The solve does not depend on the dof numbering: a random renumbering of the
finest level's active dofs (rows, columns, element maps, colours, the
prolongation's fine rows; Dirichlet dofs stay last) gives the same FGMRES
iteration count (+-1) and the renumbered solution within 1e-8 relative.

A random numbering of the 24^3 Q2 level (103,823 active dofs) puts columns
up to the level size away from their row, so the solve copy of the finest
matrix holds slices whose column deltas do not fit 16 bits and are read as
32-bit columns (the lattice-ordered levels of the other tests fit 16 bits
everywhere); the test checks that such rows exist.
Both solves do the same arithmetic up to the order of partial sums inside a
row (Gauss-Seidel within a colour does not depend on the order of its rows)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _permute_csr(rp, kc, val, p_row, p_col, n_rows):
    """CSR with row i renamed p_row[i] and columns renamed by p_col (None: kept); columns sorted."""
    rows = p_row[np.repeat(np.arange(len(rp) - 1), np.diff(rp))]
    cols = kc if p_col is None else p_col[kc]
    order = np.lexsort((cols, rows))
    nrp = np.zeros(n_rows + 1, dtype=np.int32)
    nrp[1:] = np.cumsum(np.bincount(rows, minlength=n_rows))
    return nrp, cols[order].astype(np.int32), None if val is None else val[order]


def permute_finest(levels, seed):
    L = dict(levels[-1])
    N, Na = L["N"], L["active_bound"]
    p = np.arange(N)
    p[:Na] = np.random.default_rng(seed).permutation(Na)  # new number of old dof i
    inv = np.empty(N, dtype=np.int64)
    inv[p] = np.arange(N)
    L["rowptr"], L["kcol"], _ = _permute_csr(L["rowptr"], L["kcol"], None, p, p, N)
    L["elem_dof"] = p[L["elem_dof"]].astype(np.int32)
    L["colors"] = np.ascontiguousarray(L["colors"][inv])
    L["dof_xyz"] = np.ascontiguousarray(L["dof_xyz"][inv])
    prp, pcol, pval = L["P"]
    L["P"] = _permute_csr(prp, pcol, pval, p, None, N)
    return levels[:-1] + [L], p


@pytest.mark.parametrize("prec", [0, 1])
def test_solve_independent_of_numbering(pmg, prec):
    ck = dict(kind=0, eps=1e-3, b=(1, .5, .25), f=1.0)
    dirichlet = lambda x, y, z: (np.abs(x) < 1e-12).astype(float)
    levels = pmg.struct_hierarchy(2, 24, 4)

    def run(lv):
        h = pmg.Handle(4, pmg.default_params(precision=prec))
        h.set_coefficients(pmg.coeff(**ck))
        pmg.load_hierarchy(h, lv, dirichlet=dirichlet)
        h.assemble(-1, pmg.FORM_SUPG, copy_out=False)
        _, st, rc = h.solve()
        x = h.get_solution()
        h.close()
        return rc, st, x

    rc0, st0, x0 = run(levels)
    plev, p = permute_finest(levels, 3)
    F = plev[-1]
    rows = np.repeat(np.arange(F["N"]), np.diff(F["rowptr"]))
    active = (rows < F["active_bound"]) & (F["kcol"] < F["active_bound"])
    assert np.max(np.abs(F["kcol"][active] - rows[active])) > 32767  # rows that need 32-bit columns
    rc1, st1, x1 = run(plev)
    assert rc0 == 0 and rc1 == 0 and st0.rel_res <= 1e-10 and st1.rel_res <= 1e-10
    assert abs(st0.iterations - st1.iterations) <= 1, (st0.iterations, st1.iterations)
    assert np.linalg.norm(x1[p] - x0) <= 1e-8 * np.linalg.norm(x0)
