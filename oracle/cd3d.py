"""ctypes front end of the C restatement in ``cd3d_oracle.c``.

Test infrastructure only: the tests, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` use it as the checker.  The product library
(``parmoon_b200``) never imports it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "cd3d_oracle.c")
LIB = os.path.join(HERE, "_build", "libcd3d_oracle.so")

Q1, Q2, P1, P2 = 1, 2, 11, 12
NQ1 = 3  # the non-conforming N_Q1 hexahedron (face-midpoint values)
FORM_GALERKIN, FORM_SUPG, FORM_MASS, FORM_MASS_SUPG, FORM_STIFF_SUPG = 1, 2, 3, 4, 5
COEF_CONST, COEF_SINE_RHS, COEF_LOGNORMAL, COEF_CURL_FOURIER, COEF_ROTATING, COEF_AMC = range(6)

_i = ctypes.c_int
_d = ctypes.c_double
_p = ctypes.c_void_p


class Coeff(ctypes.Structure):
    _fields_ = [("kind", _i), ("eps", _d), ("b", _d * 3), ("c", _d), ("f", _d), ("t", _d),
                ("n_modes", _i), ("modes", _p)]


class Level(ctypes.Structure):
    _fields_ = [("N", _i), ("Na", _i), ("rp", _p), ("kc", _p), ("a", _p), ("n_colors", _i),
                ("colors", _p), ("prp", _p), ("pcol", _p), ("pval", _p)]


class MGParams(ctypes.Structure):
    _fields_ = [("pre", _i), ("post", _i), ("coarse_maxit", _i), ("coarse_red", _d),
                ("omega", _d), ("damp", _d), ("coarse_direct", _i), ("smoother", _i), ("coarse_smoother", _i),
                ("slc_all", _i), ("slc_fine", _i)]


def build(force=False):
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        os.makedirs(os.path.dirname(LIB), exist_ok=True)
        subprocess.check_call(["gcc", "-O2", "-shared", "-fPIC", SRC, "-lm", "-o", LIB])
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build())
        _lib.orc_fgmres_mg.restype = _i
        _lib.orc_defect.restype = _d
    return _lib


def _ptr(a):
    return a.ctypes.data_as(_p) if a is not None else None


def nloc_of(elem):
    return {Q1: 8, Q2: 27, NQ1: 6, P1: 4, P2: 10}[elem]


def default_quad(elem, linear=True):
    """Rule the reference picks with INTERNAL_PROBLEM_LINEAR=1 (linear) or 0."""
    if elem == Q1:
        return 2 if linear else 3
    if elem in (Q2, NQ1):
        return 3 if linear else 4
    if elem == P1:
        return 104 if linear else 111
    return 111


def make_coeff(kind=COEF_CONST, eps=1.0, b=(0, 0, 0), c=0.0, f=1.0, t=0.0, modes=None):
    co = Coeff()
    co.kind, co.eps, co.c, co.f, co.t = kind, eps, c, f, t
    for k in range(3):
        co.b[k] = b[k]
    if modes is not None:
        modes = np.ascontiguousarray(modes, dtype=np.float64)
        co.n_modes = modes.shape[0]
        co.modes = modes.ctypes.data_as(_p)
        co._keep = modes
    return co


def assemble(elem, elem_dof, cell_vert, N, active_bound, rowptr, kcol, form, coeff,
             quad=None, poly=None, delta0=1.0, dir_values=None):
    """TAssembleMat3D::Reset + Assemble3D restated; returns (entries, rhs)."""
    elem_dof = np.ascontiguousarray(elem_dof, dtype=np.int32)
    cell_vert = np.ascontiguousarray(cell_vert, dtype=np.float64)
    rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
    kcol = np.ascontiguousarray(kcol, dtype=np.int32)
    nloc = nloc_of(elem)
    n_cells = elem_dof.size // nloc
    if quad is None:
        quad = default_quad(elem)
    if poly is None:
        poly = 2 if elem in (Q2, P2) else 1
    entries = np.zeros(int(rowptr[N]), dtype=np.float64)
    rhs = np.zeros(N, dtype=np.float64)
    dv = None if dir_values is None else np.ascontiguousarray(dir_values, dtype=np.float64)
    rc = lib().orc_assemble(_i(elem), _i(n_cells), _ptr(elem_dof), _ptr(cell_vert), _i(N), _i(active_bound),
                            _ptr(rowptr), _ptr(kcol), _i(form), _i(quad), ctypes.byref(coeff), _i(poly),
                            _d(delta0), _ptr(dv), _ptr(entries), _ptr(rhs))
    if rc != 0:
        raise RuntimeError(f"orc_assemble failed: {rc}")
    return entries, rhs


def struct_mesh(elem, n, jitter=0.0, seed=0):
    """Structured unit-cube level: dict(elem_dof, cell_vert, dof_xyz, dof_lat, N, active_bound, n_cells)."""
    nc, N, nl = _i(), _i(), _i()
    lib().orc_struct_sizes(_i(elem), _i(n), ctypes.byref(nc), ctypes.byref(N), ctypes.byref(nl))
    ed = np.zeros(nc.value * nl.value, dtype=np.int32)
    cv = np.zeros(nc.value * 24, dtype=np.float64)
    xyz = np.zeros(N.value * 3, dtype=np.float64)
    lat = np.zeros(N.value, dtype=np.int32)
    ab = _i()
    lib().orc_build_struct(_i(elem), _i(n), _d(jitter), ctypes.c_ulonglong(seed), _ptr(ed), _ptr(cv),
                           _ptr(xyz), _ptr(lat), ctypes.byref(ab))
    return dict(elem=elem, n=n, elem_dof=ed, cell_vert=cv, dof_xyz=xyz, dof_lat=lat, N=N.value,
                active_bound=ab.value, n_cells=nc.value)


def csr(elem_dof, nloc, N, active_bound):
    elem_dof = np.ascontiguousarray(elem_dof, dtype=np.int32)
    n_cells = elem_dof.size // nloc
    rp = np.zeros(N + 1, dtype=np.int32)
    lib().orc_build_csr(_i(n_cells), _i(nloc), _ptr(elem_dof), _i(N), _i(active_bound), _ptr(rp), None)
    kc = np.zeros(int(rp[N]), dtype=np.int32)
    lib().orc_build_csr(_i(n_cells), _i(nloc), _ptr(elem_dof), _i(N), _i(active_bound), _ptr(rp), _ptr(kc))
    return rp, kc


def prolongation(elem, nc, lat_c, lat_f):
    lat_c = np.ascontiguousarray(lat_c, dtype=np.int32)
    lat_f = np.ascontiguousarray(lat_f, dtype=np.int32)
    Nf = lat_f.size
    rp = np.zeros(Nf + 1, dtype=np.int32)
    lib().orc_build_prolongation(_i(elem), _i(nc), _ptr(lat_c), _i(lat_c.size), _ptr(lat_f), _i(Nf), _ptr(rp), None, None)
    col = np.zeros(int(rp[Nf]), dtype=np.int32)
    val = np.zeros(int(rp[Nf]), dtype=np.float64)
    lib().orc_build_prolongation(_i(elem), _i(nc), _ptr(lat_c), _i(lat_c.size), _ptr(lat_f), _i(Nf), _ptr(rp),
                                 _ptr(col), _ptr(val))
    return rp, col, val


def lattice_colors(elem, n, dof_lat):
    dof_lat = np.ascontiguousarray(dof_lat, dtype=np.int32)
    colors = np.zeros(dof_lat.size, dtype=np.int32)
    nc = _i()
    lib().orc_lattice_colors(_i(elem), _i(n), _i(dof_lat.size), _ptr(dof_lat), _ptr(colors), ctypes.byref(nc))
    return colors, nc.value


def spmv(rp, kc, a, x):
    N = rp.size - 1
    y = np.zeros(N)
    lib().orc_spmv(_i(N), _ptr(rp), _ptr(kc), _ptr(a), _ptr(np.ascontiguousarray(x, dtype=np.float64)), _ptr(y))
    return y


def sor(rp, kc, a, f, x, active_bound, omega=1.0, colors=None, n_colors=0):
    x = np.array(x, dtype=np.float64)
    N = rp.size - 1
    lib().orc_sor(_i(N), _i(active_bound), _ptr(rp), _ptr(kc), _ptr(a), _ptr(np.ascontiguousarray(f, dtype=np.float64)),
                  _ptr(x), _d(omega), _i(n_colors), _ptr(colors))
    return x


def jacobi(rp, kc, a, f, x, active_bound, omega=1.0):
    x = np.array(x, dtype=np.float64)
    N = rp.size - 1
    lib().orc_jacobi(_i(N), _i(active_bound), _ptr(rp), _ptr(kc), _ptr(a),
                     _ptr(np.ascontiguousarray(f, dtype=np.float64)), _ptr(x), _d(omega))
    return x


def ssor(rp, kc, a, f, x, active_bound, omega=1.0, colors=None, n_colors=0):
    x = np.array(x, dtype=np.float64)
    N = rp.size - 1
    lib().orc_ssor(_i(N), _i(active_bound), _ptr(rp), _ptr(kc), _ptr(a), _ptr(np.ascontiguousarray(f, dtype=np.float64)),
                   _ptr(x), _d(omega), _i(n_colors), _ptr(colors))
    return x


def _levels(levels, keep):
    """ctypes array of orc_level for a list (coarse..fine) of dicts rp, kc, a, N, Na,
    [colors, n_colors], [P=(rp,col,val)]; the arrays it points to are kept in `keep`."""
    arr = (Level * len(levels))()
    for i, L in enumerate(levels):
        arr[i].N, arr[i].Na = L["N"], L["Na"]
        for name in ("rp", "kc", "a"):
            keep.append(L[name])
        arr[i].rp, arr[i].kc, arr[i].a = _ptr(L["rp"]), _ptr(L["kc"]), _ptr(L["a"])
        if L.get("colors") is not None:
            arr[i].colors, arr[i].n_colors = _ptr(L["colors"]), L["n_colors"]
            keep.append(L["colors"])
        if L.get("P") is not None:
            prp, pcol, pval = L["P"]
            arr[i].prp, arr[i].pcol, arr[i].pval = _ptr(prp), _ptr(pcol), _ptr(pval)
            keep += [prp, pcol, pval]
    return arr


def mg_apply(levels, v, pre=2, post=2, coarse_maxit=10, coarse_red=0.1, omega=1.0, damp=1.0, coarse_direct=True,
             smoother=3, coarse_smoother=3, slc_all=False, slc_fine=False):
    """z = MG(v): one V-cycle from zero with the Dirichlet part of v (MultiGridScaIte.C:89-130).
    smoother / coarse_smoother: 1 Jacobi, 2 SOR, 3 SSOR; slc_*: step-length control."""
    keep = []
    arr = _levels(levels, keep)
    mp = MGParams(pre, post, coarse_maxit, coarse_red, omega, damp, int(coarse_direct), smoother, coarse_smoother,
                  int(slc_all), int(slc_fine))
    v = np.ascontiguousarray(v, dtype=np.float64)
    z = np.zeros(levels[-1]["N"])
    lib().orc_mg_apply(_i(len(levels)), arr, ctypes.byref(mp), _ptr(v), _ptr(z))
    return z


def fgmres_mg(levels, rhs, sol0=None, pre=2, post=2, coarse_maxit=10, coarse_red=0.1, omega=1.0, damp=1.0,
              coarse_direct=False, red=1e-10, res_min=0.0, maxit=1000, restart=20, div=1e10,
              reference_restart_rule=False, smoother=3, coarse_smoother=3, slc_all=False, slc_fine=False):
    """levels: list (coarse..fine) of dicts rp, kc, a, N, Na, [colors, n_colors], [P=(rp,col,val)]."""
    keep = []
    arr = (Level * len(levels))()
    for i, L in enumerate(levels):
        arr[i].N, arr[i].Na = L["N"], L["Na"]
        for name in ("rp", "kc", "a"):
            keep.append(L[name])
        arr[i].rp, arr[i].kc, arr[i].a = _ptr(L["rp"]), _ptr(L["kc"]), _ptr(L["a"])
        if L.get("colors") is not None:
            arr[i].colors, arr[i].n_colors = _ptr(L["colors"]), L["n_colors"]
            keep.append(L["colors"])
        if L.get("P") is not None:
            prp, pcol, pval = L["P"]
            arr[i].prp, arr[i].pcol, arr[i].pval = _ptr(prp), _ptr(pcol), _ptr(pval)
            keep += [prp, pcol, pval]
    mp = MGParams(pre, post, coarse_maxit, coarse_red, omega, damp, int(coarse_direct), smoother, coarse_smoother,
                  int(slc_all), int(slc_fine))
    N = levels[-1]["N"]
    sol = np.zeros(N) if sol0 is None else np.array(sol0, dtype=np.float64)
    rhs = np.ascontiguousarray(rhs, dtype=np.float64)
    hist = np.zeros(maxit + 1)
    res = _d()
    it = lib().orc_fgmres_mg(_i(len(levels)), arr, ctypes.byref(mp), _ptr(rhs), _ptr(sol), _d(red), _d(res_min),
                             _i(maxit), _i(restart), _d(div), _i(int(reference_restart_rule)), _ptr(hist),
                             ctypes.byref(res))
    return sol, it, res.value, hist


def errors(elem, elem_dof, cell_vert, sol, quad, exact_kind, t=0.0):
    """(L2, H1-semi) errors of a finite-element function (GetErrors + L2H1Errors restated)."""
    elem_dof = np.ascontiguousarray(elem_dof, dtype=np.int32)
    out = np.zeros(2)
    rc = lib().orc_errors(_i(elem), _i(elem_dof.size // nloc_of(elem)), _ptr(elem_dof),
                          _ptr(np.ascontiguousarray(cell_vert, dtype=np.float64)),
                          _ptr(np.ascontiguousarray(sol, dtype=np.float64)), _i(quad), _i(exact_kind), _d(t), _ptr(out))
    if rc != 0:
        raise RuntimeError("orc_errors failed")
    return out


def cell_transfer(mode, c_elem, c_elem_dof, c_cell_vert, n_coarse, f_elem, f_elem_dof, f_cell_vert, f_parent,
                  n_fine, vec):
    """Prolongate (mode 0: coarse -> fine) or DefectRestriction (mode 1: fine -> coarse)
    restated operationally for any pair of spaces on nested meshes (cell averaging)."""
    ced = np.ascontiguousarray(c_elem_dof, dtype=np.int32)
    fed = np.ascontiguousarray(f_elem_dof, dtype=np.int32)
    ccv = np.ascontiguousarray(c_cell_vert, dtype=np.float64)
    fcv = np.ascontiguousarray(f_cell_vert, dtype=np.float64)
    par = np.ascontiguousarray(f_parent, dtype=np.int32)
    v = np.ascontiguousarray(vec, dtype=np.float64)
    out = np.zeros(n_fine if mode == 0 else n_coarse)
    rc = lib().orc_cell_transfer(_i(mode), _i(c_elem), _i(ced.size // nloc_of(c_elem)), _ptr(ced), _ptr(ccv),
                                 _i(n_coarse), _i(f_elem), _i(fed.size // nloc_of(f_elem)), _ptr(fed), _ptr(fcv),
                                 _ptr(par), _i(n_fine), _ptr(v), _ptr(out))
    if rc != 0:
        raise RuntimeError(f"orc_cell_transfer failed: {rc}")
    return out
