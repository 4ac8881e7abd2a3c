"""parmoon_b200 -- B200 implementation of ParMooN's 3D scalar convection-
diffusion hot path (assembly + multigrid-preconditioned FGMRES), driven
through the C ABI of ``libpmg_b200.so`` (include/pmg_b200.h).

The Python layer is a thin ctypes binding used by the tests and the
benchmark; the C++ host binding with the reference class names lives in
``parmoon_b200/shim``.  There is no CPU fallback: every call runs the CUDA
library, and importing this package fails loudly if the library cannot be
loaded.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpmg_b200.so")

# ------------------------------------------------------------------ constants
OK = 0
ERR = {-1: "ARG", -2: "CUDA", -3: "STATE", -4: "NOT_CONVERGED", -5: "DIVERGED", -6: "SLOT",
       -7: "NONFINITE", -8: "SINGULAR", -9: "UNSUPPORTED"}
(ERR_ARG, ERR_CUDA, ERR_STATE, ERR_NOT_CONVERGED, ERR_DIVERGED, ERR_SLOT, ERR_NONFINITE, ERR_SINGULAR,
 ERR_UNSUPPORTED) = range(-1, -10, -1)
Q1_HEX, Q2_HEX, P1_TET, P2_TET = 1, 2, 11, 12
NQ1_HEX = 3  # non-conforming N_Q1 (levels of SC_MG_TYPE_SCALAR = 1)
NLOC = {Q1_HEX: 8, Q2_HEX: 27, NQ1_HEX: 6, P1_TET: 4, P2_TET: 10}
HEX_ELEMS = (Q1_HEX, Q2_HEX, NQ1_HEX)
FORM_GALERKIN, FORM_SUPG, FORM_MASS, FORM_MASS_SUPG, FORM_STIFF_SUPG = 1, 2, 3, 4, 5
COEF_CONST, COEF_SINE_RHS, COEF_LOGNORMAL, COEF_CURL_FOURIER, COEF_ROTATING, COEF_AMC, COEF_TABLE = range(7)
SMOOTHER_JACOBI, SMOOTHER_SOR, SMOOTHER_SSOR, SMOOTHER_LEARNED = 1, 2, 3, 30
COARSE_JACOBI, COARSE_SOR, COARSE_SSOR, COARSE_DIRECT = 1, 2, 3, 17
PREC_FP64, PREC_FP32 = 0, 1
QUAD_AUTO, QUAD_GAUSS2, QUAD_GAUSS3, QUAD_GAUSS4, QUAD_KEAST4, QUAD_KEAST5, QUAD_KEAST11 = 0, 2, 3, 4, 104, 105, 111

_i, _d, _p = ctypes.c_int, ctypes.c_double, ctypes.c_void_p


class Params(ctypes.Structure):
    _fields_ = [("smoother", _i), ("pre_smooth", _i), ("post_smooth", _i), ("coarse_smoother", _i),
                ("coarse_maxit", _i), ("coarse_red", _d), ("smooth_omega", _d), ("gmg_damp", _d),
                ("lin_red", _d), ("lin_res_min", _d), ("lin_maxit", _i), ("restart", _i), ("div_factor", _d),
                ("precision", _i), ("sdfem_type", _i), ("poly_degree", _i), ("delta0", _d),
                ("reference_restart_rule", _i), ("problem_linear", _i), ("learned_steps", _i),
                ("assembly_kernel", _i), ("slc_all", _i), ("slc_fine", _i), ("quad_rule", _i),
                ("learned_guard_off", _i), ("assembly_scatter", _i)]


class CoeffDesc(ctypes.Structure):
    _fields_ = [("kind", _i), ("eps", _d), ("b", _d * 3), ("c", _d), ("f", _d), ("t", _d), ("n_modes", _i),
                ("modes", _p)]


class SolveStats(ctypes.Structure):
    _fields_ = [("iterations", _i), ("res0", _d), ("res_final", _d), ("rel_res", _d), ("mean_contraction", _d),
                ("smoother_used", _i), ("seconds", _d), ("setup_seconds", _d), ("vcycle_seconds", _d),
                ("rho_plain", _d), ("rho_learned", _d), ("learned_cycles", _i)]


class PmgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"pmg error {code} ({ERR.get(code, '?')}): {msg}")
        self.code = code


_lib = None


def lib():
    """Load libpmg_b200.so (built in-tree by parmoon_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} missing: run `python -m parmoon_b200.build`")
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.pmg_last_error.restype = ctypes.c_char_p
    return _lib


def _check(rc):
    if rc != OK:
        raise PmgError(rc, lib().pmg_last_error().decode())
    return rc


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_p)


def _c_i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _c_f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _out_f64(out, n):
    """A caller-provided output array (contiguous float64 of length n, used in
    place), or a new one."""
    if out is None:
        return np.empty(n)
    if not (isinstance(out, np.ndarray) and out.dtype == np.float64 and out.flags.c_contiguous and out.size == n):
        raise ValueError("out must be a contiguous float64 array of the level's size")
    return out


def default_params(**kw):
    p = Params()
    if lib().pmg_params_size() != ctypes.sizeof(Params):
        raise RuntimeError(f"libpmg_b200 pmg_params is {lib().pmg_params_size()} bytes, the Params mirror "
                           f"{ctypes.sizeof(Params)}: the binding and the library are out of step")
    lib().pmg_default_params(ctypes.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def coeff(kind=COEF_CONST, eps=1.0, b=(0.0, 0.0, 0.0), c=0.0, f=1.0, t=0.0, modes=None):
    d = CoeffDesc()
    d.kind, d.eps, d.c, d.f, d.t = kind, eps, c, f, t
    for k in range(3):
        d.b[k] = b[k]
    if modes is not None:
        m = _c_f64(modes).reshape(-1, 8)
        d.n_modes, d.modes = m.shape[0], m.ctypes.data_as(_p)
        d._keep = m
    return d


class Handle:
    """One multigrid hierarchy on the current CUDA device (TSystemCD3D analogue)."""

    def __init__(self, n_levels, params=None):
        self.h = _p()
        self.params = params if params is not None else default_params()
        _check(lib().pmg_create(ctypes.byref(self.h), _i(n_levels), ctypes.byref(self.params)))
        self.n_levels = n_levels
        self.sizes = [None] * n_levels
        self._ncells = [0] * n_levels

    def close(self):
        if self.h:
            lib().pmg_destroy(self.h)
            self.h = _p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, params):
        self.params = params
        _check(lib().pmg_set_params(self.h, ctypes.byref(params)))

    def set_level_csr(self, level, rowptr, kcol, active_bound):
        rowptr, kcol = _c_i32(rowptr), _c_i32(kcol)
        n = rowptr.size - 1
        _check(lib().pmg_set_level_csr(self.h, _i(level), _i(n), _i(active_bound), _ptr(rowptr), _ptr(kcol)))
        self.sizes[level] = (n, int(rowptr[-1]), active_bound)

    def set_level_mesh(self, level, elem_type, elem_dof, cell_vert, brick=False):
        elem_dof, cell_vert = _c_i32(elem_dof), _c_f64(cell_vert)
        nloc = NLOC[elem_type]
        n_cells = elem_dof.size // nloc
        if cell_vert.size != n_cells * 24:
            raise ValueError("cell_vert must hold 8 vertex slots x 3 coordinates per cell")
        _check(lib().pmg_set_level_mesh(self.h, _i(level), _i(elem_type), _i(n_cells), _ptr(elem_dof),
                                        _ptr(cell_vert), _i(int(brick))))
        self._ncells[level] = n_cells

    def build_level_csr(self, level, elem_dof, nloc, n_rows, active_bound):
        """TSquareStructure3D + Sort on the device from the element->dof map; returns nnz."""
        ed = _c_i32(elem_dof)
        nnz = _i()
        _check(lib().pmg_build_level_csr(self.h, _i(level), _i(n_rows), _i(active_bound), _i(ed.size // nloc),
                                         _i(nloc), _ptr(ed), ctypes.byref(nnz)))
        self.sizes[level] = (n_rows, nnz.value, active_bound)
        return nnz.value

    def get_level_csr(self, level):
        n, nnz, _ = self.sizes[level]
        rp = np.empty(n + 1, dtype=np.int32)
        kc = np.empty(nnz, dtype=np.int32)
        _check(lib().pmg_get_level_csr(self.h, _i(level), _ptr(rp), _ptr(kc)))
        return rp, kc

    def build_transfer(self, level, f_dof_xyz, f_dof_cell):
        """The prolongation from level-1 built on the device (fine dof r in coarse cell f_dof_cell[r])."""
        xyz, fc = _c_f64(f_dof_xyz), _c_i32(f_dof_cell)
        _check(lib().pmg_build_transfer(self.h, _i(level), _i(fc.size), _ptr(xyz), _ptr(fc)))

    def get_transfer(self, level):
        n = self.sizes[level][0]
        rp = np.empty(n + 1, dtype=np.int32)
        _check(lib().pmg_get_transfer(self.h, _i(level), _ptr(rp), None, None))
        col = np.empty(int(rp[-1]), dtype=np.int32)
        val = np.empty(int(rp[-1]))
        _check(lib().pmg_get_transfer(self.h, _i(level), _ptr(rp), _ptr(col), _ptr(val)))
        return rp, col, val

    def set_row_colors(self, level, colors, n_colors):
        colors = _c_i32(colors)
        _check(lib().pmg_set_level_row_colors(self.h, _i(level), _i(n_colors), _ptr(colors)))

    def set_transfer(self, level, p_rowptr, p_col, p_val, n_coarse):
        p_rowptr, p_col, p_val = _c_i32(p_rowptr), _c_i32(p_col), _c_f64(p_val)
        _check(lib().pmg_set_transfer(self.h, _i(level), _i(p_rowptr.size - 1), _i(n_coarse), _ptr(p_rowptr),
                                      _ptr(p_col), _ptr(p_val)))

    def set_dirichlet_values(self, level, values):
        values = _c_f64(values)
        _check(lib().pmg_set_dirichlet_values(self.h, _i(level), _ptr(values)))

    def set_coefficients(self, desc):
        self._coef = desc
        _check(lib().pmg_set_coefficients(self.h, ctypes.byref(desc)))

    def quad_points(self, level):
        """Physical quadrature points of one level's assembly rule: [n_cells, nq, 3]."""
        nq = ctypes.c_int(0)
        _check(lib().pmg_quad_points(self.h, _i(level), ctypes.byref(nq), None))
        nc = self._ncells[level]
        xyz = np.empty((nc, nq.value, 3))
        _check(lib().pmg_quad_points(self.h, _i(level), ctypes.byref(nq), _ptr(xyz)))
        return xyz

    def set_coefficient_table(self, level, values):
        """values [n_cells, nq, 6]: eps, b1, b2, b3, c, f at each quadrature point (PMG_COEF_TABLE)."""
        v = np.ascontiguousarray(values, dtype=np.float64)
        _check(lib().pmg_set_coefficient_table(self.h, _i(level), _ptr(v)))

    def assemble(self, level, form, copy_out=True):
        """Assemble one level (level=-1: all); returns (entries, rhs) host copies if copy_out."""
        if level >= 0 and copy_out:
            n, nnz, _ = self.sizes[level]
            e = np.empty(nnz)
            r = np.empty(n)
            _check(lib().pmg_assemble(self.h, _i(level), _i(form), _ptr(e), _ptr(r)))
            return e, r
        _check(lib().pmg_assemble(self.h, _i(level), _i(form), None, None))
        return None

    def get_matrix(self, level, which=0):
        e = np.empty(self.sizes[level][1])
        _check(lib().pmg_get_matrix(self.h, _i(level), _i(which), _ptr(e)))
        return e

    def set_matrix(self, level, entries, which=0):
        entries = _c_f64(entries)
        _check(lib().pmg_set_matrix(self.h, _i(level), _i(which), _ptr(entries)))

    def get_rhs(self, level, out=None):
        """Right-hand side of a level; `out` (contiguous float64, e.g. page-locked) receives it if given."""
        r = _out_f64(out, self.sizes[level][0])
        _check(lib().pmg_get_rhs(self.h, _i(level), _ptr(r)))
        return r

    def matvec(self, level, x):
        x = _c_f64(x)
        y = np.empty(self.sizes[level][0])
        _check(lib().pmg_matvec(self.h, _i(level), _ptr(x), _ptr(y)))
        return y

    def defect(self, level, x, b):
        x, b = _c_f64(x), _c_f64(b)
        r = np.empty(self.sizes[level][0])
        nrm = _d()
        _check(lib().pmg_defect(self.h, _i(level), _ptr(x), _ptr(b), _ptr(r), ctypes.byref(nrm)))
        return r, nrm.value

    def ssor(self, level, rhs, sol, n_sweeps=1):
        sol = np.array(sol, dtype=np.float64)
        rhs = _c_f64(rhs)
        _check(lib().pmg_ssor(self.h, _i(level), _ptr(rhs), _ptr(sol), _i(n_sweeps)))
        return sol

    def prolongate(self, level, coarse):
        coarse = _c_f64(coarse)
        fine = np.empty(self.sizes[level][0])
        _check(lib().pmg_prolongate(self.h, _i(level), _ptr(coarse), _ptr(fine)))
        return fine

    def restrict(self, level, fine):
        fine = _c_f64(fine)
        coarse = np.empty(self.sizes[level - 1][0])
        _check(lib().pmg_restrict(self.h, _i(level), _ptr(fine), _ptr(coarse)))
        return coarse

    def solve(self, sol=None, rhs=None, raise_on_error=True, inplace=False):
        """FGMRES + V-cycle on the finest level; returns (solution or None, stats, status).

        sol is the start vector; with inplace=True a contiguous float64 `sol`
        (e.g. page-locked) receives the solution itself instead of a copy."""
        st = SolveStats()
        if sol is not None:
            sol = _out_f64(sol, len(sol)) if inplace else np.array(sol, dtype=np.float64)
        rhs = None if rhs is None else _c_f64(rhs)
        rc = lib().pmg_solve(self.h, _ptr(sol), _ptr(rhs), ctypes.byref(st))
        if raise_on_error and rc != OK:
            _check(rc)
        return sol, st, rc

    def tcd_system(self, tau, theta, f_old=None, u_old=None):
        """TSystemTCD3D::AssembleSystMat on the device; returns the right-hand side B."""
        th = (ctypes.c_double * 4)(*theta)
        f_old = None if f_old is None else _c_f64(f_old)
        u_old = None if u_old is None else _c_f64(u_old)
        B = np.empty(self.sizes[-1][0])
        _check(lib().pmg_tcd_system(self.h, _d(tau), th, _ptr(f_old), _ptr(u_old), _ptr(B)))
        return B

    def tcd_restore(self):
        _check(lib().pmg_tcd_restore(self.h))

    # ---------------------------------------------------------------- learned smoother
    def set_lattice(self, level, n1, dof_lat):
        dof_lat = _c_i32(dof_lat)
        _check(lib().pmg_set_level_lattice(self.h, _i(level), _i(n1), _i(n1), _i(n1), _ptr(dof_lat)))

    def set_learned_weights(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        _check(lib().pmg_set_learned_weights(self.h, _ptr(w)))

    def get_learned_weights(self):
        w = np.empty(learned_num_params(), dtype=np.float32)
        _check(lib().pmg_get_learned_weights(self.h, _ptr(w)))
        return w

    def learned_stencil(self, level):
        W = np.empty(27 * self.sizes[level][0], dtype=np.float32)
        _check(lib().pmg_learned_stencil(self.h, _i(level), _ptr(W)))
        return W.reshape(27, -1)

    def learned_train_step(self, level, e_ptr, r_ptr, n_samples, lr, want_grad=False):
        """One device training step from device arrays (n_samples x N doubles); returns (loss, grad or None)."""
        loss = _d()
        g = np.empty(learned_num_params(), dtype=np.float32) if want_grad else None
        _check(lib().pmg_learned_train_step(self.h, _i(level), _i(n_samples), _p(e_ptr), _p(r_ptr),
                                            ctypes.c_float(lr), ctypes.byref(loss), _ptr(g)))
        return loss.value, g

    def learned_apply_gradient(self, grad, lr):
        """Adam step from a host gradient (data-parallel training applies the ranks' mean)."""
        g = np.ascontiguousarray(grad, dtype=np.float32)
        _check(lib().pmg_learned_apply_gradient(self.h, _ptr(g), ctypes.c_float(lr)))

    def vcycle(self, v_ptr, z_ptr):
        """z = MG(v) on device vectors of the finest level."""
        _check(lib().pmg_vcycle(self.h, _p(v_ptr), _p(z_ptr)))

    def set_halo(self, send_idx, recv_idx, send_buf_ptr, recv_buf_ptr):
        """Halo of a subdomain's finest level (pmg_set_halo): owned rows packed for the
        neighbours, ghost rows filled from them, device buffers of the transport."""
        si, ri = _c_i32(send_idx), _c_i32(recv_idx)
        _check(lib().pmg_set_halo(self.h, _i(si.size), _ptr(si), _i(ri.size), _ptr(ri), _p(send_buf_ptr),
                                  _p(recv_buf_ptr)))

    def solve_dd(self, comm, sol=None, rhs=None, raise_on_error=True):
        """FGMRES over the ranks' subdomains (pmg_solve_dd) with a pmg_comm structure."""
        st = SolveStats()
        sol = None if sol is None else np.array(sol, dtype=np.float64)
        rhs = None if rhs is None else _c_f64(rhs)
        rc = lib().pmg_solve_dd(self.h, ctypes.byref(comm), _ptr(sol), _ptr(rhs), ctypes.byref(st))
        if raise_on_error and rc != OK:
            _check(rc)
        return sol, st, rc

    def get_solution(self, out=None):
        x = _out_f64(out, self.sizes[-1][0])
        _check(lib().pmg_get_solution(self.h, _ptr(x)))
        return x

    def write_vtk(self, path, name="u", level=-1, values=None, region_ids=None):
        """Legacy VTK file of a level's function (TOutput3D::WriteVtk); values=None
        writes the device-resident solution of the finest level."""
        lv = self.n_levels - 1 if level < 0 else level
        v = None if values is None else _c_f64(values)
        r = None if region_ids is None else _c_i32(region_ids)
        _check(lib().pmg_write_vtk(self.h, _i(lv), _ptr(v), _ptr(r), str(path).encode(), name.encode()))

    def timings(self):
        a, s, k = _d(), _d(), _d()
        _check(lib().pmg_last_timings(self.h, ctypes.byref(a), ctypes.byref(s), ctypes.byref(k)))
        return a.value, s.value, k.value


def measure_peaks():
    """(FP64 FMA, FP64 DMMA, BF16 mma.sync) throughput in TFLOP/s on the current device."""
    v = [ctypes.c_double() for _ in range(3)]
    _check(lib().pmg_measure_peaks(*[ctypes.byref(x) for x in v]))
    return tuple(x.value for x in v)


def learned_num_params():
    n = _i()
    _check(lib().pmg_learned_num_params(ctypes.byref(n)))
    return n.value


# ------------------------------------------------------------------ structured set-up (host, C++)
def struct_level(elem, n, jitter=0.0, seed=0):
    nc, N, nl = _i(), _i(), _i()
    _check(lib().pmg_struct_sizes(_i(elem), _i(n), ctypes.byref(nc), ctypes.byref(N), ctypes.byref(nl)))
    ed = np.empty(nc.value * nl.value, dtype=np.int32)
    cv = np.empty(nc.value * 24, dtype=np.float64)
    xyz = np.empty(N.value * 3, dtype=np.float64)
    lat = np.empty(N.value, dtype=np.int32)
    ab = _i()
    _check(lib().pmg_struct_build(_i(elem), _i(n), _d(jitter), ctypes.c_ulonglong(seed), _ptr(ed), _ptr(cv),
                                  _ptr(xyz), _ptr(lat), ctypes.byref(ab)))
    rp = np.empty(N.value + 1, dtype=np.int32)
    _check(lib().pmg_struct_csr(_i(nc.value), _i(nl.value), _ptr(ed), N, ab, _ptr(rp), None))
    kc = np.empty(int(rp[-1]), dtype=np.int32)
    _check(lib().pmg_struct_csr(_i(nc.value), _i(nl.value), _ptr(ed), N, ab, _ptr(rp), _ptr(kc)))
    colors, ncol = None, _i(0)
    if elem != NQ1_HEX:  # N_Q1 has no node lattice: the library colours its rows greedily
        colors = np.empty(N.value, dtype=np.int32)
        _check(lib().pmg_struct_row_colors(_i(elem), _i(n), N, _ptr(lat), _ptr(colors), ctypes.byref(ncol)))
    return dict(elem=elem, n=n, elem_dof=ed, cell_vert=cv, dof_xyz=xyz.reshape(-1, 3), dof_lat=lat, N=N.value,
                active_bound=ab.value, n_cells=nc.value, rowptr=rp, kcol=kc, colors=colors, n_colors=ncol.value)


def struct_csr_of(elem_dof, nloc, n_dofs, active_bound):
    """TSquareStructure3D + Sort of any element->dof map (host builder): (rowptr, kcol)."""
    ed = _c_i32(elem_dof)
    rp = np.empty(n_dofs + 1, dtype=np.int32)
    _check(lib().pmg_struct_csr(_i(ed.size // nloc), _i(nloc), _ptr(ed), _i(n_dofs), _i(active_bound), _ptr(rp), None))
    kc = np.empty(int(rp[-1]), dtype=np.int32)
    _check(lib().pmg_struct_csr(_i(ed.size // nloc), _i(nloc), _ptr(ed), _i(n_dofs), _i(active_bound), _ptr(rp),
                                _ptr(kc)))
    return rp, kc


def struct_prolongation(elem, nc, lat_c, lat_f):
    lat_c, lat_f = _c_i32(lat_c), _c_i32(lat_f)
    rp = np.empty(lat_f.size + 1, dtype=np.int32)
    _check(lib().pmg_struct_prolongation(_i(elem), _i(nc), _ptr(lat_c), _i(lat_c.size), _ptr(lat_f), _i(lat_f.size),
                                         _ptr(rp), None, None))
    col = np.empty(int(rp[-1]), dtype=np.int32)
    val = np.empty(int(rp[-1]), dtype=np.float64)
    _check(lib().pmg_struct_prolongation(_i(elem), _i(nc), _ptr(lat_c), _i(lat_c.size), _ptr(lat_f), _i(lat_f.size),
                                         _ptr(rp), _ptr(col), _ptr(val)))
    return rp, col, val


def nested_prolongation(elem, c_elem_dof, c_cell_vert, n_coarse, f_dof_xyz, f_dof_cell):
    """Interpolation from a coarse level onto the dofs of a nested fine level of any mesh:
    f_dof_cell[r] names a coarse cell containing fine dof r.  Returns CSR (rp, col, val)."""
    ed, cv = _c_i32(c_elem_dof), _c_f64(c_cell_vert)
    xyz, fc = _c_f64(f_dof_xyz), _c_i32(f_dof_cell)
    nf = fc.size
    nloc = NLOC[elem]
    ncc = ed.size // nloc
    rp = np.empty(nf + 1, dtype=np.int32)
    args = (_i(elem), _i(ncc), _ptr(ed), _ptr(cv), _i(n_coarse), _i(nf), _ptr(xyz), _ptr(fc))
    _check(lib().pmg_nested_prolongation(*args, _ptr(rp), None, None))
    col = np.empty(int(rp[-1]), dtype=np.int32)
    val = np.empty(int(rp[-1]), dtype=np.float64)
    _check(lib().pmg_nested_prolongation(*args, _ptr(rp), _ptr(col), _ptr(val)))
    return rp, col, val


def cell_prolongation(c_elem, c_elem_dof, c_cell_vert, n_coarse, f_elem, f_elem_dof, f_cell_vert, f_parent, n_fine):
    """Prolongate's operator for any pair of spaces on nested meshes (cell averaging,
    pmg_cell_prolongation): CSR (rp, col, val) of n_fine x n_coarse."""
    ced, ccv = _c_i32(c_elem_dof), _c_f64(c_cell_vert)
    fed, fcv, par = _c_i32(f_elem_dof), _c_f64(f_cell_vert), _c_i32(f_parent)
    args = (_i(c_elem), _i(ced.size // NLOC[c_elem]), _ptr(ced), _ptr(ccv), _i(n_coarse), _i(f_elem),
            _i(fed.size // NLOC[f_elem]), _ptr(fed), _ptr(fcv), _ptr(par), _i(n_fine))
    rp = np.empty(n_fine + 1, dtype=np.int32)
    _check(lib().pmg_cell_prolongation(*args, _ptr(rp), None, None))
    col = np.empty(int(rp[-1]), dtype=np.int32)
    val = np.empty(int(rp[-1]), dtype=np.float64)
    _check(lib().pmg_cell_prolongation(*args, _ptr(rp), _ptr(col), _ptr(val)))
    return rp, col, val


def struct_parents(n):
    """Parent (in the (n/2)^3 mesh) of every cell of the structured n^3 hexahedral mesh."""
    i = np.arange(n ** 3)
    x, y, z = i % n, (i // n) % n, i // (n * n)
    m = n // 2
    return (x // 2 + m * (y // 2 + m * (z // 2))).astype(np.int32)


def mdml_hierarchy(elem, n_fine, n_geo):
    """The SC_MG_TYPE_SCALAR = 1 hierarchy of the unit cube (CD3D_ParMooN.C:258-313):
    N_Q1 on each of the n_geo meshes (n_fine >> (n_geo-1) .. n_fine cells per
    direction), then `elem` (Q1 or Q2) on the finest mesh as one more level.
    Transfers by cell averaging (Prolongate): N_Q1 -> N_Q1 between meshes, N_Q1 ->
    elem on the finest mesh."""
    levels = []
    for g in range(n_geo):
        n = n_fine >> (n_geo - 1 - g)
        L = struct_level(NQ1_HEX, n)
        if g > 0:
            C = levels[-1]
            L["P"] = cell_prolongation(NQ1_HEX, C["elem_dof"], C["cell_vert"], C["N"], NQ1_HEX, L["elem_dof"],
                                       L["cell_vert"], struct_parents(n), L["N"])
        levels.append(L)
    F = struct_level(elem, n_fine)
    C = levels[-1]
    F["P"] = cell_prolongation(NQ1_HEX, C["elem_dof"], C["cell_vert"], C["N"], elem, F["elem_dof"], F["cell_vert"],
                               np.arange(n_fine ** 3, dtype=np.int32), F["N"])
    levels.append(F)
    return levels


def struct_hierarchy(elem, n_fine, n_levels, jitter=0.0, seed=0):
    """Levels coarse..fine of the unit cube with n_fine cells per direction on the finest."""
    levels = []
    for l in range(n_levels):
        n = n_fine >> (n_levels - 1 - l)
        L = struct_level(elem, n, jitter=jitter if l == n_levels - 1 else 0.0, seed=seed)
        if l > 0 and elem == NQ1_HEX:  # no node lattice: Prolongate's cell average
            C = levels[-1]
            L["P"] = cell_prolongation(elem, C["elem_dof"], C["cell_vert"], C["N"], elem, L["elem_dof"],
                                       L["cell_vert"], struct_parents(n), L["N"])
        elif l > 0:
            L["P"] = struct_prolongation(elem, n // 2, levels[-1]["dof_lat"], L["dof_lat"])
        levels.append(L)
    return levels


def load_hierarchy(handle, levels, dirichlet=None, lattice_colors=True):
    """Hand a struct_hierarchy to a Handle: CSR, mesh, row colours, transfers, Dirichlet values.

    dirichlet: function (x, y, z) -> values on the Dirichlet dofs (default 0)."""
    for l, L in enumerate(levels):
        handle.set_level_csr(l, L["rowptr"], L["kcol"], L["active_bound"])
        handle.set_level_mesh(l, L["elem"], L["elem_dof"], L["cell_vert"], brick=L["elem"] in HEX_ELEMS)
        if lattice_colors and L.get("colors") is not None:
            handle.set_row_colors(l, L["colors"], L["n_colors"])
        if l > 0:
            rp, col, val = L["P"]
            handle.set_transfer(l, rp, col, val, levels[l - 1]["N"])
        xyz = L["dof_xyz"][L["active_bound"]:]
        vals = np.zeros(len(xyz)) if dirichlet is None else dirichlet(xyz[:, 0], xyz[:, 1], xyz[:, 2])
        handle.set_dirichlet_values(l, vals)
