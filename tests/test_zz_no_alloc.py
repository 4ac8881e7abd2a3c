"""pmg_defect_noalloc against pmg_defect.

The allocation-free entry point serves hosts that hand the library device
memory from their own pool and must not have it call cudaMalloc/cudaFree
during a call.  Here the caller's device buffers come from torch (standing
in for such a pool); the result must equal the allocating pmg_defect's
(r = b - A x and |r|) to 1e-12 relative, on two calls in a row (the shared
scratch array keeps the previous call's contents)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_defect_noalloc_matches_defect(pmg):
    import torch
    levels = pmg.struct_hierarchy(pmg.Q2_HEX, 8, 2)
    h = pmg.Handle(2)
    h.set_coefficients(pmg.coeff(kind=pmg.COEF_CONST, eps=1e-6, b=(1.0, 0.5, 0.25), f=1.0))
    pmg.load_hierarchy(h, levels)
    h.assemble(-1, pmg.FORM_SUPG, copy_out=False)
    N = levels[-1]["N"]
    rng = np.random.default_rng(11)
    lib = pmg.lib()
    for call in range(2):
        x = rng.standard_normal(N)
        b = rng.standard_normal(N) * (call + 1)
        r_ref, n_ref = h.defect(1, x, b)
        dx = torch.from_numpy(x).cuda()
        db = torch.from_numpy(b).cuda()
        dr = torch.full((N,), float("nan"), dtype=torch.float64, device="cuda")
        dn = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = lib.pmg_defect_noalloc(h.h, ctypes.c_int(1), ctypes.c_void_p(dx.data_ptr()),
                                    ctypes.c_void_p(db.data_ptr()), ctypes.c_void_p(dr.data_ptr()),
                                    ctypes.c_void_p(dn.data_ptr()))
        assert rc == 0, lib.pmg_last_error().decode()
        r = dr.cpu().numpy()
        nrm = float(dn.cpu().numpy()[0])
        assert np.max(np.abs(r - r_ref)) <= 1e-12 * np.max(np.abs(r_ref))
        assert abs(nrm - n_ref) <= 1e-12 * n_ref
    h.close()


@pytest.mark.parametrize("elem,n", [("Q1_HEX", 8), ("P1_TET", 6)])
def test_defect_noalloc_narrow_rows_match_oracle(pmg, oracle, elem, n):
    """Levels with short rows (Q1: 27 entries, 16 lanes per row; P1 on
    tetrahedra: ~15, 8 lanes per row) against the oracle's defect
    r = b - A x on the assembled matrix (1e-12 relative)."""
    import torch
    et = getattr(pmg, elem)
    levels = pmg.struct_hierarchy(et, n, 1, jitter=0.2 if elem == "P1_TET" else 0.0, seed=3)
    L = levels[-1]
    h = pmg.Handle(1)
    h.set_coefficients(pmg.coeff(kind=pmg.COEF_CONST, eps=1e-2, b=(1.0, -0.5, 0.25), f=1.0))
    pmg.load_hierarchy(h, levels)
    h.assemble(-1, pmg.FORM_SUPG, copy_out=False)
    A = h.get_matrix(0)
    N = L["N"]
    rng = np.random.default_rng(5)
    x, b = rng.standard_normal(N), rng.standard_normal(N)
    r_ref = b - oracle.spmv(L["rowptr"], L["kcol"], A, x)
    dx, db = torch.from_numpy(x).cuda(), torch.from_numpy(b).cuda()
    dr = torch.empty(N, dtype=torch.float64, device="cuda")
    dn = torch.empty(1, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    lib = pmg.lib()
    rc = lib.pmg_defect_noalloc(h.h, ctypes.c_int(0), ctypes.c_void_p(dx.data_ptr()), ctypes.c_void_p(db.data_ptr()),
                                ctypes.c_void_p(dr.data_ptr()), ctypes.c_void_p(dn.data_ptr()))
    assert rc == 0, lib.pmg_last_error().decode()
    r = dr.cpu().numpy()
    assert np.max(np.abs(r - r_ref)) <= 1e-12 * np.max(np.abs(r_ref))
    assert abs(float(dn.cpu().numpy()[0]) - np.linalg.norm(r_ref)) <= 1e-12 * np.linalg.norm(r_ref)
    h.close()


def test_defect_noalloc_before_assembly_is_a_state_error(pmg):
    import torch
    levels = pmg.struct_hierarchy(pmg.Q1_HEX, 4, 1)
    h = pmg.Handle(1)
    pmg.load_hierarchy(h, levels)
    N = levels[-1]["N"]
    d = torch.zeros(N + 1, dtype=torch.float64, device="cuda")
    rc = pmg.lib().pmg_defect_noalloc(h.h, ctypes.c_int(0), ctypes.c_void_p(d.data_ptr()),
                                      ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(d.data_ptr()),
                                      ctypes.c_void_p(d.data_ptr() + 8 * N))
    assert rc == pmg.ERR_STATE
    h.close()
