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
