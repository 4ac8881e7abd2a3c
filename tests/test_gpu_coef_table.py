"""Tabulated coefficients (PMG_COEF_TABLE): a host CoeffFct3D callback
evaluated at the points pmg_quad_points returns gives the same matrix and rhs
as the device-evaluated field.  The quadrature points are checked against the
affine maps written out here (HexaAffin on vertices 0, 1, 3, 4; TetraAffin on
0..3), and the table values against the analytic field: matrices agree to
1e-12 relative (host and device libm may differ in the last bits)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def lognormal_field(modes, eps, X):
    m = modes.reshape(-1, 8)
    arg = 2 * np.pi * (X[..., None, 0] * m[:, 0] + X[..., None, 1] * m[:, 1] + X[..., None, 2] * m[:, 2]) + m[:, 4]
    return eps * np.exp((m[:, 3] * np.cos(arg)).sum(-1))


def ref_points(elem_hex, cell_vert, qx):
    """Physical points of reference points qx [nq, 3] in every cell."""
    v = cell_vert.reshape(-1, 8, 3)
    if elem_hex:
        J = np.stack([(v[:, 1] - v[:, 0]) / 2, (v[:, 3] - v[:, 0]) / 2, (v[:, 4] - v[:, 0]) / 2], axis=2)
        x0 = (v[:, 1] + v[:, 3] + v[:, 4] - v[:, 0]) / 2
    else:
        J = np.stack([v[:, 1] - v[:, 0], v[:, 2] - v[:, 0], v[:, 3] - v[:, 0]], axis=2)
        x0 = v[:, 0]
    return x0[:, None, :] + np.einsum("cdk,qk->cqd", J, qx)


@pytest.mark.parametrize("elem,form,jitter", [("Q2_HEX", "SUPG", 0.0), ("P2_TET", "GALERKIN", 0.2),
                                              ("Q1_HEX", "SUPG", 0.0)])
def test_table_matches_device_field(pmg, elem, form, jitter):
    from parmoon_b200.configs import lognormal_modes
    et = getattr(pmg, elem)
    fm = getattr(pmg, "FORM_" + form)
    modes = lognormal_modes(5)
    b = (1.0, 0.5, -0.25)
    levels = pmg.struct_hierarchy(et, 4, 2, jitter=jitter, seed=3)
    hd = pmg.Handle(2, pmg.default_params())
    hd.set_coefficients(pmg.coeff(kind=pmg.COEF_LOGNORMAL, eps=0.01, b=b, c=0.5, f=1.0, modes=modes))
    pmg.load_hierarchy(hd, levels)
    hd.assemble(-1, fm, copy_out=False)
    ht = pmg.Handle(2, pmg.default_params())
    ht.set_coefficients(pmg.coeff(kind=pmg.COEF_TABLE))
    pmg.load_hierarchy(ht, levels)
    with pytest.raises(pmg.PmgError):
        ht.assemble(-1, fm, copy_out=False)  # no table yet
    for lvl, L in enumerate(levels):
        X = ht.quad_points(lvl)
        nq = X.shape[1]
        # the points are the affine images of the rule's reference points: recover those
        # from the first cell and check every cell's map against them
        v = L["cell_vert"].reshape(-1, 8, 3)
        hexa = et in (pmg.Q1_HEX, pmg.Q2_HEX)
        if hexa:
            J0 = np.stack([(v[0, 1] - v[0, 0]) / 2, (v[0, 3] - v[0, 0]) / 2, (v[0, 4] - v[0, 0]) / 2], axis=1)
            x00 = (v[0, 1] + v[0, 3] + v[0, 4] - v[0, 0]) / 2
        else:
            J0 = np.stack([v[0, 1] - v[0, 0], v[0, 2] - v[0, 0], v[0, 3] - v[0, 0]], axis=1)
            x00 = v[0, 0]
        qx = np.linalg.solve(J0, (X[0] - x00).T).T
        assert np.allclose(ref_points(hexa, L["cell_vert"], qx), X, atol=1e-13)
        T = np.zeros(X.shape[:2] + (6,))
        T[..., 0] = lognormal_field(modes, 0.01, X)
        T[..., 1:4] = b
        T[..., 4] = 0.5
        T[..., 5] = 1.0
        ht.set_coefficient_table(lvl, T)
    ht.assemble(-1, fm, copy_out=False)
    for lvl in range(2):
        Ad, At = hd.get_matrix(lvl), ht.get_matrix(lvl)
        rd, rt = hd.get_rhs(lvl), ht.get_rhs(lvl)
        assert np.max(np.abs(Ad - At)) <= 1e-12 * np.max(np.abs(Ad))
        assert np.max(np.abs(rd - rt)) <= 1e-12 * np.max(np.abs(rd))
    hd.close()
    ht.close()
