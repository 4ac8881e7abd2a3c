"""Time-dependent CD3D (TSystemTCD3D's theta scheme) on the device.

1. The reference's own recorded run (ReadIn/tcd3d_GMG.out: amc.h, Q1 on 16^3
   cells, Crank-Nicolson, tau = 0.1082532, default quadrature Gauss3): the
   device path reproduces the printed L2 errors at every step to all 7
   printed digits, and the H1-semi errors of the compiled reference.
2. A SUPG step with the rotating convection field of the TCD3D benchmark
   configuration against the oracle's dense theta-scheme step (1e-10; solved
   to |r| <= 1e-14 |r0|)."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

THETA_CN = (0.5, 0.5, 0.5, 0.5)


def amc_exact(x, y, z, t):
    return np.exp(-0.1 * t) * np.sin(np.pi * x) * np.cos(np.pi * y) * np.cos(np.pi * z)


def test_tcd_amc_reproduces_recorded_log(pmg, oracle):
    g = golden("tcd3d_amc")
    log = g["recorded_log"]
    tau = 0.1082532
    levels = pmg.struct_hierarchy(pmg.Q1_HEX, 16, 3)
    F = levels[-1]
    params = pmg.default_params(problem_linear=0, lin_red=1e-12, restart=30)
    h = pmg.Handle(3, params)

    def set_bc(t):
        for l, L in enumerate(levels):
            xyz = L["dof_xyz"][L["active_bound"]:]
            h.set_dirichlet_values(l, amc_exact(xyz[:, 0], xyz[:, 1], xyz[:, 2], t))

    h.set_coefficients(pmg.coeff(kind=pmg.COEF_AMC, t=0.0))
    pmg.load_hierarchy(h, levels)
    set_bc(0.0)
    u = amc_exact(*F["dof_xyz"].T, 0.0)  # Interpolate(InitialCondition)
    err = oracle.errors(1, F["elem_dof"], F["cell_vert"], u, 3, 1, 0.0)
    assert f"{err[0]:.6e}" == f"{log[0, 1]:.6e}"
    h.assemble(-1, pmg.FORM_MASS, copy_out=False)  # AssembleMRhs
    t = 0.0
    for step in range(3):
        t += tau
        h.set_coefficients(pmg.coeff(kind=pmg.COEF_AMC, t=t))
        set_bc(t)
        h.assemble(-1, pmg.FORM_GALERKIN, copy_out=False)  # AssembleARhs
        h.tcd_system(tau, THETA_CN, u_old=u if step == 0 else None)
        _, st, rc = h.solve()
        assert rc == 0
        h.tcd_restore()
        u = h.get_solution()
        err = oracle.errors(1, F["elem_dof"], F["cell_vert"], u, 3, 1, t)
        row = np.argmin(np.abs(log[:, 0] - t))
        assert abs(log[row, 0] - t) < 1e-6
        assert f"{err[0]:.6e}" == f"{log[row, 1]:.6e}", (step, err[0], log[row, 1])
        # H1-semi against the compiled reference (the recorded log's H1 column came from an older build)
        assert abs(err[1] - g["h1"][step + 1]) <= 1e-9 * g["h1"][step + 1]
    h.close()


def csr_dense(rp, kc, a, N):
    D = np.zeros((N, N))
    D[np.repeat(np.arange(N), np.diff(rp)), kc] = a
    return D


def test_tcd_supg_step_matches_oracle(pmg, oracle):
    """One Crank-Nicolson step with SUPG mass and stiffness, rotating b (the TCD3D config's field)."""
    levels = pmg.struct_hierarchy(pmg.Q1_HEX, 8, 2)
    F = levels[-1]
    N, Na = F["N"], F["active_bound"]
    tau, t0 = 1e-3, 0.25
    h = pmg.Handle(2, pmg.default_params(lin_red=1e-14, lin_maxit=300, restart=30))
    ck = lambda t: dict(kind=pmg.COEF_ROTATING, eps=1e-4, f=1.0, t=t)
    pmg.load_hierarchy(h, levels)
    h.set_coefficients(pmg.coeff(**ck(t0)))
    h.assemble(-1, pmg.FORM_MASS_SUPG, copy_out=False)
    M = h.get_matrix(1, which=1)
    f_old = h.get_rhs(1)
    h.set_coefficients(pmg.coeff(**ck(t0 + tau)))
    h.assemble(-1, pmg.FORM_SUPG, copy_out=False)
    A = h.get_matrix(1)
    f_new = h.get_rhs(1)
    rng = np.random.default_rng(3)
    u_old = rng.standard_normal(N)
    u_old[Na:] = 0.0
    B = h.tcd_system(tau, THETA_CN, u_old=u_old)
    _, st, rc = h.solve()
    assert rc == 0
    x = h.get_solution()
    h.tcd_restore()
    assert np.array_equal(h.get_matrix(1), A)  # RestoreMassMat puts the stiffness matrix back
    # oracle: the same forms and the theta-scheme right-hand side, dense solve
    quad = 2
    Mo, fo_old = oracle.assemble(1, F["elem_dof"], F["cell_vert"], N, Na, F["rowptr"], F["kcol"], oracle.FORM_MASS_SUPG,
                                 oracle.make_coeff(kind=4, eps=1e-4, f=1.0, t=t0), quad=quad,
                                 dir_values=np.zeros(N - Na))
    Ao, fo_new = oracle.assemble(1, F["elem_dof"], F["cell_vert"], N, Na, F["rowptr"], F["kcol"], oracle.FORM_SUPG,
                                 oracle.make_coeff(kind=4, eps=1e-4, f=1.0, t=t0 + tau), quad=quad,
                                 dir_values=np.zeros(N - Na))
    scale = lambda e, r: np.max(np.abs(e - r)) / np.max(np.abs(r))
    assert scale(M, Mo) < 1e-12 and scale(A, Ao) < 1e-12
    Md, Ad = csr_dense(F["rowptr"], F["kcol"], Mo, N), csr_dense(F["rowptr"], F["kcol"], Ao, N)
    Bo = tau * 0.5 * fo_old + tau * 0.5 * fo_new + (Md - tau * 0.5 * Ad) @ u_old
    Bo[Na:] = fo_new[Na:]
    assert np.max(np.abs(B - Bo)) <= 1e-12 * np.max(np.abs(Bo))
    S = Md + tau * 0.5 * Ad
    S[Na:, :] = Md[Na:, :]
    xo = np.linalg.solve(S, Bo)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-10
    h.close()
