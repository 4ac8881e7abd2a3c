"""The FP64 restatement of the learned stencil smoother (oracle/learned_oracle.py)
against finite differences: the learned smoother has no reference
counterpart, so its oracle is pinned by the mathematics of its own loss."""
import numpy as np

from oracle import cd3d as O
from oracle import learned_oracle as LO


def small_problem(n=3, seed=0):
    m = O.struct_mesh(O.Q1, n)
    rp, kc = O.csr(m["elem_dof"], 8, m["N"], m["active_bound"])
    rng = np.random.default_rng(seed)
    modes = np.zeros((2, 8))
    modes[:, 0:3] = [[1, 0, 1], [0, 1, 1]]
    modes[:, 3] = [0.7, -0.4]
    modes[:, 4] = rng.uniform(0, 6, 2)
    modes[:, 5:8] = rng.normal(size=(2, 3))
    A, _ = O.assemble(O.Q1, m["elem_dof"], m["cell_vert"], m["N"], m["active_bound"], rp, kc, O.FORM_SUPG,
                      O.make_coeff(kind=O.COEF_CURL_FOURIER, eps=1e-3, b=(3.0, 0, 0), f=1.0, modes=modes), quad=2,
                      dir_values=np.zeros(m["N"] - m["active_bound"]))
    return m, rp, kc, A


def test_learned_oracle_gradient_matches_finite_differences():
    m, rp, kc, A = small_problem()
    N, Na, n1 = m["N"], m["active_bound"], 4
    rng = np.random.default_rng(1)
    theta = rng.standard_normal(LO.n_params()) * 0.05
    e = rng.standard_normal(N)
    e[Na:] = 0
    Ad = np.zeros((N, N))
    Ad[np.repeat(np.arange(N), np.diff(rp)), kc] = A
    r = Ad @ e
    loss, g = LO.loss_and_grad(theta, n1, rp, kc, A, Na, m["dof_lat"], e, r, act_bf16=False)
    for trial in range(4):
        d = rng.standard_normal(theta.size)
        h = 1e-6
        lp, _ = LO.loss_and_grad(theta + h * d, n1, rp, kc, A, Na, m["dof_lat"], e, r, act_bf16=False)
        lm, _ = LO.loss_and_grad(theta - h * d, n1, rp, kc, A, Na, m["dof_lat"], e, r, act_bf16=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g @ d) <= 1e-6 * max(1.0, abs(fd)), (trial, fd, g @ d)


def test_bf16_rounding_matches_definition():
    x = np.array([1.0, 1.00390625, 1.0 + 2 ** -9, -3.14159, 1e-8], dtype=np.float32)
    y = LO.bf16_round(x)
    # 8 significant bits: the rounding error is below 2^-9 relative
    assert np.all(np.abs(y - x) <= np.abs(x) * 2 ** -8)
    assert y[0] == 1.0
