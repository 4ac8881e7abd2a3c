"""Learned stencil smoother on the device: inference and gradients against the
FP64 oracle (with the same BF16-rounded weights), and what training buys.

Tolerances: the device keeps weights in BF16 and accumulates in FP32, the
oracle computes in FP64 from the same BF16 values: stencils within 1e-4 and
gradients within 1e-3 (relative, L2 over the parameter vector)."""
import numpy as np
import pytest

from oracle import learned_oracle as LO

pytestmark = pytest.mark.gpu


def problem(pmg, n, levels=2, seed=5):
    from parmoon_b200 import learned as PL
    return PL.make_problem(seed, n, levels)


def test_learned_stencil_matches_oracle(pmg):
    h, lv = problem(pmg, 4)
    F = lv[-1]
    rng = np.random.default_rng(2)
    w = (rng.standard_normal(LO.n_params()) * 0.05).astype(np.float32)
    h.set_learned_weights(w)
    W = h.learned_stencil(1)
    A = h.get_matrix(1)
    Wo = LO.stencil(LO.bf16_round(w), F["n"] + 1, F["rowptr"], F["kcol"], A, F["active_bound"], F["dof_lat"])
    Wo = Wo.reshape(27, -1)
    assert np.max(np.abs(W - Wo)) <= 1e-4 * np.max(np.abs(Wo))
    h.close()


def test_learned_gradient_matches_oracle(pmg):
    import torch
    h, lv = problem(pmg, 4)
    F = lv[-1]
    N, Na = F["N"], F["active_bound"]
    rng = np.random.default_rng(3)
    w = (rng.standard_normal(LO.n_params()) * 0.05).astype(np.float32)
    h.set_learned_weights(w)
    A = h.get_matrix(1)
    e = rng.standard_normal(N)
    e[Na:] = 0
    r = h.matvec(1, e)
    r[Na:] = 0
    E = torch.from_numpy(e[None].copy()).cuda()
    R = torch.from_numpy(r[None].copy()).cuda()
    loss, g = h.learned_train_step(1, E.data_ptr(), R.data_ptr(), 1, 0.0, want_grad=True)
    lo, go = LO.loss_and_grad(LO.bf16_round(w), F["n"] + 1, F["rowptr"], F["kcol"], A, Na, F["dof_lat"], e, r)
    assert abs(loss - lo) <= 1e-4 * lo
    assert np.linalg.norm(g - go) <= 1e-3 * np.linalg.norm(go), np.linalg.norm(g - go) / np.linalg.norm(go)
    h.close()


def test_training_gain_and_guarded_solve(pmg):
    """Training on plain-GMG error samples lowers the held-out loss; the learned-smoother
    solve (with its SSOR guard) reaches 1e-10 in the FP64 residual."""
    from parmoon_b200 import learned as PL
    w0 = PL.init_weights(0)
    probs = []
    for s in range(3):
        h, lv = PL.make_problem(100 + s, 16, 3)
        E, R = PL.generate_pairs(h, lv, 2, 3, s)
        probs.append((h, lv, E, R))
    hv, lvv = PL.make_problem(999, 16, 3)
    Ev, Rv = PL.generate_pairs(hv, lvv, 2, 3, 99)

    def held_out(w):
        hv.set_learned_weights(w)
        loss, _ = hv.learned_train_step(2, Ev.data_ptr(), Rv.data_ptr(), Ev.shape[0], 0.0)
        return loss

    l0 = held_out(w0)
    w, hist = PL.train(probs, w0, 150, lr=2e-3, batch=3)
    l1 = held_out(w)
    assert l1 < 0.9 * l0, (l0, l1)
    # solve the held-out problem with the trained smoother
    hv.set_params(pmg.default_params(precision=pmg.PREC_FP32, smoother=pmg.SMOOTHER_LEARNED))
    hv.set_learned_weights(w)
    _, st, rc = hv.solve()
    assert rc == 0 and st.rel_res <= 1e-10
    assert st.smoother_used in (pmg.SMOOTHER_LEARNED, pmg.SMOOTHER_SSOR)
    for h, *_ in probs:
        h.close()
    hv.close()


def test_data_parallel_step_equals_device_step(pmg):
    """One rank of the data-parallel loop (gradient to the host, mean over
    ranks, pmg_learned_apply_gradient) reproduces the fused device step
    (pmg_learned_train_step with lr > 0) exactly."""
    from parmoon_b200 import learned as PL
    w0 = PL.init_weights(1)
    h, lv = PL.make_problem(7, 8, 2)
    E, R = PL.generate_pairs(h, lv, 2, 3, 1)
    probs = [(h, lv, E, R)]
    wa, ha = PL.train(probs, w0, 12, lr=2e-3, batch=2, seed=3)
    h2, lv2 = PL.make_problem(7, 8, 2)
    wb, hb = PL.train_dp_device([(h2, lv2, E, R)], w0, 12, lr=2e-3, batch=2, seed=3)
    assert np.array_equal(wa, wb)
    assert np.allclose(ha, hb, rtol=1e-6)
    h.close()
    h2.close()
