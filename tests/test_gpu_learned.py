"""Learned stencil smoother on the device: inference and gradients against the
FP64 oracle (with the same BF16-rounded weights and BF16-rounded layer
inputs), and what training buys.

Tolerances: the device accumulates in FP32 on the tensor cores, the oracle in
FP64.  A hidden activation whose FP32 and FP64 values round to different BF16
neighbours differs by one BF16 unit (2^-8 relative); that changes the 27 x 32
outputs it feeds by |w| 2^-8 |a|, about 1e-4 of their size, and such flips are
rare (the FP32 accumulation error is ~1e-6 of a BF16 unit's width).  So the
stencils agree within 2e-3 of max|W| everywhere and within 1e-5 for the
median entry; the loss and the gradient within 1e-3 (relative; L2 over the
parameter vector for the gradient)."""
import numpy as np
import pytest

from oracle import learned_oracle as LO

pytestmark = pytest.mark.gpu


def problem(pmg, n, levels=2, seed=5):
    from parmoon_b200 import learned as PL
    return PL.make_problem(seed, n, levels)


@pytest.mark.parametrize("n", [4, 20])
def test_learned_stencil_matches_oracle(pmg, n):
    """The tensor-core forward on lattices of 5^3 (one partial brick) and 21^3
    nodes (bricks of 16 x 8 x 2 nodes cut by the lattice's edge in every
    direction)."""
    h, lv = problem(pmg, n)
    F = lv[-1]
    rng = np.random.default_rng(2)
    w = (rng.standard_normal(LO.n_params()) * 0.05).astype(np.float32)
    h.set_learned_weights(w)
    W = h.learned_stencil(1)
    A = h.get_matrix(1)
    Wo = LO.stencil(LO.bf16_round(w), F["n"] + 1, F["rowptr"], F["kcol"], A, F["active_bound"], F["dof_lat"])
    Wo = Wo.reshape(27, -1)
    err = np.abs(W - Wo)
    scale = np.max(np.abs(Wo))
    assert np.max(err) <= 2e-3 * scale, np.max(err) / scale
    assert np.median(err) <= 1e-5 * scale, np.median(err) / scale
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
    assert abs(loss - lo) <= 1e-3 * lo, abs(loss - lo) / lo
    assert np.linalg.norm(g - go) <= 1e-3 * np.linalg.norm(go), np.linalg.norm(g - go) / np.linalg.norm(go)
    h.close()


def test_training_gain_and_guard(pmg):
    """What training buys, and what the guard does with it.

    1. Training on plain-GMG error samples lowers the held-out loss.
    2. Measured in the solve itself, with the learned smoother in every cycle
       (guard off): the trained stencils contract the FP64 residual per
       V-cycle faster than the untrained network, which starts as damped
       Jacobi (W = 0.7 / a_ii).
    3. With the guard on, the learned smoother is kept exactly when its
       measured per-cycle contraction is no worse than the plain SSOR cycles';
       otherwise SSOR takes over.  Either way the solve reaches 1e-10 in the
       FP64 residual.
    Whether the trained smoother beats SSOR is measured, not assumed: the
    C4 evaluation (parmoon_b200/learned.py c4) records it per held-out seed."""
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

    def solve(weights, **prm):
        hv.set_params(pmg.default_params(precision=pmg.PREC_FP32, lin_maxit=300, **prm))
        if weights is not None:
            hv.set_learned_weights(weights)
        _, st, rc = hv.solve()
        return st, rc

    st_untrained, rc_untrained = solve(w0, smoother=pmg.SMOOTHER_LEARNED, learned_guard_off=1)
    st_trained, rc_trained = solve(w, smoother=pmg.SMOOTHER_LEARNED, learned_guard_off=1)
    assert rc_trained == 0 and st_trained.rel_res <= 1e-10
    assert st_trained.learned_cycles == st_trained.iterations
    assert rc_untrained != 0 or st_trained.mean_contraction < st_untrained.mean_contraction, \
        (st_trained.mean_contraction, st_untrained.mean_contraction)
    st_g, rc_g = solve(w, smoother=pmg.SMOOTHER_LEARNED)
    assert rc_g == 0 and st_g.rel_res <= 1e-10
    assert st_g.rho_plain > 0
    if st_g.smoother_used == pmg.SMOOTHER_LEARNED:
        assert st_g.rho_learned <= st_g.rho_plain and st_g.learned_cycles == st_g.iterations - 2
    else:
        assert st_g.smoother_used == pmg.SMOOTHER_SSOR
        assert st_g.rho_learned > st_g.rho_plain and st_g.learned_cycles <= st_g.iterations - 2
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
