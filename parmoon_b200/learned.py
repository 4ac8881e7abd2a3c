"""Training driver of the learned stencil smoother (config: Q1 CD3D with SUPG,
eps = 1e-3, convection b = curl of a seeded 8-mode Fourier vector potential
scaled so that max|b| lies in [1, 100]).

Residual / error pairs come from the plain GMG itself: starting from a random
error e_0 (zero on Dirichlet nodes) the plain V-cycle's error propagation
e_{k+1} = e_k - MG(A e_k) is run on the device and every (e_k, r_k = A e_k)
is a sample.  The network is trained on the device by the library's own
forward / backward / Adam kernels (pmg_learned_train_step); torch only holds
device buffers.
"""
import numpy as np

import parmoon_b200 as P
from parmoon_b200.configs import curl_modes

EPS = 1e-3


def init_weights(seed=0, omega=0.7):
    """He-initialised hidden layers; the output starts as damped Jacobi (W = omega / a_ii)."""
    rng = np.random.default_rng(seed)
    sizes = [(32, 27), (32, 32), (27, 32)]
    parts = []
    for li, (co, ci) in enumerate(sizes):
        fan_in = ci * 27
        scale = np.sqrt(2.0 / fan_in) if li < 2 else 1e-3
        parts.append((rng.standard_normal(co * ci * 27) * scale).astype(np.float32))
        b = np.zeros(co, dtype=np.float32)
        if li == 2:
            b[13] = omega
        parts.append(b)
    return np.concatenate(parts)


def make_problem(seed, n, levels, precision=P.PREC_FP32, weights=None, smoother=P.SMOOTHER_SSOR):
    """One CD3D SUPG problem on Q1 n^3 cells: (handle, hierarchy)."""
    modes, scale = curl_modes(seed)
    lv = P.struct_hierarchy(P.Q1_HEX, n, levels)
    h = P.Handle(levels, P.default_params(precision=precision, smoother=smoother))
    h.set_coefficients(P.coeff(kind=P.COEF_CURL_FOURIER, eps=EPS, b=(scale, 0, 0), f=1.0, modes=modes))
    P.load_hierarchy(h, lv)
    for l, L in enumerate(lv):
        h.set_lattice(l, L["n"] + 1, L["dof_lat"])
    h.assemble(-1, P.FORM_SUPG, copy_out=False)
    if weights is not None:
        h.set_learned_weights(weights)
    return h, lv


def generate_pairs(h, lv, n_start, n_steps, seed):
    """(E, R) torch tensors (n_start * n_steps x N, FP64, cuda) from the plain GMG error propagation."""
    import torch
    F = lv[-1]
    N, Na = F["N"], F["active_bound"]
    rng = np.random.default_rng(seed)
    E, R = [], []
    for _ in range(n_start):
        e = rng.standard_normal(N)
        e[Na:] = 0.0
        for _k in range(n_steps):
            r = h.matvec(len(lv) - 1, e)
            r[Na:] = 0.0
            E.append(e.copy()); R.append(r.copy())
            rd = torch.from_numpy(r).cuda()
            zd = torch.empty_like(rd)
            h.vcycle(rd.data_ptr(), zd.data_ptr())
            torch.cuda.synchronize()
            e = e - zd.cpu().numpy()
            e[Na:] = 0.0
            e /= max(np.linalg.norm(e), 1e-300)
    return torch.from_numpy(np.stack(E)).cuda(), torch.from_numpy(np.stack(R)).cuda()


def train(problems, weights, steps, lr=1e-3, batch=4, seed=0, log_every=0):
    """Adam on the device over (handle, E, R) problems; returns (weights, loss history)."""
    rng = np.random.default_rng(seed)
    for h, _, _, _ in problems:
        h.set_learned_weights(weights)
    hist = []
    cur = weights
    for it in range(steps):
        pi = rng.integers(len(problems))
        h, lv, E, R = problems[pi]
        h.set_learned_weights(cur)
        idx = rng.integers(E.shape[0] - batch + 1)
        loss, _ = h.learned_train_step(len(lv) - 1, E[idx].data_ptr(), R[idx].data_ptr(), batch, lr)
        cur = h.get_learned_weights()
        hist.append(loss)
        if log_every and it % log_every == 0:
            print(f"step {it} loss {loss:.4f}")
    return cur, hist


def allreduce_mean(g, dist=None):
    """Mean of a host array over the ranks of the default process group (identity without one).
    Runs on the backend's device: CPU tensors under gloo, CUDA tensors under nccl."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return np.asarray(g, dtype=np.float32)
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.from_numpy(np.ascontiguousarray(g, dtype=np.float32)).to(dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return (t / dist.get_world_size()).cpu().numpy()


def train_data_parallel(grad_fn, apply_fn, steps, dist=None):
    """Data-parallel training: every rank computes the gradient on its own
    problems (grad_fn(step) -> (loss, grad)), the gradients are averaged over
    the ranks (one all-reduce of the 57k-float gradient per step) and every
    rank applies the same update (apply_fn(mean_grad)), so the ranks' weights
    stay identical.  Returns the ranks' mean loss per step."""
    hist = []
    for it in range(steps):
        loss, g = grad_fn(it)
        g = allreduce_mean(g, dist)
        loss = float(allreduce_mean(np.array([loss], dtype=np.float32), dist)[0])
        apply_fn(g)
        hist.append(loss)
    return hist


def train_dp_device(problems, weights, steps, lr=1e-3, batch=4, seed=0, dist=None):
    """train() spread over the ranks of `dist`: each rank holds its own problems
    (handle, hierarchy, E, R) on its GPU; the mean gradient drives one Adam step
    per rank (pmg_learned_apply_gradient)."""
    rank = dist.get_rank() if dist is not None and dist.is_initialized() else 0
    rng = np.random.default_rng(seed + 1000 * rank)
    for h, _, _, _ in problems:
        h.set_learned_weights(weights)
    state = {"w": np.asarray(weights, dtype=np.float32)}

    def grad_fn(it):
        h, lv, E, R = problems[rng.integers(len(problems))]
        h.set_learned_weights(state["w"])
        idx = rng.integers(E.shape[0] - batch + 1)
        return h.learned_train_step(len(lv) - 1, E[idx].data_ptr(), R[idx].data_ptr(), batch, 0.0, want_grad=True)

    h0 = problems[0][0]

    def apply_fn(g):
        h0.learned_apply_gradient(g, lr)
        state["w"] = h0.get_learned_weights()

    hist = train_data_parallel(grad_fn, apply_fn, steps, dist)
    return state["w"], hist


def evaluate(weights, seeds, n=128, levels=5, learned_steps=(2, 4)):
    """Time to |r|/|r0| <= 1e-10 on held-out problems: plain FP64 GMG (SSOR), FP32 SSOR
    V-cycle and FP32 learned-smoother V-cycle (with its SSOR guard), all in FP64 FGMRES."""
    rows = []
    for s in seeds:
        h, lv = make_problem(s, n, levels, precision=P.PREC_FP64, weights=weights)
        out = {"seed": int(s), "n_dofs": int(lv[-1]["N"])}
        variants = [("fp64_ssor", dict(precision=P.PREC_FP64)), ("fp32_ssor", dict(precision=P.PREC_FP32))]
        for k in learned_steps:
            variants.append((f"fp32_learned_{k}", dict(precision=P.PREC_FP32, smoother=P.SMOOTHER_LEARNED,
                                                       learned_steps=k)))
        for name, prm in variants:
            h.set_params(P.default_params(**prm))
            h.solve()  # warm-up (graph capture, SELL copies)
            _, st, rc = h.solve()
            out[name] = {"seconds": st.seconds, "iterations": st.iterations, "rel_res": st.rel_res,
                         "status": rc, "smoother_used": st.smoother_used}
        rows.append(out)
        h.close()
    return rows


if __name__ == "__main__":
    import argparse
    import json
    import os
    ap = argparse.ArgumentParser()
    ap.add_argument("mode", choices=["train", "eval"])
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--levels", type=int, default=4)
    ap.add_argument("--problems", type=int, default=8)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--weights", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights",
                                                      "stencil_net_q1.f32"))
    ap.add_argument("--seeds", default="5000,5001,5002,5003")
    ap.add_argument("--out", default=None)
    ap.add_argument("--learned-steps", default="2,4")
    a = ap.parse_args()
    if a.mode == "train":
        w0 = init_weights(0)
        probs = []
        for s in range(a.problems):
            h, lv = make_problem(1000 + s, a.n, a.levels)
            E, R = generate_pairs(h, lv, 2, 4, s)
            probs.append((h, lv, E, R))
        w, hist = train(probs, w0, a.steps, lr=a.lr, log_every=50)
        os.makedirs(os.path.dirname(a.weights), exist_ok=True)
        w.astype(np.float32).tofile(a.weights)
        res = {"loss_first": hist[0], "loss_last20": float(np.mean(hist[-20:])), "steps": a.steps,
               "problems": a.problems, "n": a.n}
    else:
        w = np.fromfile(a.weights, dtype=np.float32)
        res = {"rows": evaluate(w, [int(x) for x in a.seeds.split(",")], n=a.n, levels=a.levels,
                                learned_steps=[int(x) for x in a.learned_steps.split(",")])}
    print(json.dumps(res))
    if a.out:
        with open(a.out, "w") as f:
            json.dump(res, f)
