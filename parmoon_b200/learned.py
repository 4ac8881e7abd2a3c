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


def generate_pairs(h, lv, n_start, n_steps, seed, precision=P.PREC_FP32, post_cgc=True):
    """(E, R) torch tensors (FP64, cuda) of what the smoothers see inside the plain GMG:
    starting from a random error e_0 (zero on Dirichlet nodes) the plain V-cycle's error
    propagation e_{k+1} = e_k - MG(A e_k) gives the pre-smoother's inputs e_k (n_start *
    n_steps samples); with post_cgc the same e_k go once more through the V-cycle without
    post-smoothing, whose error e_k - MG_0(A e_k) is what the post-smoother sees after the
    coarse-grid correction (as many samples again).  Every error is scaled to |e| = 1."""
    import torch
    F = lv[-1]
    N, Na = F["N"], F["active_bound"]
    rng = np.random.default_rng(seed)
    top = len(lv) - 1

    def cycle(e):
        r = h.matvec(top, e)
        r[Na:] = 0.0
        rd = torch.from_numpy(r).cuda()
        zd = torch.empty_like(rd)
        h.vcycle(rd.data_ptr(), zd.data_ptr())
        torch.cuda.synchronize()
        e = e - zd.cpu().numpy()
        e[Na:] = 0.0
        return e / max(np.linalg.norm(e), 1e-300)

    pre = []
    for _ in range(n_start):
        e = rng.standard_normal(N)
        e[Na:] = 0.0
        e /= np.linalg.norm(e)
        for _k in range(n_steps):
            pre.append(e.copy())
            e = cycle(e)
    samples = list(pre)
    if post_cgc:
        h.set_params(P.default_params(precision=precision, post_smooth=0))
        samples += [cycle(e) for e in pre]
        h.set_params(P.default_params(precision=precision))
    E, R = [], []
    for e in samples:
        r = h.matvec(top, e)
        r[Na:] = 0.0
        E.append(e)
        R.append(r)
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
    V-cycle and FP32 learned-smoother V-cycles (k learned steps per phase) with the SSOR
    guard and without it, all in FP64 FGMRES.  Each variant is solved once to warm up
    (graph capture, SELL copies); before the timed solve of a learned variant the weights
    are set again, so its time includes the network's forward pass on every level."""
    rows = []
    for s in seeds:
        h, lv = make_problem(s, n, levels, precision=P.PREC_FP64, weights=weights)
        out = {"seed": int(s), "n_dofs": int(lv[-1]["N"])}
        variants = [("fp64_ssor", dict(precision=P.PREC_FP64)), ("fp32_ssor", dict(precision=P.PREC_FP32))]
        for k in learned_steps:
            for guard_off in (0, 1):
                name = f"fp32_learned_{k}" + ("_unguarded" if guard_off else "")
                variants.append((name, dict(precision=P.PREC_FP32, smoother=P.SMOOTHER_LEARNED, learned_steps=k,
                                            learned_guard_off=guard_off, lin_maxit=400)))
        for name, prm in variants:
            h.set_params(P.default_params(**prm))
            try:
                h.solve()  # warm-up (graph capture, SELL copies)
            except P.PmgError:
                pass  # reported by the timed solve below
            if prm.get("smoother") == P.SMOOTHER_LEARNED:
                h.set_learned_weights(weights)
            try:
                _, st, rc = h.solve()
            except P.PmgError as e:
                out[name] = {"status": e.code, "error": str(e)}
                continue
            out[name] = {"seconds": st.seconds, "setup_seconds": st.setup_seconds, "iterations": st.iterations,
                         "rel_res": st.rel_res, "contraction": st.mean_contraction, "status": rc,
                         "smoother_used": st.smoother_used, "rho_plain": st.rho_plain,
                         "rho_learned": st.rho_learned, "learned_cycles": st.learned_cycles}
        rows.append(out)
        h.close()
    return rows


def run_c4(weights_out, n_train=256, train_cells=64, train_levels=4, n_test=32, test_cells=128, test_levels=5,
           steps=2048, chunk=32, lr=1e-3, batch=4, learned_steps=(2, 4), log=print):
    """The learned-smoother configuration: train on n_train seeded problems at
    train_cells^3 (plain-GMG error samples, 2 starts x 4 cycles each), in chunks of
    `chunk` problems held on the device at a time, then evaluate on n_test held-out
    seeds at test_cells^3 against plain SSOR.  Returns the training record and the
    per-seed rows."""
    import time
    w = init_weights(0)
    rng = np.random.default_rng(0)
    train_seeds = rng.permutation(np.arange(1000, 1000 + n_train))
    val = []
    for s in (900, 901):
        h, lv = make_problem(s, train_cells, train_levels)
        E, R = generate_pairs(h, lv, 2, 4, s)
        val.append((h, lv, E, R))

    def val_loss(wt):
        tot = 0.0
        for h, lv, E, R in val:
            h.set_learned_weights(wt)
            loss, _ = h.learned_train_step(len(lv) - 1, E.data_ptr(), R.data_ptr(), E.shape[0], 0.0)
            tot += loss
        return tot / len(val)

    rec = {"val_loss_initial": val_loss(w), "loss": [], "chunks": []}
    n_chunks = (n_train + chunk - 1) // chunk
    per_chunk = max(1, steps // n_chunks)
    t0 = time.time()
    for c in range(n_chunks):
        seeds = train_seeds[c * chunk:(c + 1) * chunk]
        probs = []
        for s in seeds:
            h, lv = make_problem(int(s), train_cells, train_levels)
            E, R = generate_pairs(h, lv, 2, 4, int(s))
            probs.append((h, lv, E, R))
        w, hist = train(probs, w, per_chunk, lr=lr, batch=batch, seed=c)
        for h, *_ in probs:
            h.close()
        rec["loss"] += [float(x) for x in hist]
        vl = val_loss(w)
        rec["chunks"].append({"seeds": [int(x) for x in seeds], "train_loss_mean": float(np.mean(hist)),
                              "val_loss": vl, "elapsed_s": time.time() - t0})
        log(f"chunk {c}: train loss {np.mean(hist):.4f}  held-out loss {vl:.4f}  ({time.time() - t0:.0f} s)")
    for h, *_ in val:
        h.close()
    rec["val_loss_final"] = val_loss_final = rec["chunks"][-1]["val_loss"]
    rec.update(n_train=n_train, train_cells=train_cells, steps=per_chunk * n_chunks, batch=batch, lr=lr)
    w.astype(np.float32).tofile(weights_out)
    test_seeds = list(range(5000, 5000 + n_test))
    rows = evaluate(w, test_seeds, n=test_cells, levels=test_levels, learned_steps=learned_steps)
    return rec, rows, val_loss_final


def summarise(rows, learned_steps=(2, 4)):
    """Per-variant medians over the seeds, and how often the guard kept the learned smoother."""
    out = {}
    names = ["fp64_ssor", "fp32_ssor"] + [f"fp32_learned_{k}{g}" for k in learned_steps for g in ("", "_unguarded")]
    for nm in names:
        ok = [r[nm] for r in rows if nm in r and r[nm].get("status", 1) == 0]
        if not ok:
            out[nm] = {"converged": 0}
            continue
        out[nm] = {"converged": len(ok), "median_seconds": float(np.median([x["seconds"] for x in ok])),
                   "median_iterations": float(np.median([x["iterations"] for x in ok])),
                   "median_contraction": float(np.median([x["contraction"] for x in ok]))}
        if "learned" in nm:
            out[nm]["kept_learned"] = int(sum(x["smoother_used"] == P.SMOOTHER_LEARNED for x in ok))
    return out


if __name__ == "__main__":
    import argparse
    import json
    import os
    ap = argparse.ArgumentParser()
    ap.add_argument("mode", choices=["train", "eval", "c4"])
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
    ap.add_argument("--n-train", type=int, default=256)
    ap.add_argument("--n-test", type=int, default=32)
    ap.add_argument("--test-n", type=int, default=128)
    ap.add_argument("--test-levels", type=int, default=5)
    a = ap.parse_args()
    ls = [int(x) for x in a.learned_steps.split(",")]
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
    elif a.mode == "eval":
        w = np.fromfile(a.weights, dtype=np.float32)
        rows = evaluate(w, [int(x) for x in a.seeds.split(",")], n=a.n, levels=a.levels, learned_steps=ls)
        res = {"rows": rows, "summary": summarise(rows, ls)}
    else:
        os.makedirs(os.path.dirname(a.weights), exist_ok=True)
        rec, rows, _ = run_c4(a.weights, n_train=a.n_train, train_cells=a.n, train_levels=a.levels,
                              n_test=a.n_test, test_cells=a.test_n, test_levels=a.test_levels, steps=a.steps,
                              lr=a.lr, learned_steps=ls)
        res = {"training": rec, "rows": rows, "summary": summarise(rows, ls)}
    print(json.dumps(res.get("summary", res)))
    if a.out:
        with open(a.out, "w") as f:
            json.dump(res, f)
