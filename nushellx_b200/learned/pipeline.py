"""Interaction sweep, training and the learned start vector.

    python -m nushellx_b200.learned.pipeline sweep    --workload fp_6p6n_0 --variants 512 --out sweep.npz
    python -m nushellx_b200.learned.pipeline train    --data sweep.npz --train 400 --out model.npz
    python -m nushellx_b200.learned.pipeline evaluate --model model.npz --data sweep.npz --count 8

Sweep: variants TBME = base + sum_i lam_i P_i (lam ~ U[-0.3, 0.3]^8, seeded; gen.variants)
of one workload.  One solver handle is planned once; every variant is loaded into it with
nsx_set_interaction and its ground state is found by the solver itself (FP32 H.v, FP64
Lanczos, FP64 Rayleigh-Ritz refinement) and kept in HBM.  The training variants' ground
states fix the K = 256 kept sub-blocks and their shapes (learned.compress); each variant's
ground state is stored as its K projections.

Training: the network (nsx_mlp, FP32 weights, BF16 activations, trained by libnsx's CUDA
kernels) maps lam / 0.3 to the standardised projections; full-batch Adam.

Start vector: the predicted projections, decompressed onto the kept sub-blocks and
normalised, plus beta (default 1) times the normalised standard seeded random vector, so
that every eigenvector keeps a component comparable to the standard start's (a start that
is almost only the ground state can let Lanczos meet its stopping test with one of the
lowest states still missing); the solve then starts from it without the power
pre-iterations.  The standard
start vector remains the fallback (no model for the workload, or a dimension mismatch).
"""
import argparse
import json
import time

import numpy as np

LAM_SCALE = 0.3
NPERTURB = 8
PERTURB_SEED0 = 1000


def solver_and_family(workload):
    """(problem, interaction family with the 8 seeded perturbations, solver handle on cuda) of a
    named workload; variants are loaded into the handle with Solver.set_interaction."""
    from ..gen.space import WORKLOADS
    from ..gen.problem import JProblem
    from ..gen.variants import InteractionFamily
    from ..nsx import Solver
    P = JProblem.from_workload(WORKLOADS[workload])
    fam = InteractionFamily(P, NPERTURB, PERTURB_SEED0)
    return P, fam, Solver.from_problem(P)


def ground_state(S, tol=1e-5):
    from ..nsx import NSX_FP32
    ev, vecs, rep = S.solve(nev=1, tol=tol, precision=NSX_FP32, window=100, max_iter=3000, refine=True,
                            want_vectors=True)
    return float(ev[0]), vecs[0], rep


def standard_start(S, seed=5):
    """The seeded uniform vector on the parity mask (what nsx_solve draws itself), host side."""
    return np.random.default_rng(seed).uniform(-0.5, 0.5, S.dim) * S.lcoef


def sweep(workload, nvar, seed, K, out, ntrain=None, tol=1e-5, log=print):
    """Ground states of nvar seeded variants; the compression is built from the first ntrain
    of them (default: all) and every variant is stored as its K projections."""
    import torch
    from .compress import SubBlocks, Compressor
    from ..gen.variants import sample_lambdas
    ntrain = nvar if ntrain is None else ntrain
    t0 = time.time()
    P, fam, S = solver_and_family(workload)
    log(f"setup {time.time() - t0:.1f} s, dim {S.dim}")
    lams = sample_lambdas(nvar, NPERTURB, seed, LAM_SCALE)
    G = torch.zeros((nvar, S.dim), dtype=torch.float32, device="cuda")   # ground states, kept in HBM
    E0 = np.zeros(nvar)
    iters = np.zeros(nvar, dtype=np.int64)
    t1 = time.time()
    for v in range(nvar):
        S.set_interaction(*fam.arrays(lams[v]))
        E0[v], g, rep = ground_state(S, tol)
        G[v] = torch.from_numpy(g.astype(np.float32)).to("cuda")
        iters[v] = rep["iterations"]
        if v % 32 == 0 or v == nvar - 1:
            log(f"variant {v}: E0 {E0[v]:.5f} MeV, {iters[v]} iterations, {(time.time() - t1) / (v + 1):.2f} s per variant")
    sub = SubBlocks(P)
    comp = Compressor.from_training(sub, G[:ntrain], K)
    W = np.zeros((nvar, K))
    for v in range(nvar):
        W[v] = comp.compress(G[v].double().cpu().numpy())
    captured = (W ** 2).sum(1)
    log(f"{len(sub)} sub-blocks; the {K} kept hold {captured[:ntrain].mean():.4f} of |g|^2 on average over the "
        f"training variants (min {captured.min():.4f}), {captured[ntrain:].mean() if nvar > ntrain else float('nan'):.4f} "
        f"over the others")
    np.savez(out, workload=workload, lams=lams, W=W, E0=E0, iterations=iters, captured=captured,
             desc=comp.desc, shapes=comp.shapes.astype(np.float32), rank=comp.rank, dim=S.dim, ntrain=ntrain,
             lam_scale=LAM_SCALE, perturb_seed0=PERTURB_SEED0, nperturb=NPERTURB, variant_seed=seed)
    del G
    S.close()
    return out


def train(data, ntrain, out, width=256, steps=4000, lr=2e-3, seed=1, log=print):
    from ..nsx import Network
    d = np.load(data)
    lams, W = d["lams"], d["W"]
    X = (lams / float(d["lam_scale"])).astype(np.float32)
    mu, sd = W[:ntrain].mean(0), W[:ntrain].std(0) + 1e-12
    T = ((W - mu) / sd).astype(np.float32)
    net = Network(X.shape[1], width, W.shape[1], seed=seed)
    t0 = time.time()
    loss = net.train(X[:ntrain], T[:ntrain], steps, lr)
    t_train = time.time() - t0
    pred = net.forward(X) * sd + mu
    def rel(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))
    err_train = rel(pred[:ntrain], W[:ntrain])
    err_test = rel(pred[ntrain:], W[ntrain:]) if len(W) > ntrain else float("nan")
    base = rel(np.broadcast_to(mu, W[ntrain:].shape), W[ntrain:]) if len(W) > ntrain else float("nan")
    log(f"trained {steps} Adam steps in {t_train:.2f} s: loss {loss:.3e}; relative error of the projections "
        f"train {err_train:.4f}, test {err_test:.4f} (mean of the training set: {base:.4f})")
    np.savez(out, params=net.params, n_in=X.shape[1], width=width, n_out=W.shape[1], y_mean=mu, y_std=sd,
             lam_scale=float(d["lam_scale"]), desc=d["desc"], shapes=d["shapes"], rank=d["rank"], dim=int(d["dim"]),
             workload=str(d["workload"]), perturb_seed0=int(d["perturb_seed0"]), nperturb=int(d["nperturb"]),
             ntrain=ntrain, variant_seed=int(d["variant_seed"]), err_train=err_train, err_test=err_test)
    net.close()
    return {"loss": loss, "err_train": err_train, "err_test": err_test, "err_mean_predictor": base,
            "train_seconds": t_train}


class LearnedStart:
    """The network and the compressor of one workload (a model file written by train())."""

    def __init__(self, model, device=0):
        from ..nsx import Network
        from .compress import Compressor
        m = np.load(model) if isinstance(model, str) else model
        self.workload = str(m["workload"])
        self.lam_scale = float(m["lam_scale"])
        self.mu, self.sd = np.asarray(m["y_mean"]), np.asarray(m["y_std"])
        self.net = Network(int(m["n_in"]), int(m["width"]), int(m["n_out"]), device=device)
        self.net.params = m["params"]
        self.comp = Compressor(m["desc"], m["shapes"], int(m["dim"]), m["rank"])
        self.dim = int(m["dim"])
        self._rand = {}   # (solver dimension, seed) -> normalised standard random vector

    def projections(self, lam):
        x = np.asarray(lam, dtype=np.float32).reshape(1, -1) / self.lam_scale
        return self.net.forward(x)[0] * self.sd + self.mu

    def start_vector(self, S, lam, beta=1.0, seed=5):
        """Start vector for the variant lam on solver S, or None (fallback: the standard start)
        when the model does not describe S's vector space."""
        if S.dim != self.dim:
            return None
        x0 = self.comp.decompress(self.projections(lam))
        n0 = np.linalg.norm(x0)
        if not np.isfinite(n0) or n0 == 0.0:
            return None
        key = (S.dim, seed)
        if key not in self._rand:   # the same seeded vector for every variant of the space
            r = standard_start(S, seed)
            self._rand[key] = r / np.linalg.norm(r)
        return x0 / n0 + beta * self._rand[key]

    def close(self):
        self.net.close()


def compare(S, fam, learned, lams, nev=10, tol=1e-4, beta=1.0, log=print):
    """Standard vs learned start on the given variants: iterations, seconds, eigenvalues."""
    from ..nsx import NSX_FP32
    rows = []
    for lam in lams:
        S.set_interaction(*fam.arrays(lam))
        kw = dict(nev=nev, tol=tol, precision=NSX_FP32, window=100, max_iter=3000, refine=True)
        t0 = time.perf_counter()
        e_std, _, r_std = S.solve(**kw)
        t_std = time.perf_counter() - t0
        t0 = time.perf_counter()
        st = learned.start_vector(S, lam, beta)
        e_l, _, r_l = S.solve(start=st, pre_iter=0 if st is not None else 2, **kw)
        t_l = time.perf_counter() - t0
        rows.append({"iter_standard": r_std["iterations"], "iter_learned": r_l["iterations"],
                     "s_standard": t_std, "s_learned": t_l, "max_dE": float(np.abs(e_std - e_l).max())})
        log(json.dumps(rows[-1]))
    return rows


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=["sweep", "train", "evaluate"])
    ap.add_argument("--workload", default="fp_6p6n_0")
    ap.add_argument("--variants", type=int, default=512)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--K", type=int, default=256)
    ap.add_argument("--data", default="sweep.npz")
    ap.add_argument("--model", default="model.npz")
    ap.add_argument("--train", type=int, default=400)   # training variants (the rest are held out)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--count", type=int, default=8)
    ap.add_argument("--beta", type=float, default=1.0)
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    if a.cmd == "sweep":
        sweep(a.workload, a.variants, a.seed, a.K, a.out or a.data, ntrain=a.train)
    elif a.cmd == "train":
        print(json.dumps(train(a.data, a.train, a.out or a.model, steps=a.steps, lr=a.lr)))
    else:
        d = np.load(a.data)
        learned = LearnedStart(a.model)
        P, fam, S = solver_and_family(learned.workload)
        ntrain = int(np.load(a.model)["ntrain"])
        rows = compare(S, fam, learned, d["lams"][ntrain:ntrain + a.count], beta=a.beta)
        it_s = np.mean([r["iter_standard"] for r in rows])
        it_l = np.mean([r["iter_learned"] for r in rows])
        print(json.dumps({"mean_iter_standard": it_s, "mean_iter_learned": it_l,
                          "iterations_saved": 1 - it_l / it_s,
                          "max_dE": max(r["max_dE"] for r in rows)}))


if __name__ == "__main__":
    main()
