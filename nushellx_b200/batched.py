"""Batched independent solves (the 64-problem workload): the fp (f7/2 p3/2 f5/2 p1/2) 4p+4n
space at J^pi = 0+ .. 4+, each J with interaction variants TBME = base + sum_i lam_i P_i
(lam ~ U[-0.3, 0.3]^8, seeded), 10 eigenpairs each.  Reports the aggregate H.v rate of the
problems solved one after another and through nsx_batch_solve (every handle on its own
stream, host threads overlapping the small problems' round trips).

    python -m nushellx_b200.batched [--problems 64] [--precision fp32|fp64]
"""
import argparse
import json
import time

import numpy as np


def build_problems(n, seed=11):
    from .gen import space as S
    from .gen.problem import JProblem
    from .gen.variants import InteractionFamily, sample_lambdas
    from .nsx import Solver
    solvers, meta = [], []
    Js = [0, 2, 4, 6, 8]
    per = [n // len(Js) + (1 if i < n % len(Js) else 0) for i in range(len(Js))]
    for J2, k in zip(Js, per):
        P = JProblem.from_workload(S.Workload(f"fp_4p4n_{J2}", S.FP, 4, 4, J2, 1, 2024))
        fam = InteractionFamily(P)
        for lam in sample_lambdas(k, 8, seed + J2):
            Sv = Solver.from_problem(P)
            Sv.set_interaction(*fam.arrays(lam))
            solvers.append(Sv)
            meta.append({"J2": J2, "dim": Sv.dim})
    return solvers, meta


def main():
    import torch
    from .build import build
    from .nsx import Solver, NSX_FP32, NSX_FP64
    ap = argparse.ArgumentParser()
    ap.add_argument("--problems", type=int, default=64)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    a = ap.parse_args()
    build()
    t0 = time.time()
    solvers, meta = build_problems(a.problems)
    t_setup = time.time() - t0
    prec = NSX_FP32 if a.precision == "fp32" else NSX_FP64
    kw = dict(nev=10, tol=1e-4, precision=prec, refine=prec == NSX_FP32)
    Solver.batch_solve(solvers[:4], **kw)           # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    one = [S.solve(**kw) for S in solvers]
    t_one = time.perf_counter() - t0
    t0 = time.perf_counter()
    many = Solver.batch_solve(solvers, **kw)
    t_many = time.perf_counter() - t0
    mv_one = sum(r["matvecs"] for _, _, r in one)
    mv_many = sum(r["matvecs"] for _, _, r in many)
    dE = max(float(np.abs(e1 - e2).max()) for (e1, _, _), (e2, _, _) in zip(one, many))
    print(json.dumps({"problems": len(solvers), "precision": a.precision,
                      "dims": sorted({m["dim"] for m in meta}), "setup_s": t_setup,
                      "one_by_one_s": t_one, "batched_s": t_many,
                      "matvecs_per_s_one_by_one": mv_one / t_one, "matvecs_per_s_batched": mv_many / t_many,
                      "speedup": t_one / t_many, "max_dE_batched_vs_one_by_one": dE}))
    for S in solvers:
        S.close()


if __name__ == "__main__":
    main()
