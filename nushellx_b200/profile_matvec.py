"""Runs a few H.v products of one workload on cuda:0 (the command profiled by ncu).

    python -m nushellx_b200.profile_matvec [workload] [fp32|fp64] [reps]
"""
import sys


def main():
    import torch
    from nushellx_b200.gen.space import WORKLOADS
    from nushellx_b200.gen.problem import JProblem
    from nushellx_b200.nsx import Solver, NSX_FP64, NSX_FP32
    name = sys.argv[1] if len(sys.argv) > 1 else "fp_6p6n_0"
    prec = NSX_FP64 if (len(sys.argv) > 2 and sys.argv[2] == "fp64") else NSX_FP32
    reps = int(sys.argv[3]) if len(sys.argv) > 3 else 3
    S = Solver.from_problem(JProblem.from_workload(WORKLOADS[name]))
    x = torch.randn(S.dim, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    for _ in range(reps):
        S.matvec(x.data_ptr(), y.data_ptr(), prec)
    torch.cuda.synchronize()
    S.stats_reset(timing=True)
    for _ in range(reps):
        S.matvec(x.data_ptr(), y.data_ptr(), prec)
    st = S.stats()["stages"]
    per = {k: round(v["ms"] / v["launches"], 4) for k, v in st.items() if v["launches"]}
    print(name, "dim", S.dim, "ok", float(y.abs().max()), "ms/launch", per)
    S.close()


if __name__ == "__main__":
    main()
