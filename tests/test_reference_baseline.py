"""The host-core baseline: a complete solve of the C restatement of NuLnz (the reference's
standard Lanczos and its own stopping rule, src/NuLnz/NuCoreX.f90:595-751) against its
eigenvalues from an independent eigensolver, and the bounded-sample estimate that the GPU arm's
cpu_baseline reports against the measured time of that complete solve (fp 4p+4n, J=0+)."""
import numpy as np
import pytest

from conftest import make_problem


def test_complete_reference_solve_and_the_sample_estimate():
    import scipy.sparse.linalg as sla
    from oracle.ref import RefSolver
    import bench
    P = make_problem("fp_4p4n_0")
    R = RefSolver(P)
    ev, iters, secs = R.solve(nlev=10)
    # the reference's rule stops between its first test (90 steps) and its cap (300)
    assert 90 <= iters <= 300
    # its eigenvalues against ARPACK on the same FP32 operator, restricted to the allowed parity
    from nushellx_b200.nsx import Solver
    mask = Solver.from_problem(P, device=-1).lcoef
    idx = np.flatnonzero(mask)

    def mv(v):
        x = np.zeros(R.dim, dtype=np.float32)
        x[idx] = v
        return R.matvec(x)[idx].astype(np.float64)

    op = sla.LinearOperator((len(idx), len(idx)), matvec=mv, dtype=np.float64)
    ref = np.sort(sla.eigsh(op, k=14, which="SA", tol=1e-9)[0])
    # level_limit is 5e-4 MeV between tests; the FP32 storage adds its rounding.  The lowest,
    # well separated levels match; every Ritz value lies at an eigenvalue.  The stagnation rule
    # can stop before a close cluster is resolved: here it reports one level of a cluster near
    # 0.38 MeV and misses two, which a residual test (the GPU solver's) does not allow.
    assert np.abs(ev[:5] - ref[:5]).max() < 1e-3, (ev, ref)
    assert all(np.abs(ref - e).min() < 5e-3 for e in ev), (ev, ref)
    # the sampled estimate (2 pre-iterations + 6 steps, extrapolated) of a solve of as many steps
    est, threads, sample = bench.cpu_reference_sample(P, iters)
    err = est / secs - 1.0
    print(f"complete solve {secs:.2f} s ({iters} steps, {threads} threads); estimate {est:.2f} s; error {err:+.1%}")
    assert abs(err) < 0.5, (est, secs)
    R.close()
