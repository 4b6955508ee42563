"""nsx_batch_solve: independent problems (different J^pi, interaction variants, sizes)
solved at once on per-handle streams give the same eigenpairs as solving them one by one.

Tolerance: FP64 solves to Ritz residual 1e-9, so eigenvalues agree to 1e-8 MeV (the
product's atomic partial sums make repeated solves differ in the last bits)."""
import time
import numpy as np
import pytest

from conftest import make_problem, custom_problem

pytestmark = pytest.mark.gpu


def test_batch_matches_one_by_one():
    from nushellx_b200.build import build
    from nushellx_b200.nsx import Solver, NSX_FP64, NSX_FP32, NsxError
    from nushellx_b200.gen.variants import InteractionFamily, sample_lambdas
    build()
    probs = [make_problem("sd_2p2n_0"), make_problem("sd_2p2n_2"), make_problem("fp_4p4n_0"),
             custom_problem("FP", 4, 4, 2, 1, 2024)]
    solvers = [Solver.from_problem(P) for P in probs]
    fam = InteractionFamily(make_problem("fp_4p4n_0"))
    for lam in sample_lambdas(2, 8, 3):
        S = Solver.from_problem(make_problem("fp_4p4n_0"))
        S.set_interaction(*fam.arrays(lam))
        solvers.append(S)
    kw = dict(nev=6, tol=1e-9, precision=NSX_FP64)
    t0 = time.perf_counter()
    one = [S.solve(**kw) for S in solvers]
    t_one = time.perf_counter() - t0
    t0 = time.perf_counter()
    many = Solver.batch_solve(solvers, want_vectors=True, **kw)
    t_many = time.perf_counter() - t0
    print(f"one by one {t_one:.3f} s, batched {t_many:.3f} s")
    for (e1, _, r1), (e2, v2, r2) in zip(one, many):
        assert np.abs(e1 - e2).max() < 1e-8
        assert r2["converged"] == 6 and v2.shape[0] == 6
    # mixed precision in one batch too
    many32 = Solver.batch_solve(solvers, nev=6, tol=1e-5, precision=NSX_FP32, refine=True)
    for (e1, _, _), (e2, _, _) in zip(one, many32):
        assert np.abs(e1 - e2).max() < 1e-5
    with pytest.raises(NsxError):
        Solver.batch_solve([solvers[0], solvers[0]], **kw)
    for S in solvers:
        S.close()
