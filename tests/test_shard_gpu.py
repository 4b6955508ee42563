"""Output-block shards of H.v on one GPU, through the C ABI.

* Each shard handle's product writes exactly its rows, equal to the whole handle's product
  there (FP64 and the FP32 tensor-core form), and leaves every other row as it was.
* A sharded solve: two shard handles solve in two host threads, each product completed by an
  exchange that copies the ranks' rows through a shared device buffer (a host-side barrier
  between the threads; no kernel waits on another).  Both ranks run the same recurrence and
  reach the unsharded eigenvalues.  On several GPUs the exchange is nushellx_b200.sharded's
  NCCL all-gather; the recurrence and the products are the same."""
import threading

import numpy as np
import pytest

from conftest import make_problem

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,world", [("fp_4p4n_0", 2), ("fp_4p4n_0", 3), ("fp_5p3n_2", 2)])
def test_shard_products_write_their_rows_only(name, world):
    from conftest import custom_problem
    from nushellx_b200.build import build
    from nushellx_b200.nsx import Solver, NSX_FP64, NSX_FP32
    build()
    P = make_problem(name) if name == "fp_4p4n_0" else custom_problem("FP", 5, 3, 2, 1, 5)
    full = Solver.from_problem(P)
    x = np.random.default_rng(3).standard_normal(full.dim) * full.lcoef
    for prec, tol in ((NSX_FP64, 1e-12), (NSX_FP32, 1e-6)):
        ref = full.matvec_host(x, prec)
        got = np.full(full.dim, np.nan)
        for r in range(world):
            S = Solver.from_problem(P, shard=(r, world))
            rows = S.shard_info()["rows"]
            y = np.full(full.dim, np.nan)
            S.matvec_host(x, prec, out=y)
            a, b = rows[r], rows[r + 1]
            assert np.all(np.isnan(y[:a])) and np.all(np.isnan(y[b:]))
            assert not np.any(np.isnan(y[a:b]))
            got[a:b] = y[a:b]
            S.close()
        assert not np.any(np.isnan(got))
        assert np.abs(got - ref).max() <= tol * np.abs(ref).max()
    full.close()


class _Array:
    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def test_sharded_solve_reaches_the_unsharded_eigenvalues():
    import torch
    from nushellx_b200.build import build
    from nushellx_b200.nsx import Solver, NSX_FP64, NSX_FP32, NsxError
    build()
    P = make_problem("fp_4p4n_0")
    world = 2
    full = Solver.from_problem(P)
    e_ref, _, _ = full.solve(nev=6, tol=1e-8, precision=NSX_FP64)
    full.close()
    shards = [Solver.from_problem(P, shard=(r, world)) for r in range(world)]
    rows = shards[0].shard_info()["rows"]
    with pytest.raises(NsxError, match="exchange"):   # a shard cannot solve on its own rows
        shards[0].solve(nev=2, tol=1e-6, precision=NSX_FP64)
    dev = torch.device("cuda", 0)
    whole = torch.empty(int(rows[-1]), dtype=torch.float64, device=dev)
    bar = threading.Barrier(world, timeout=120)
    calls = [0] * world

    def make_exchange(r):
        a, b = int(rows[r]), int(rows[r + 1])

        def fn(y_ptr, n, stream_ptr):
            y = torch.as_tensor(_Array(y_ptr, n), device=dev)
            s = torch.cuda.ExternalStream(stream_ptr, device=dev)
            with torch.cuda.stream(s):
                whole[a:b].copy_(y[a:b])
            s.synchronize()
            bar.wait()
            with torch.cuda.stream(s):
                y.copy_(whole)
            s.synchronize()
            bar.wait()
            calls[r] += 1
        return fn

    for r, S in enumerate(shards):
        S.set_exchange(make_exchange(r))
    results = [None] * world

    def run(r):
        try:
            results[r] = shards[r].solve(nev=6, tol=1e-8, precision=prec, refine=prec == NSX_FP32)
        except BaseException as e:
            results[r] = e
            bar.abort()

    for prec in (NSX_FP64, NSX_FP32):
        bar.reset()
        ts = [threading.Thread(target=run, args=(r,)) for r in range(world)]
        for t in ts:
            t.start()
        for t in ts:
            t.join(timeout=600)
        for r in range(world):
            assert not isinstance(results[r], BaseException), (results[r], shards[r].exchange_error)
        (e0, _, r0), (e1, _, r1) = results
        assert np.array_equal(e0, e1) and r0["iterations"] == r1["iterations"]
        assert np.abs(e0 - e_ref).max() < (1e-8 if prec == NSX_FP64 else 1e-5)
    assert calls[0] == calls[1] > 0
    for S in shards:
        S.close()


def test_a_failing_exchange_fails_the_product():
    """The exchange is the shards' only communication: when it reports a failure (an exception
    in the host function: a rank gone, a collective timed out), the product fails with an error
    code and the exception is kept for the caller; the handle stays usable."""
    from nushellx_b200.build import build
    from nushellx_b200.nsx import Solver, NSX_FP64, NsxError
    build()
    P = make_problem("sd_2p2n_2")
    S = Solver.from_problem(P, shard=(0, 2))

    def broken(y_ptr, n, stream_ptr):
        raise TimeoutError("peer rank did not answer")

    S.set_exchange(broken)
    x = np.random.default_rng(0).standard_normal(S.dim)
    with pytest.raises(NsxError, match="exchange"):
        S.matvec_host(x, NSX_FP64)
    assert isinstance(S.exchange_error, TimeoutError)
    S.set_exchange(None)   # without an exchange the rank's rows are still computed
    y = np.full(S.dim, np.nan)
    S.matvec_host(x, NSX_FP64, out=y)
    rows = S.shard_info()["rows"]
    assert not np.any(np.isnan(y[rows[0]:rows[1]])) and np.all(np.isnan(y[rows[1]:]))
    S.close()
