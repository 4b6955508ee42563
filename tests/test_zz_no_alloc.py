"""nsx_matvec_noalloc: the FP64 H.v whose scratch is a fixed device array.

It is for callers that cannot have device memory allocated during the call
(cudaMalloc synchronises the device; some hosts give all device memory to
their own pool).  This file is collected last on purpose.  Each test checks the
entry point through the C ABI against nsx_matvec, two calls in a row, within
the FP64 parity tolerance of the other GPU tests (1e-12 relative).
"""
import numpy as np
import pytest

from conftest import make_problem, custom_problem

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.fixture(scope="module", autouse=True)
def _lib():
    from nushellx_b200.build import build
    build()


def _rel(a, b):
    return float((a - b).abs().max() / b.abs().max())


@pytest.mark.parametrize("which", ["sd_2p2n_2", "mixed"])
def test_noalloc_matches_matvec_twice(which):
    import torch
    from nushellx_b200.nsx import Solver, NSX_FP64
    P = make_problem("sd_2p2n_2") if which == "sd_2p2n_2" else custom_problem("F5PG9", 2, 1, 3, -1, 9)
    S = Solver.from_problem(P)
    g = torch.Generator(device="cuda").manual_seed(11)
    for call in range(2):
        x = torch.randn(S.dim, dtype=torch.float64, device="cuda", generator=g)
        y_ref = torch.empty_like(x)
        y = torch.full_like(x, float("nan"))
        S.matvec(x.data_ptr(), y_ref.data_ptr(), NSX_FP64)
        S.matvec_noalloc(x.data_ptr(), y.data_ptr())
        torch.cuda.synchronize()
        assert _rel(y, y_ref) < TOL, (call, _rel(y, y_ref))
    S.close()


def test_noalloc_after_a_different_problem_leaves_no_stale_scratch():
    """The shared array keeps the previous call's contents: a second problem must not see them."""
    import torch
    from nushellx_b200.nsx import Solver, NSX_FP64
    for name in ("sd_2p2n_2", "sd_2p2n_0"):
        S = Solver.from_problem(make_problem(name))
        x = torch.randn(S.dim, dtype=torch.float64, device="cuda")
        y_ref, y = torch.empty_like(x), torch.empty_like(x)
        S.matvec(x.data_ptr(), y_ref.data_ptr(), NSX_FP64)
        S.matvec_noalloc(x.data_ptr(), y.data_ptr())
        torch.cuda.synchronize()
        assert _rel(y, y_ref) < TOL
        S.close()


def test_noalloc_rejects_problems_beyond_the_fixed_size():
    import torch
    from nushellx_b200.nsx import Solver, NsxError
    S = Solver.from_problem(make_problem("fp_4p4n_0"))   # needs about 11.5 Mi scratch elements
    x = torch.randn(S.dim, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    with pytest.raises(NsxError, match="scratch"):
        S.matvec_noalloc(x.data_ptr(), y.data_ptr())
    S.close()


def test_noalloc_first_on_a_fresh_handle_allocates_nothing():
    """No nsx_matvec before it on the handle (so nothing it allocated can be relied on), and the
    device's free memory is the same before and after further calls.  The first call on a
    device may load the library's module (and with it the fixed array), so the free-memory
    check brackets the calls after it."""
    import torch
    from nushellx_b200.nsx import Solver, NSX_FP64
    S = Solver.from_problem(make_problem("sd_2p2n_2"))
    g = torch.Generator(device="cuda").manual_seed(5)
    xs = [torch.randn(S.dim, dtype=torch.float64, device="cuda", generator=g) for _ in range(3)]
    ys = [torch.full_like(xs[0], float("nan")) for _ in range(3)]
    S.matvec_noalloc(xs[0].data_ptr(), ys[0].data_ptr())
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for i in (1, 2):
        S.matvec_noalloc(xs[i].data_ptr(), ys[i].data_ptr())
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    for x, y in zip(xs, ys):
        y_ref = torch.empty_like(x)
        S.matvec(x.data_ptr(), y_ref.data_ptr(), NSX_FP64)
        torch.cuda.synchronize()
        assert _rel(y, y_ref) < TOL
    S.close()
