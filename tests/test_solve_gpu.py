"""Thick-restart Lanczos on the GPU (nsx_solve) against dense diagonalisation."""
import numpy as np
import pytest

from conftest import make_problem, custom_problem

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _lib():
    from nushellx_b200.build import build
    build()


def _exact(P, nev):
    from test_generator import dense_jscheme
    H = dense_jscheme(P)
    return np.linalg.eigvalsh(H[np.ix_(P.lcoef, P.lcoef)])[:nev]


@pytest.mark.parametrize("name", ["sd_2p2n_0", "sd_2p2n_2"])
def test_small_space_all_levels(name):
    """dim < window: the Krylov space is exhausted and the projection is exact."""
    from nushellx_b200.nsx import Solver, NSX_FP64
    P = make_problem(name)
    S = Solver.from_problem(P)
    ev, _, rep = S.solve(nev=10, tol=1e-8, precision=NSX_FP64, window=100)
    assert np.abs(ev - _exact(P, 10)).max() < 1e-9


def test_thick_restart_fp64_matches_dense():
    """fp 4p+4n J=0 is too large for dense here; use a small window to force restarts on sd 2p2n J=2."""
    from nushellx_b200.nsx import Solver, NSX_FP64
    P = make_problem("sd_2p2n_2")
    S = Solver.from_problem(P)
    ev, vecs, rep = S.solve(nev=5, tol=1e-9, precision=NSX_FP64, window=24, keep=10, want_vectors=True)
    assert rep["restarts"] >= 1
    assert np.abs(ev - _exact(P, 5)).max() < 1e-8
    # Ritz vectors: orthonormal, of the requested parity, small residuals
    G = vecs @ vecs.T
    assert np.abs(G - np.eye(5)).max() < 1e-8
    if (~S.lcoef).any():
        assert np.abs(vecs[:, ~S.lcoef]).max() < 1e-12
    for k in range(5):
        r = S.matvec_host(vecs[k]) - ev[k] * vecs[k]
        assert np.linalg.norm(r) < 1e-7


def test_fp32_matvec_with_fp64_refinement_reaches_1e5():
    """FP32 contractions + FP64 Lanczos + FP64 Rayleigh-Ritz: |dE| < 1e-5 MeV vs the FP64 answer."""
    from nushellx_b200.nsx import Solver, NSX_FP64, NSX_FP32
    P = make_problem("fp_4p4n_0")
    S = Solver.from_problem(P)
    e64, _, r64 = S.solve(nev=10, tol=1e-7, precision=NSX_FP64, window=100)
    e32, _, r32 = S.solve(nev=10, tol=1e-4, precision=NSX_FP32, window=100, refine=True)
    assert r64["converged"] == 10
    assert np.abs(e32 - e64).max() < 1e-5, np.abs(e32 - e64)


def test_breakdown_invariant_subspace():
    """A start vector inside an invariant subspace (an eigenvector) triggers the breakdown restart."""
    from nushellx_b200.nsx import Solver, NSX_FP64
    from test_generator import dense_jscheme
    P = make_problem("sd_2p2n_0")
    H = dense_jscheme(P)
    w, V = np.linalg.eigh(H)
    S = Solver.from_problem(P)
    start = V[:, 3] + V[:, 7]        # 2-dimensional invariant subspace
    ev, _, rep = S.solve(nev=4, tol=1e-9, precision=NSX_FP64, window=40, start=start, pre_iter=0)
    assert np.abs(ev - w[:4]).max() < 1e-8


def test_mixed_parity_negative_parity_levels():
    from nushellx_b200.nsx import Solver, NSX_FP64
    P = custom_problem("F5PG9", 2, 1, 3, -1, 9)
    S = Solver.from_problem(P)
    ev, _, _ = S.solve(nev=6, tol=1e-9, precision=NSX_FP64, window=60)
    assert np.abs(ev - _exact(P, 6)).max() < 1e-8
