"""Interaction variants TBME = base + sum lam_i P_i: the linear-combination generator
(nushellx_b200.gen.variants) against direct generation, and nsx_set_interaction on the
GPU against a handle created from the variant problem."""
import numpy as np
import pytest

from conftest import make_problem

LAM = np.array([0.21, -0.13, 0.05, -0.29, 0.17, 0.0, -0.08, 0.26])


def _family(name):
    from nushellx_b200.gen.variants import InteractionFamily
    return InteractionFamily(make_problem(name))


def _direct(P, inter):
    """The base problem's structure with another interaction (multipoles and segments recomputed)."""
    import copy
    from nushellx_b200.gen.pnint import multipole_pn
    Q = copy.copy(P)
    Q.inter = inter
    Q.vlam = multipole_pn(inter)
    Q.segA = P.A.hamiltonian_segments(inter, P.renorm)
    Q.segB = Q.segA if P.segB is P.segA else P.B.hamiltonian_segments(inter, P.renorm)
    return Q


@pytest.mark.parametrize("name", ["sd_2p2n_0", "sd_2p2n_2"])
def test_family_arrays_match_direct_generation(name):
    from nushellx_b200.gen.writer import segment_arrays
    from nushellx_b200.gen.pnint import op_values
    P = make_problem(name)
    fam = _family(name)
    op, a, b = fam.arrays(LAM)
    Q = _direct(P, fam.interaction(LAM))
    assert np.allclose(op, op_values(Q.vlam, fam.order), rtol=0, atol=1e-13)
    assert np.allclose(a, segment_arrays(Q.A, Q.segA)["vals"], rtol=0, atol=1e-12)
    assert np.allclose(b, segment_arrays(Q.B, Q.segB)["vals"], rtol=0, atol=1e-12)
    # zero coefficients give the base problem back exactly
    op0, a0, b0 = fam.arrays(np.zeros(fam.nperturb))
    assert np.array_equal(op0, fam.op0) and np.array_equal(a0, fam.a0) and np.array_equal(b0, fam.b0)


def test_variant_lambdas_are_seeded_and_bounded():
    from nushellx_b200.gen.variants import sample_lambdas
    L1, L2 = sample_lambdas(64), sample_lambdas(64)
    assert L1.shape == (64, 8) and np.array_equal(L1, L2)
    assert np.abs(L1).max() <= 0.3


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["sd_2p2n_2", "fp_4p4n_0"])
def test_set_interaction_matches_a_fresh_handle(name):
    from nushellx_b200.build import build
    from nushellx_b200.nsx import Solver, NSX_FP64, NSX_FP32
    build()
    P = make_problem(name)
    fam = _family(name)
    Q = _direct(P, fam.interaction(LAM))
    S = Solver.from_problem(P)
    F = Solver.from_problem(Q)
    x = np.random.default_rng(3).standard_normal(S.dim) * S.lcoef
    y_base64 = S.matvec_host(x, NSX_FP64)
    y_base32 = S.matvec_host(x, NSX_FP32)
    S.set_interaction(*fam.arrays(LAM))
    for prec, tol in ((NSX_FP64, 1e-12), (NSX_FP32, 2e-5)):
        y, yf = S.matvec_host(x, prec), F.matvec_host(x, prec)
        assert np.abs(y - yf).max() <= tol * np.abs(yf).max(), prec
    # and back: the base interaction restores the base product (to rounding: the proton-side
    # stage adds its K-split partial sums atomically, so repeated products may differ in the
    # last bits)
    S.set_interaction(fam.op0, fam.a0, fam.b0)
    assert np.abs(S.matvec_host(x, NSX_FP64) - y_base64).max() <= 1e-13 * np.abs(y_base64).max()
    assert np.abs(S.matvec_host(x, NSX_FP32) - y_base32).max() <= 1e-6 * np.abs(y_base32).max()
    # wrong sizes are refused
    from nushellx_b200.nsx import NsxError
    with pytest.raises(NsxError):
        S.set_interaction(fam.op0[:-1], fam.a0, fam.b0)
    S.close()
    F.close()
