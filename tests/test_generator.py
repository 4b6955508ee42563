"""Pins of the synthetic input generator (CPU).

The reference ships no tests, fixtures or golden outputs for this path, so the
generator -- and with it every phase and normalisation convention the J-scheme
product depends on (partition J-projection, NuOpd's reduced densities, NuOp's
multipole pn weights, NuCoreX's Racah weights) -- is pinned against an
independent M-scheme diagonalisation and against closed-form known answers.
"""
import numpy as np
import pytest

from conftest import make_problem, custom_problem
from nushellx_b200.gen.angmom import cg, sixj, racah_w
from nushellx_b200.gen.pnint import racah_weight
from nushellx_b200.gen.space import WORKLOADS, gaussian_interaction, Interaction, SD, FP, tbme_keys
from nushellx_b200.gen.species import Species


def dense_jscheme(P, rho_a=None, rho_b=None):
    """Dense J-scheme H from the generator's in-memory data (kron form of the pn product)."""
    A, B = P.A, P.B
    rho_a = rho_a or P.rhoA
    rho_b = rho_b or P.rhoB
    n = P.no_state
    H = np.zeros((n, n))
    for kl, (jal, jbl) in enumerate(P.blocks):
        ol = P.offsets[kl]
        dal, dbl = P.dims[kl]
        if dal * dbl == 0:
            continue
        H[ol:ol + dal * dbl, ol:ol + dal * dbl] += (np.kron(np.eye(dbl), P.dense_like(A, P.segA, jal))
                                                   + np.kron(P.dense_like(B, P.segB, jbl), np.eye(dal)))
        for kr, (jar, jbr) in enumerate(P.blocks):
            orr = P.offsets[kr]
            dar, dbr = P.dims[kr]
            if dar * dbr == 0:
                continue
            for (o1, o3, o2, o4, lam), V in P.vlam.items():
                ka, kb = (jal, jar, o1, o3, lam), (jbl, jbr, o2, o4, lam)
                if ka not in rho_a or kb not in rho_b or V == 0:
                    continue
                w = racah_weight(jal, jbl, jar, jbr, P.J2, lam)
                if w == 0:
                    continue
                H[ol:ol + dal * dbl, orr:orr + dar * dbr] += V * w * np.kron(
                    P.dense_rho(B, rho_b, kb), P.dense_rho(A, rho_a, ka))
    return H


def test_cg_and_sixj_against_sympy():
    from sympy import Rational
    from sympy.physics.quantum.cg import CG
    from sympy.physics.wigner import wigner_6j
    h = Rational(1, 2)
    rng = np.random.default_rng(1)
    for _ in range(200):
        j1, j2 = rng.integers(0, 10, 2)
        J = rng.integers(abs(j1 - j2), j1 + j2 + 1)
        if (j1 + j2 + J) % 2:
            continue
        m1 = rng.choice(range(-j1, j1 + 1, 2))
        m2 = rng.choice(range(-j2, j2 + 1, 2))
        ref = float(CG(j1 * h, m1 * h, j2 * h, m2 * h, J * h, (m1 + m2) * h).doit()) if abs(m1 + m2) <= J else 0.0
        assert abs(cg(int(j1), int(j2), int(J), int(m1), int(m2), int(m1 + m2)) - ref) < 1e-12
    for _ in range(200):
        a, b, d, e = (int(v) for v in rng.integers(0, 9, 4))
        c = int(rng.integers(abs(a - b), a + b + 1))
        f = int(rng.integers(abs(a - e), a + e + 1))
        if any((x + y + z) % 2 for x, y, z in ((a, b, c), (a, e, f), (d, b, f), (d, e, c))):
            assert sixj(a, b, c, d, e, f) == 0.0
            continue
        ref = float(wigner_6j(a * h, b * h, c * h, d * h, e * h, f * h))
        assert abs(sixj(a, b, c, d, e, f) - ref) < 1e-12


@pytest.mark.parametrize("name", ["sd_2p2n_0", "sd_2p2n_2"])
def test_jscheme_spectrum_matches_mscheme(name):
    from oracle.mscheme import jscheme_spectrum_from_mscheme
    P = make_problem(name)
    H = dense_jscheme(P)
    assert np.abs(H - H.T).max() < 1e-12
    e = np.linalg.eigvalsh(H[np.ix_(P.lcoef, P.lcoef)])
    w = WORKLOADS[name]
    em = jscheme_spectrum_from_mscheme(gaussian_interaction(w.space, w.seed), w.nprot, w.nneut, w.J2)
    assert len(e) == len(em)
    assert np.abs(e - em).max() < 1e-10


def test_mixed_parity_odd_nucleons_matches_mscheme():
    """f5/2 p3/2 p1/2 g9/2 (mixed parity), 2 protons + 1 neutron, J = 3/2, both parities."""
    from oracle.mscheme import jscheme_spectrum_from_mscheme
    from nushellx_b200.gen.space import F5PG9
    P = custom_problem("F5PG9", 2, 1, 3, -1, 9)
    H = dense_jscheme(P)
    e = np.linalg.eigvalsh(H)
    em = jscheme_spectrum_from_mscheme(gaussian_interaction(F5PG9, 9), 2, 1, 3)
    assert np.abs(e - em).max() < 1e-10


def test_zero_interaction_gives_spe_sums():
    """Known answer: with V = 0 every eigenvalue is a sum of SPEs over occupations."""
    w = WORKLOADS["sd_2p2n_0"]
    zero = Interaction(w.space, {})
    from nushellx_b200.gen.problem import JProblem
    P = JProblem(w.space, zero, 2, 2, 0, 1)
    H = dense_jscheme(P)
    assert np.abs(H - np.diag(np.diag(H))).max() < 1e-12
    e = np.sort(np.diag(H))
    # allowed totals: sums of 2 proton + 2 neutron SPEs over orbits
    spe = w.space.spe
    allowed = {round(spe[a] + spe[b] + spe[c] + spe[d], 9) for a in range(3) for b in range(3)
               for c in range(3) for d in range(3)}
    assert all(round(x, 9) in allowed for x in e)
    assert abs(e.min() - (2 * min(spe) * 2)) < 1e-12


def test_two_identical_nucleons_known_answer():
    """2 protons, 0 neutrons: the J-spectrum is eig(V_J,T=1 + SPE pair sums) over pair labels."""
    from nushellx_b200.gen.angmom import triangle
    sp = SD
    inter = gaussian_interaction(sp, 3)
    S = Species(sp.j2, sp.parity, sp.spe, 2, 0)
    segs = S.hamiltonian_segments(inter)
    for J2 in S.J2_values():
        o = [0]
        for ip in range(len(S.parts)):
            o.append(o[-1] + S.njt(ip, J2))
        Hd = np.zeros((o[-1], o[-1]))
        for ipl, ipr, M in segs[J2]:
            Hd[o[ipl]:o[ipl + 1], o[ipr]:o[ipr + 1]] = M
            Hd[o[ipr]:o[ipr + 1], o[ipl]:o[ipl + 1]] = M.T
        pairs = [(a, b) for a in range(3) for b in range(a, 3)
                 if triangle(sp.j2[a], sp.j2[b], J2) and not (a == b and (J2 // 2) % 2)]
        V = np.array([[inter.V(a, b, c, d, J2, 1) for (c, d) in pairs] for (a, b) in pairs])
        V += np.diag([sp.spe[a] + sp.spe[b] for a, b in pairs])
        assert np.allclose(np.linalg.eigvalsh(Hd), np.linalg.eigvalsh(V), atol=1e-12)


def test_jscheme_dimensions_match_mscheme_counting():
    """nJT sums equal N(M=J) - N(M=J+1) from plain M-scheme counting (fp, 4 particles)."""
    from itertools import combinations
    sp = FP
    S = Species(sp.j2, sp.parity, sp.spe, 4, 0)
    ms = [m for jj in sp.j2 for m in range(-jj, jj + 1, 2)]
    cnt = {}
    for c in combinations(range(len(ms)), 4):
        M = sum(ms[i] for i in c)
        cnt[M] = cnt.get(M, 0) + 1
    for J2 in range(0, S.maxJ2 + 1, 2):
        assert S.dimJ(J2) == cnt.get(J2, 0) - cnt.get(J2 + 2, 0)


def test_canonical_basis_is_orthonormal_and_deterministic():
    sp = FP
    S1 = Species(sp.j2, sp.parity, sp.spe, 3, 0)
    S2 = Species(sp.j2, sp.parity, sp.spe, 3, 0)
    for key, B in S1.HW.items():
        assert np.allclose(B.T @ B, np.eye(B.shape[1]), atol=1e-12)
        assert np.array_equal(B, S2.HW[key])


def test_tbme_set_is_symmetric_and_seeded():
    a = gaussian_interaction(SD, 11)
    b = gaussian_interaction(SD, 11)
    assert a.tbme == b.tbme
    keys = tbme_keys(SD)
    assert len(a.tbme) == len(keys)
    # V(ab;cd) = V(cd;ab) through the accessor
    for (p, q, r, s, J2, T) in keys[:50]:
        assert a.V(p, q, r, s, J2, T) == a.V(r, s, p, q, J2, T)
