"""M-scheme FP64 oracle (test infrastructure only; never on the product path).

An independent full-space check of the J-scheme pipeline.  It builds the
shell-model Hamiltonian directly in the product basis |proton SD> x |neutron SD>
at fixed total M from the isospin-formalism TBMEs and SPEs -- no J projection,
no reduced densities, no multipole recoupling, no Racah weights -- so a J-scheme
spectrum that agrees with it pins every phase and normalisation convention of
the generator (partition J-projection, NuOpd's reduced densities, NuOp's
multipole pn weights, NuCoreX's Racah weights), none of which the reference
itself can pin: it ships no tests, fixtures or golden outputs.

Physics conventions (stated, not taken from the reference):
* like particles: H_pp = sum_{a<=b,c<=d,J,M} V_{J,T=1}(ab;cd) A+_{JM}(ab) A_{JM}(cd),
  A+_{JM}(ab) = (1+d_ab)^(-1/2) sum <ja ma jb mb|JM> a+_a a+_b;
* proton-neutron: V_pn(ab;cd;J) = sqrt((1+d_ab)(1+d_cd))/2 * sum_T V_JT(ab;cd),
  H_pn = sum V_pn B+_{JM}(a_p b_n) B_{JM}(c_p d_n), B+ = sum <ja ma jb mb|JM> a+_p a+_n,
  which factorises exactly as (a+_p a_p) x (a+_n a_n) in the product basis.
Clebsch-Gordan coefficients come from sympy (independent of the package's own).
The J-scheme spectrum for total J is spec(M=J) minus spec(M=J+1) as multisets.
"""
from functools import lru_cache
from itertools import combinations
import numpy as np
import scipy.sparse as sp


@lru_cache(maxsize=None)
def _cg(j1, j2, J, m1, m2, M):
    from sympy import Rational
    from sympy.physics.quantum.cg import CG
    if m1 + m2 != M or abs(m1) > j1 or abs(m2) > j2 or abs(M) > J:
        return 0.0
    if not (abs(j1 - j2) <= J <= j1 + j2):
        return 0.0
    h = Rational(1, 2)
    return float(CG(j1 * h, m1 * h, j2 * h, m2 * h, J * h, M * h).doit())


class SDSpace:
    """All SDs of n identical nucleons in orbits j2 (bitmask, orbit-major, m ascending)."""

    def __init__(self, j2, spe, n):
        self.j2 = j2
        self.spe = spe
        self.states = [(o, m) for o, jj in enumerate(j2) for m in range(-jj, jj + 1, 2)]
        self.nsp = len(self.states)
        sds, ms = [], []
        for c in combinations(range(self.nsp), n):
            sds.append(sum(1 << i for i in c))
            ms.append(sum(self.states[i][1] for i in c))
        self.sds = np.array(sds, dtype=np.int64)
        self.M = np.array(ms)
        self.by_M = {m: np.sort(self.sds[self.M == m]) for m in np.unique(self.M)}

    def index(self, o, m):
        return self.states.index((o, m))


def _sgn(sd, k):
    return -1.0 if bin(sd & ((1 << k) - 1)).count("1") % 2 else 1.0


def _onebody(space, Min, i, k):
    """matrix of a+_i a_k from sector Min to sector Min + m_i - m_k (dense)."""
    src = space.by_M.get(Min)
    Mout = Min + space.states[i][1] - space.states[k][1]
    dst = space.by_M.get(Mout)
    if src is None or dst is None:
        return None, Mout
    pos = {int(s): n for n, s in enumerate(dst)}
    A = np.zeros((len(dst), len(src)))
    for c, s in enumerate(src):
        s = int(s)
        if not (s >> k) & 1:
            continue
        g = _sgn(s, k)
        s1 = s ^ (1 << k)
        if (s1 >> i) & 1:
            continue
        g *= _sgn(s1, i)
        A[pos[s1 | (1 << i)], c] += g
    return A, Mout


def _pair_amp(space, a, b, J, M):
    """coefficients on ordered sp pairs (i,j) of the normalised coupled pair (a b)JM."""
    j2 = space.j2
    N = 1 / np.sqrt(2.0) if a == b else 1.0
    amp = {}
    for ma in range(-j2[a], j2[a] + 1, 2):
        mb = M - ma
        if abs(mb) > j2[b]:
            continue
        c = _cg(j2[a], j2[b], J, ma, mb, M)
        if c == 0.0:
            continue
        i, j = space.index(a, ma), space.index(b, mb)
        if i == j:
            continue
        amp[(i, j)] = amp.get((i, j), 0.0) + N * c
    return amp


def _like_particle(space, inter, Msec):
    """H_pp (or H_nn) including SPE, dense, on sector Msec."""
    sds = space.by_M[Msec]
    pos = {int(s): n for n, s in enumerate(sds)}
    n = len(sds)
    H = np.diag([sum(space.spe[space.states[k][0]] for k in range(space.nsp) if (int(s) >> k) & 1) for s in sds])
    norb = len(space.j2)
    for a in range(norb):
        for b in range(a, norb):
            for c in range(norb):
                for d in range(c, norb):
                    for J in range(0, 2 * max(space.j2) + 1, 2):
                        V = inter.V(a, b, c, d, J, 1)
                        if V == 0.0:
                            continue
                        for M in range(-J, J + 1, 2):
                            A = _pair_amp(space, a, b, J, M)
                            B = _pair_amp(space, c, d, J, M)
                            if not A or not B:
                                continue
                            for col, s in enumerate(sds):
                                s = int(s)
                                for (k, l), y in B.items():       # A_JM(cd) = sum y a_l a_k
                                    if not ((s >> k) & 1 and (s >> l) & 1):
                                        continue
                                    g = _sgn(s, k)
                                    s1 = s ^ (1 << k)
                                    g *= _sgn(s1, l)
                                    s2 = s1 ^ (1 << l)
                                    for (i, j), x in A.items():   # A+ = sum x a+_i a+_j
                                        if (s2 >> i) & 1 or (s2 >> j) & 1:
                                            continue
                                        h = g * _sgn(s2, j)
                                        s3 = s2 | (1 << j)
                                        h *= _sgn(s3, i)
                                        s4 = s3 | (1 << i)
                                        H[pos[s4], col] += V * x * y * h
    return H


def mscheme_hamiltonian(inter, nprot, nneut, M2):
    """Dense product-basis Hamiltonian at total 2M, rows ordered (M_p sector, proton SD, neutron SD)."""
    spc = inter.space
    P = SDSpace(spc.j2, spc.spe, nprot)
    N = SDSpace(spc.j2, spc.spe, nneut)
    sectors = [(mp, M2 - mp) for mp in sorted(P.by_M) if (M2 - mp) in N.by_M]
    offs, tot = {}, 0
    for mp, mn in sectors:
        offs[mp] = tot
        tot += len(P.by_M[mp]) * len(N.by_M[mn])
    H = np.zeros((tot, tot))
    hp = {mp: _like_particle(P, inter, mp) for mp, _ in sectors} if nprot > 1 else None
    hn = {mn: _like_particle(N, inter, mn) for _, mn in sectors} if nneut > 1 else None
    for mp, mn in sectors:
        dp, dn = len(P.by_M[mp]), len(N.by_M[mn])
        o = offs[mp]
        Hp = hp[mp] if hp else np.diag([sum(spc.spe[P.states[k][0]] for k in range(P.nsp) if (int(s) >> k) & 1) for s in P.by_M[mp]])
        Hn = hn[mn] if hn else np.diag([sum(spc.spe[N.states[k][0]] for k in range(N.nsp) if (int(s) >> k) & 1) for s in N.by_M[mn]])
        H[o:o + dp * dn, o:o + dp * dn] += np.kron(Hp, np.eye(dn)) + np.kron(np.eye(dp), Hn)
    # pn part
    norb = spc.norb
    j2 = spc.j2
    for a in range(norb):
        for b in range(norb):
            for c in range(norb):
                for d in range(norb):
                    for J in range(0, 2 * max(j2) + 1, 2):
                        Vpn = 0.5 * np.sqrt((1 + (a == b)) * (1 + (c == d))) * sum(inter.V(a, b, c, d, J, T) for T in (0, 1))
                        if Vpn == 0.0:
                            continue
                        for M in range(-J, J + 1, 2):
                            for ma in range(-j2[a], j2[a] + 1, 2):
                                mb = M - ma
                                x = _cg(j2[a], j2[b], J, ma, mb, M) if abs(mb) <= j2[b] else 0.0
                                if x == 0.0:
                                    continue
                                for mc in range(-j2[c], j2[c] + 1, 2):
                                    md = M - mc
                                    y = _cg(j2[c], j2[d], J, mc, md, M) if abs(md) <= j2[d] else 0.0
                                    if y == 0.0:
                                        continue
                                    ip, kp = P.index(a, ma), P.index(c, mc)
                                    jn, ln = N.index(b, mb), N.index(d, md)
                                    for mp, mn in sectors:
                                        Ap, mp2 = _onebody(P, mp, ip, kp)
                                        An, mn2 = _onebody(N, mn, jn, ln)
                                        if Ap is None or An is None or mp2 not in offs:
                                            continue
                                        o_in, o_out = offs[mp], offs[mp2]
                                        blk = Vpn * x * y * np.kron(Ap, An)
                                        H[o_out:o_out + blk.shape[0], o_in:o_in + blk.shape[1]] += blk
    return H


def jscheme_spectrum_from_mscheme(inter, nprot, nneut, J2):
    """Eigenvalues of the total-J states: spec(M=J) minus spec(M=J+1) (as multisets)."""
    e0 = np.linalg.eigvalsh(mscheme_hamiltonian(inter, nprot, nneut, J2))
    try:
        e1 = np.linalg.eigvalsh(mscheme_hamiltonian(inter, nprot, nneut, J2 + 2))
    except ValueError:
        e1 = np.zeros(0)
    out = list(e0)
    for e in e1:
        k = int(np.argmin(np.abs(np.array(out) - e)))
        assert abs(out[k] - e) < 1e-8, ("unmatched M=J+1 level", e, out[k])
        out.pop(k)
    return np.array(sorted(out))
