"""One nucleon species (protons or neutrons) of the pn J-scheme basis.

This is the synthetic replacement for the reference's NuBasis -> NuProj ->
NuOper/NuMatrix/NuOrth -> NuOpm/NuOpd chain for one species:

* Slater determinants (SDs) are bitmasks over single-particle states ordered
  orbit-major, m ascending; the fermion sign of a_k / a^+_k is (-1)^(number of
  occupied states with index below k).
* A *partition* is the occupation of each orbit (the reference's
  ``spartition``, src/NuCommon/NuCommon.f90:200-213).  J-scheme states are
  built per partition: the highest-weight states |J, M=J> are the null space of
  J+ from the M=J sector to the M=J+1 sector.  The basis inside each null
  space is made canonical (pivoted Gram-Schmidt of the null-space projector in
  SD order) so that it does not depend on the SVD's arbitrary rotation.
* ``nJT[p][J2]`` is the number of J-states of partition p (the reference's
  ``nJT(partition, J)``, src/NuLnz/NuCoreX.f90:850-867).
* One-body reduced densities follow NuOpd's definition
  (src/NuOpd/NuOpd.f90:422-449 with the m-scheme phase of
  src/NuOpm/NuOpm.f90:466-467):

      rho(Jl,Jr; l,r; lam)[a,b] = sum_{ml,mr} <jl ml jr -mr | lam mu> (-1)^(jr-mr)
                                  <Jl Jl a| a+_{l ml} a_{r mr} |Jr Jr b>
                                  / <Jl Jl Jr -Jr | lam mu>,        mu = Jl - Jr.

* The like-particle Hamiltonian per J (the reference's .mat segments,
  src/NuOrth/NuOrth.f90:179-230) is <J J a|H|J J b> in the M=J sector with
  H = sum SPE*n + T=1 two-body part.
"""
from itertools import product, combinations
import numpy as np
from scipy.linalg import null_space

from .angmom import cg

_U1 = np.uint64(1)


def _popcount_below(sd, k):
    """number of set bits of sd strictly below bit k (vectorised over sd)."""
    mask = np.uint64((1 << k) - 1)
    return np.bitwise_count(sd & mask).astype(np.int64)


def _sign(n):
    return 1.0 - 2.0 * (n & 1)


def canonical_basis(Q, tol=1e-8):
    """Deterministic orthonormal basis of span(Q): pivoted Gram-Schmidt of the
    projector Q Q^T taking columns in index order."""
    n, d = Q.shape
    if d == 0:
        return Q
    P = Q @ Q.T
    out = []
    for i in range(n):
        v = P[:, i].copy()
        for u in out:
            v -= u * (u @ v)
        for u in out:          # second pass for stability
            v -= u * (u @ v)
        nv = np.linalg.norm(v)
        if nv > tol:
            out.append(v / nv)
            if len(out) == d:
                break
    B = np.array(out).T
    assert B.shape == (n, d), (B.shape, d)
    return B


class Species:
    def __init__(self, j2, parity, spe, n, shell_offset):
        self.j2 = list(j2)
        self.par = list(parity)
        self.spe = list(spe)
        self.n = n
        self.norb = len(j2)
        self.shell_offset = shell_offset  # global shell number = offset + orbit + 1
        sp_orb, sp_m2 = [], []
        self.orb_first = []
        for o, jj in enumerate(self.j2):
            self.orb_first.append(len(sp_orb))
            for m2 in range(-jj, jj + 1, 2):
                sp_orb.append(o)
                sp_m2.append(m2)
        self.sp_orb = np.array(sp_orb)
        self.sp_m2 = np.array(sp_m2)
        self.nsp = len(sp_orb)
        assert self.nsp <= 63
        self._build_partitions()
        self._build_sds()
        self._project()

    # -- partitions and SDs ---------------------------------------------------
    def _build_partitions(self):
        caps = [jj + 1 for jj in self.j2]
        parts = []
        for occ in product(*[range(c + 1) for c in caps]):
            if sum(occ) == self.n:
                parts.append(tuple(occ))
        self.parts = parts
        self.part_index = {p: i for i, p in enumerate(parts)}
        self.part_parity = [int(np.prod([self.par[o] ** k for o, k in enumerate(p)])) for p in parts]

    def sp_index(self, o, m2):
        return self.orb_first[o] + (m2 + self.j2[o]) // 2

    def _orbit_combos(self, o, k):
        jj = self.j2[o]
        first = self.orb_first[o]
        masks, ms = [], []
        for c in combinations(range(jj + 1), k):
            masks.append(sum(1 << (first + i) for i in c))
            ms.append(sum(2 * i - jj for i in c))
        return np.array(masks, dtype=np.uint64), np.array(ms, dtype=np.int64)

    def _build_sds(self):
        self.sectors = {}      # (p, M2) -> sorted uint64 array
        self.maxM2 = {}
        for ip, occ in enumerate(self.parts):
            sd = np.zeros(1, dtype=np.uint64)
            M = np.zeros(1, dtype=np.int64)
            for o, k in enumerate(occ):
                cm, cmm = self._orbit_combos(o, k)
                sd = (sd[:, None] | cm[None, :]).ravel()
                M = (M[:, None] + cmm[None, :]).ravel()
            self.maxM2[ip] = int(M.max())
            for m2 in np.unique(M):
                if m2 < 0:
                    continue
                self.sectors[(ip, int(m2))] = np.sort(sd[M == m2])
        mx = max(self.maxM2.values())
        self.minJ2 = self.n % 2
        self.maxJ2 = mx

    def sector(self, ip, M2):
        return self.sectors.get((ip, M2), np.zeros(0, dtype=np.uint64))

    # -- J projection -----------------------------------------------------------
    def _jplus(self, ip, M2):
        """Dense J+ matrix from sector M2 to M2+2 of partition ip."""
        src = self.sector(ip, M2)
        dst = self.sector(ip, M2 + 2)
        Jp = np.zeros((len(dst), len(src)))
        if len(dst) == 0 or len(src) == 0:
            return Jp
        cols = np.arange(len(src))
        for o, jj in enumerate(self.j2):
            for m2 in range(-jj, jj, 2):       # m -> m+1 inside orbit o
                k = self.sp_index(o, m2)
                has = (src >> np.uint64(k)) & _U1
                emp = 1 - ((src >> np.uint64(k + 1)) & _U1)
                sel = (has & emp).astype(bool)
                if not sel.any():
                    continue
                new = src[sel] ^ (_U1 << np.uint64(k)) ^ (_U1 << np.uint64(k + 1))
                idx = np.searchsorted(dst, new)
                coef = np.sqrt((jj * (jj + 2) - m2 * (m2 + 2)) / 4.0)
                Jp[idx, cols[sel]] += coef    # adjacent states: fermion sign +1
        return Jp

    def _project(self):
        self.HW = {}      # (ip, J2) -> (n_sector, nJT) orthonormal columns
        self.nJT = np.zeros((len(self.parts), (self.maxJ2 - self.minJ2) // 2 + 1), dtype=np.int64)
        for ip in range(len(self.parts)):
            for J2 in range(self.minJ2, self.maxM2[ip] + 1, 2):
                n0 = len(self.sector(ip, J2))
                n1 = len(self.sector(ip, J2 + 2))
                d = n0 - n1
                if d <= 0:
                    continue
                Jp = self._jplus(ip, J2)
                if Jp.shape[0] == 0:
                    Q = np.eye(n0)
                else:
                    Q = null_space(Jp, rcond=1e-10)
                assert Q.shape[1] == d, (ip, J2, Q.shape, d)
                self.HW[(ip, J2)] = canonical_basis(Q)
                self.nJT[ip, (J2 - self.minJ2) // 2] = d

    def njt(self, ip, J2):
        if J2 < self.minJ2 or J2 > self.maxJ2:
            return 0
        return int(self.nJT[ip, (J2 - self.minJ2) // 2])

    def dimJ(self, J2):
        return int(sum(self.njt(ip, J2) for ip in range(len(self.parts))))

    def J2_values(self):
        return [J2 for J2 in range(self.minJ2, self.maxJ2 + 1, 2) if self.dimJ(J2) > 0]

    # -- one-body transitions -------------------------------------------------
    def hop(self, src, k_from, k_to):
        """Apply a+_{k_to} a_{k_from} to the SDs in src.  Returns (mask, new_sds, sign)."""
        has = ((src >> np.uint64(k_from)) & _U1).astype(bool)
        sd1 = src ^ (_U1 << np.uint64(k_from))
        if k_to == k_from:
            ok = has
        else:
            ok = has & ~((sd1 >> np.uint64(k_to)) & _U1).astype(bool)
        s = src[ok]
        sd1 = sd1[ok]
        sg = _sign(_popcount_below(s, k_from)) * _sign(_popcount_below(sd1, k_to))
        new = sd1 | (_U1 << np.uint64(k_to))
        return ok, new, sg

    def partner(self, ip, l, r):
        """Left partition reached from partition ip by a+_l a_r, or None."""
        occ = list(self.parts[ip])
        if occ[r] == 0:
            return None
        occ[r] -= 1
        occ[l] += 1
        if occ[l] > self.j2[l] + 1:
            return None
        return self.part_index[tuple(occ)]

    def densities(self, lam_max=None):
        """All nonzero reduced one-body densities.

        Returns dict key=(J2l, J2r, l, r, lam2) -> dict (ipl, ipr) -> ndarray(nJT_l, nJT_r).
        """
        out = {}
        j2 = self.j2
        for l in range(self.norb):
            for r in range(self.norb):
                lams = [lm for lm in range(abs(j2[l] - j2[r]), j2[l] + j2[r] + 1, 2)]
                if lam_max is not None:
                    lams = [lm for lm in lams if lm <= lam_max]
                if not lams:
                    continue
                for ipr in range(len(self.parts)):
                    ipl = self.partner(ipr, l, r)
                    if ipl is None:
                        continue
                    for J2r in range(self.minJ2, self.maxM2[ipr] + 1, 2):
                        HWr = self.HW.get((ipr, J2r))
                        if HWr is None:
                            continue
                        srcs = self.sector(ipr, J2r)
                        for J2l in range(max(self.minJ2, J2r - j2[l] - j2[r]), min(self.maxM2[ipl], J2r + j2[l] + j2[r]) + 1, 2):
                            HWl = self.HW.get((ipl, J2l))
                            if HWl is None:
                                continue
                            lam_ok = [lm for lm in lams if abs(J2l - J2r) <= lm <= J2l + J2r]
                            if not lam_ok:
                                continue
                            dsts = self.sector(ipl, J2l)
                            mu = J2l - J2r
                            T = {lm: np.zeros((len(dsts), HWr.shape[1])) for lm in lam_ok}
                            for mr in range(-j2[r], j2[r] + 1, 2):
                                ml = mr + mu
                                if abs(ml) > j2[l]:
                                    continue
                                kf = self.sp_index(r, mr)
                                kt = self.sp_index(l, ml)
                                ok, new, sg = self.hop(srcs, kf, kt)
                                if not ok.any():
                                    continue
                                idx = np.searchsorted(dsts, new)
                                rows = HWr[ok] * sg[:, None]
                                ph = -1.0 if ((j2[r] - mr) // 2) % 2 else 1.0
                                acc = np.zeros((len(dsts), HWr.shape[1]))
                                np.add.at(acc, idx, rows)
                                for lm in lam_ok:
                                    c = cg(j2[l], j2[r], lm, ml, -mr, mu)
                                    if c != 0.0:
                                        T[lm] += (c * ph) * acc
                            for lm in lam_ok:
                                c1 = cg(J2l, J2r, lm, J2l, -J2r, mu)
                                if c1 == 0.0:
                                    continue
                                rho = HWl.T @ T[lm] / c1
                                key = (J2l, J2r, l, r, lm)
                                out.setdefault(key, {})[(ipl, ipr)] = rho
        return out

    # -- like-particle Hamiltonian -----------------------------------------------
    def two_body_table(self, inter):
        """Coefficients W[(i,j),(k,l)] (i<j, k<l) of H2 = sum W a+_i a+_j a_l a_k for the T=1 part."""
        j2 = self.j2
        npair = {}
        pairs = [(i, j) for i in range(self.nsp) for j in range(i + 1, self.nsp)]
        for n_, p in enumerate(pairs):
            npair[p] = n_
        # pair amplitudes P_{ab,J,M}[(i<j)] = N_ab (cg(i,j) - cg(j,i))
        amps = {}
        for a in range(self.norb):
            for b in range(a, self.norb):
                Nab = 1.0 / np.sqrt(2.0) if a == b else 1.0
                for J2 in range(abs(j2[a] - j2[b]), j2[a] + j2[b] + 1, 2):
                    if a == b and (J2 // 2) % 2 == 1:
                        continue
                    for M2 in range(-J2, J2 + 1, 2):
                        vec = {}
                        for ma in range(-j2[a], j2[a] + 1, 2):
                            mb = M2 - ma
                            if abs(mb) > j2[b]:
                                continue
                            c = cg(j2[a], j2[b], J2, ma, mb, M2)
                            if c == 0.0:
                                continue
                            i = self.sp_index(a, ma)
                            j = self.sp_index(b, mb)
                            if i == j:
                                continue
                            if i < j:
                                vec[(i, j)] = vec.get((i, j), 0.0) + Nab * c
                            else:
                                vec[(j, i)] = vec.get((j, i), 0.0) - Nab * c
                        amps[(a, b, J2, M2)] = vec
        W = {}
        for a in range(self.norb):
            for b in range(a, self.norb):
                for c_ in range(self.norb):
                    for d in range(c_, self.norb):
                        for J2 in range(0, 2 * max(j2) + 1, 2):
                            if (a, b, J2, J2) not in amps or (c_, d, J2, J2) not in amps:
                                continue
                            v = inter.V(a, b, c_, d, J2, 1)
                            if v == 0.0:
                                continue
                            for M2 in range(-J2, J2 + 1, 2):
                                A = amps[(a, b, J2, M2)]
                                B = amps[(c_, d, J2, M2)]
                                for pij, x in A.items():
                                    for pkl, y in B.items():
                                        key = (pij, pkl)
                                        W[key] = W.get(key, 0.0) + v * x * y
        return W

    def apply_table(self, sds, W, spe_diag=True):
        """Sparse matrix (rows, cols, vals) of H = SPE*n + sum W a+a+aa within one M sector."""
        rows, cols, vals = [], [], []
        idx_all = np.arange(len(sds))
        # one-body diagonal
        if spe_diag:
            diag = np.zeros(len(sds))
            for k in range(self.nsp):
                occ = ((sds >> np.uint64(k)) & _U1).astype(np.float64)
                diag += self.spe[self.sp_orb[k]] * occ
            rows.append(idx_all)
            cols.append(idx_all)
            vals.append(diag)
        by_kl = {}
        for (pij, pkl), w in W.items():
            if w != 0.0:
                by_kl.setdefault(pkl, []).append((pij, w))
        for (k, l), lst in by_kl.items():
            has = (((sds >> np.uint64(k)) & _U1) & ((sds >> np.uint64(l)) & _U1)).astype(bool)
            if not has.any():
                continue
            s0 = sds[has]
            c0 = idx_all[has]
            s1 = s0 ^ (_U1 << np.uint64(k))
            sg = _sign(_popcount_below(s0, k))
            s2 = s1 ^ (_U1 << np.uint64(l))
            sg = sg * _sign(_popcount_below(s1, l))
            for (i, j), w in lst:
                emp = ~((((s2 >> np.uint64(i)) & _U1) | ((s2 >> np.uint64(j)) & _U1)).astype(bool))
                if not emp.any():
                    continue
                s3 = s2[emp] | (_U1 << np.uint64(j))
                g = sg[emp] * _sign(_popcount_below(s2[emp], j))
                s4 = s3 | (_U1 << np.uint64(i))
                g = g * _sign(_popcount_below(s3, i))
                r = np.searchsorted(sds, s4)
                assert np.all(sds[np.minimum(r, len(sds) - 1)] == s4)
                rows.append(r)
                cols.append(c0[emp])
                vals.append(w * g)
        if not rows:
            return np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros(0)
        return np.concatenate(rows), np.concatenate(cols), np.concatenate(vals)

    def hamiltonian_segments(self, inter, renorm=1.0):
        """Like-particle H per J as partition segments.

        Returns dict J2 -> list of (ipl, ipr, M) with ipl <= ipr and M = <ipl states|H|ipr states>
        of shape (nJT(ipl,J), nJT(ipr,J)); SPE*occupancy on the diagonal of ipl==ipr segments
        (not renormalised), two-body part multiplied by renorm (src/NuOrth/NuOrth.f90:200-219).
        """
        import scipy.sparse as sp
        W = self.two_body_table(inter)
        segs = {}
        for J2 in self.J2_values():
            # the M=J sector over all partitions (H may lead into partitions without J states)
            allp = [ip for ip in range(len(self.parts)) if len(self.sector(ip, J2)) > 0]
            sds_list = [self.sector(ip, J2) for ip in allp]
            pos_of = {ip: k for k, ip in enumerate(allp)}
            plist = [ip for ip in allp if self.njt(ip, J2) > 0]
            sds_all = np.concatenate(sds_list)
            order = np.argsort(sds_all)
            sds_sorted = sds_all[order]
            r, c, v = self.apply_table(sds_sorted, W, spe_diag=False)
            n = len(sds_sorted)
            H = sp.csr_matrix((v, (r, c)), shape=(n, n))
            inv = np.empty(n, dtype=np.int64)
            inv[order] = np.arange(n)
            # block-diagonal HW in concatenated order
            offs = np.cumsum([0] + [len(s) for s in sds_list])
            out = []
            for ipa in plist:
                a = pos_of[ipa]
                HWa = self.HW[(ipa, J2)]
                ra = inv[offs[a]:offs[a + 1]]
                Ha = H[ra]
                for ipb in plist:
                    if ipb < ipa:
                        continue
                    if self.part_parity[ipa] != self.part_parity[ipb]:
                        continue
                    b = pos_of[ipb]
                    HWb = self.HW[(ipb, J2)]
                    rb = inv[offs[b]:offs[b + 1]]
                    blk = Ha[:, rb]
                    if blk.nnz == 0 and ipa != ipb:
                        continue
                    M = HWa.T @ (blk @ HWb) * renorm
                    if ipa == ipb:
                        diag0 = sum(self.spe[o] * k for o, k in enumerate(self.parts[ipa]))
                        M = M + diag0 * np.eye(M.shape[0])
                    elif np.abs(M).max() < 1e-12:
                        continue
                    out.append((ipa, ipb, M))
            segs[J2] = out
        return segs
