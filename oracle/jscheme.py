"""FP64 CPU oracle of the pn-factorised J-scheme H.v (test infrastructure only).

A plain restatement of the reference's product, reading the reference-format
files with its own record reader, so that the CUDA path (libnsx) is checked
against an independent implementation of both the file parsing and the
arithmetic.  It follows, step by step:

* block list, offsets and parity mask    src/NuLnz/NuCoreX.f90:926-1030
* Racah weights racahs                    src/NuLnz/NuCoreX.f90:1071-1126
* pn table (drdbh)                        src/NuLnz/NuCoreX.f90:1428-1577
* density reading, masks and sub-blocks   src/NuLnz/NuCoreX.f90:1144-1206, src/NuCommonX/NuCommonX.f90:609-636
* like-particle segments                  src/NuLnz/NuCoreX.f90:1216-1319
* multiplyx / single_productm / single_product1: for every (output block,
  J_ar, proton operator a): T = sum_b w_b C_h rho_b^T, out += rho_a T
                                          src/NuLnz/NuCoreX.f90:128-226, src/NuCommonX/NuCommonX.f90:745-919
* multiplya / multiplyb (mulmtx)          src/NuLnz/NuCoreX.f90:76-125, src/NuCommonX/NuCommonX.f90:1009-1104

Densities, matrices and the multipole interaction are used in FP64 after
reading (the files store FP32, the .oph FP64).  Racah coefficients come from
sympy (independent of the product's own 6-j code).  The arithmetic is dense
NumPy/SciPy-sparse per block; it is meant for the small and mid-size workloads.
"""
import struct
from functools import lru_cache
import numpy as np
import scipy.sparse as sp


def _records(path):
    data = open(path, "rb").read()
    p, out = 0, []
    while p < len(data):
        (n,) = struct.unpack_from("<i", data, p)
        out.append(data[p + 4:p + 4 + n])
        (n2,) = struct.unpack_from("<i", data, p + 4 + n)
        assert n == n2, path
        p += 8 + n
    return out


AN = "0123456789_$cdefghijklmnopqrstuvwxyz@ABCDEFGHIJKLMNMPQRSTUVWXYZ\xa3a%^&=b-+#"


def _code(i, j, k):
    return "".join(AN[x + 72 if x < 0 else x] for x in (i, j, k))


def _trunc2(n):
    return int(n / 2)


@lru_cache(maxsize=None)
def racah_weight(Jal, Jbl, Jar, Jbr, J, lam):
    """(-1)^((Jal+Jbr-J-lam)/2) W(Jal Jbl Jar Jbr; J lam) sqrt(lam+1), twice-values; W via sympy 6-j."""
    from sympy import Rational
    from sympy.physics.wigner import wigner_6j
    h = Rational(1, 2)
    six = float(wigner_6j(Jal * h, Jbl * h, J * h, Jbr * h, Jar * h, lam * h))
    if six == 0.0:
        return 0.0
    W = six * (-1) ** (((Jal + Jbl + Jar + Jbr) // 2) % 2)
    ph = (-1) ** (((Jal + Jbr - J - lam) // 2) % 2)
    return ph * W * np.sqrt(lam + 1.0)


class Species:
    def __init__(self, base, like, T2, nmp, xtra, shell_parity):
        r = _records(base + ".tri")
        nsp, minJ2, maxJ2 = struct.unpack_from("<3i", r[0], 0)
        self.nsp, self.minJ2, self.maxJ2 = nsp, minJ2, maxJ2
        nJ = (maxJ2 - minJ2) // 2 + 1
        self.njt = np.frombuffer(r[1], dtype="<i4").reshape(nJ, nsp)
        occ = np.frombuffer(r[2], dtype="<i2").reshape(nsp, 32)
        par = np.ones(nsp, dtype=int)
        for i, s in enumerate(shell_parity):
            par *= np.where((occ[:, i] % 2 == 1) & (s < 0), -1, 1)
        self.par = par
        self.poff = {}
        for k in range(nJ):
            self.poff[minJ2 + 2 * k] = np.concatenate([[0], np.cumsum(self.njt[k])])
        # densities
        r = _records(base + ".trd")
        trdd = struct.unpack_from("<i", r[0], 0)[0]
        words = struct.unpack_from("<i", r[0], 12)[0]
        self.rho = {}
        if trdd:
            keys = [r[1][8 * k:8 * k + 8] for k in range(trdd)]
            dims = np.frombuffer(r[2], dtype="<i4")
            rec = 3
            for k in range(trdd):
                if dims[k] == 0:
                    continue
                vals = np.frombuffer(r[rec], dtype="<f4").astype(np.float64)
                vals = np.where(np.abs(vals) < 1e-11, 0.0, vals)
                masks = np.frombuffer(r[rec + 1], dtype="<u4").reshape(nsp, words)
                rec += 2
                J2l, J2r, sl, sr, lam = keys[k][:5]
                M = np.zeros((self.dim(J2l), self.dim(J2r)))
                p = 0
                for pr in range(nsp):
                    for pl in range(nsp):
                        if (masks[pr, pl // 32] >> np.uint32(pl % 32)) & 1:
                            nl, nr = self.n(pl, J2l), self.n(pr, J2r)
                            blk = vals[p:p + nl * nr].reshape(nr, nl).T
                            ol, orr = self.poff[J2l][pl], self.poff[J2r][pr]
                            M[ol:ol + nl, orr:orr + nr] = blk
                            p += nl * nr
                assert p == len(vals)
                self.rho[(J2l, J2r, sl, sr, lam)] = sp.csr_matrix(M)
        # like-particle H per J
        self.H = {}
        for J2 in range(minJ2, maxJ2 + 1, 2):
            name = like + _code(J2 // 2, T2 // 2, _trunc2(nmp) + 36) + xtra
            g = _records(name + ".sgt")
            nseg = struct.unpack_from("<i", g[1], 0)[0]
            m = _records(name + ".mat")
            d = self.dim(J2)
            H = np.zeros((d, d))
            for rec in m[1:1 + nseg]:
                dimpt, dimptr, npl, npr = struct.unpack_from("<4i", rec, 0)
                M = np.frombuffer(rec[16:16 + 4 * dimpt * dimptr], dtype="<f4").astype(np.float64)
                M = M.reshape(dimpt, dimptr)   # [k_l, k_r]
                ol, orr = self.poff[J2][npl - 1], self.poff[J2][npr - 1]
                H[ol:ol + dimpt, orr:orr + dimptr] = M
                H[orr:orr + dimptr, ol:ol + dimpt] = M.T
            self.H[J2] = H

    def n(self, ip, J2):
        if J2 < self.minJ2 or J2 > self.maxJ2:
            return 0
        return int(self.njt[(J2 - self.minJ2) // 2, ip])

    def dim(self, J2):
        if J2 < self.minJ2 or J2 > self.maxJ2:
            return 0
        return int(self.njt[(J2 - self.minJ2) // 2].sum())


class Oracle:
    """H.v in FP64 from the files named by a generator manifest."""

    def __init__(self, man):
        sp_par = man["shell_parity"]
        self.A = Species(man["a"], man["like_a"], man["nprot"], -man["nprot"], "x", sp_par)
        self.B = Species(man["b"], man["like_b"], man["nneut"], man["nneut"], "x", sp_par)
        self.J2, self.parity = man["J2"], man["parity"]
        A, B, J2 = self.A, self.B, self.J2
        r = _records(man["int"] + ".oph")
        nop = struct.unpack_from("<i", r[0], 0)[0]
        renorm = float(open(man["int"] + ".spe").read().split("\n")[1])
        self.renorm = renorm
        self.vop = {}
        for rec in r[1:1 + nop]:
            key = tuple(rec[:5])
            v = struct.unpack_from("<d", rec, 8)[0]
            self.vop[key] = (0.0 if abs(v) < 1e-10 else v) * renorm
        blocks = []
        for ja in range(A.minJ2, A.maxJ2 + 1, 2):
            lo, hi = max(abs(ja - J2), B.minJ2), min(ja + J2, B.maxJ2)
            lo += (lo - B.minJ2) % 2
            for jb in range(lo, hi + 1, 2):
                blocks.append((ja, jb))
        self.blocks = sorted(blocks)
        dims = [A.dim(a) * B.dim(b) for a, b in self.blocks]
        self.off = np.concatenate([[0], np.cumsum(dims)]).astype(int)
        self.dim = int(self.off[-1])
        lc = np.zeros(self.dim, dtype=bool)
        for k, (ja, jb) in enumerate(self.blocks):
            pa = np.concatenate([[A.par[ip]] * A.n(ip, ja) for ip in range(A.nsp)] + [np.zeros(0)])
            pb = np.concatenate([[B.par[ip]] * B.n(ip, jb) for ip in range(B.nsp)] + [np.zeros(0)])
            m = np.ones((len(pa), len(pb)), dtype=bool) if self.parity == 0 else (pa[:, None] * pb[None, :] == self.parity)
            lc[self.off[k]:self.off[k + 1]] = m.T.ravel()
        self.lcoef = lc
        # pn table: (out block, a-key) -> list of (b-key, in block, weight)
        bidx = {b: i for i, b in enumerate(self.blocks)}
        self.table = []
        for bl, (jal, jbl) in enumerate(self.blocks):
            for ka in A.rho:
                if ka[0] != jal:
                    continue
                jar, sal, sar, lam = ka[1], ka[2], ka[3], ka[4]
                ents = []
                for kb in B.rho:
                    if kb[0] != jbl or kb[4] != lam:
                        continue
                    jbr = kb[1]
                    hb = bidx.get((jar, jbr))
                    if hb is None:
                        continue
                    w = racah_weight(jal, jbl, jar, jbr, J2, lam)
                    v = self.vop.get((sal, sar, kb[2], kb[3], lam), 0.0)
                    if w == 0.0 or v == 0.0:
                        continue
                    ents.append((kb, hb, v * w))
                if ents:
                    self.table.append((bl, ka, ents))

    def block(self, x, k):
        ja, jb = self.blocks[k]
        return x[self.off[k]:self.off[k + 1]].reshape(self.B.dim(jb), self.A.dim(ja)).T

    def matvec(self, x, out_blocks=None):
        """H x; with out_blocks (indices into self.blocks) only those output blocks' rows are
        formed and the others are zero (one output-block shard's share)."""
        x = np.asarray(x, dtype=np.float64)
        y = np.zeros_like(x)
        A, B = self.A, self.B
        own = set(range(len(self.blocks))) if out_blocks is None else set(out_blocks)
        for k, (ja, jb) in enumerate(self.blocks):
            if k not in own:
                continue
            C = self.block(x, k)
            if C.size == 0:
                continue
            out = A.H[ja] @ C + C @ B.H[jb]
            y[self.off[k]:self.off[k + 1]] = out.T.ravel()
        for bl, ka, ents in self.table:
            if bl not in own:
                continue
            T = None
            for kb, hb, w in ents:
                Ch = self.block(x, hb)
                t = w * (B.rho[kb] @ Ch.T).T
                T = t if T is None else T + t
            out = A.rho[ka] @ T
            y[self.off[bl]:self.off[bl + 1]] += np.asarray(out).T.ravel()
        return y

    def flops(self):
        """Reference-order flop count of one H.v (the axpy loops of NuCoreX/NuCommonX)."""
        f = 0.0
        for bl, ka, ents in self.table:
            dbl = self.B.dim(self.blocks[bl][1])
            for kb, hb, w in ents:
                f += 2.0 * self.A.dim(self.blocks[hb][0]) * self.B.rho[kb].nnz
            f += 2.0 * dbl * self.A.rho[ka].nnz
        return f


def read_dop_terms(path):
    """The .dop file of NuDiop (list-directed text): {(2lam, parity, eigenvector number): (e, [(s1, s3,
    s2, s4, u), ...])} -- the layout read by src/NuTRLZ/NuCoreXZ.f90:1637-1650."""
    tok = open(path).read().split()
    p = [0]

    def nxt(f=int):
        p[0] += 1
        return f(tok[p[0] - 1])

    out = {}
    max_lmo = nxt()
    for _ in range(2 * (max_lmo // 2 + 1)):
        lam, par, nel = nxt(), nxt(), nxt()
        for i in range(1, nel + 1):
            e, nle = nxt(float), nxt()
            comps = [(nxt(), nxt(), nxt(), nxt(), nxt(float)) for _ in range(nle)]
            out[(lam, par, i)] = (e, comps)
    return out


class OracleZ(Oracle):
    """H.v with NuTRLZ's compressed pn interaction (src/NuTRLZ/NuCoreXZ.f90:1613-1887 prd, table
    :1475-1611): the densities folded into combined operators, proton e*renorm*u_e(a)*rho_a and
    neutron u_e(b)*rho_b, paired by equal (2lam, parity, e) with the Racah weight alone."""

    def __init__(self, man, dop_path):
        super().__init__(man)
        A, B, J2 = self.A, self.B, self.J2
        terms = read_dop_terms(dop_path)
        comb_a, comb_b = {}, {}
        for (lam, par, i), (e, comps) in terms.items():
            for ja in range(A.minJ2, A.maxJ2 + 1, 2):
                for jr in range(A.minJ2, A.maxJ2 + 1, 2):
                    M = None
                    for s1, s3, s2, s4, u in comps:
                        r = A.rho.get((ja, jr, s1, s3, lam))
                        if r is not None:
                            M = (e * self.renorm * u) * r if M is None else M + (e * self.renorm * u) * r
                    if M is not None:
                        comb_a[(ja, jr, lam, par, i)] = M.tocsr()
            for jb in range(B.minJ2, B.maxJ2 + 1, 2):
                for jr in range(B.minJ2, B.maxJ2 + 1, 2):
                    M = None
                    for s1, s3, s2, s4, u in comps:
                        r = B.rho.get((jb, jr, s2, s4, lam))
                        if r is not None:
                            M = u * r if M is None else M + u * r
                    if M is not None:
                        comb_b[(jb, jr, lam, par, i)] = M.tocsr()
        bidx = {b: i for i, b in enumerate(self.blocks)}
        self.table = []
        self.rho_a_z, self.rho_b_z = comb_a, comb_b
        for bl, (jal, jbl) in enumerate(self.blocks):
            for ka in comb_a:
                if ka[0] != jal:
                    continue
                jar = ka[1]
                ents = []
                for kb in comb_b:
                    if kb[0] != jbl or kb[2:] != ka[2:]:
                        continue
                    hb = bidx.get((jar, kb[1]))
                    if hb is None:
                        continue
                    w = racah_weight(jal, jbl, jar, kb[1], J2, ka[2])
                    if w != 0.0:
                        ents.append((kb, hb, w))
                if ents:
                    self.table.append((bl, ka, ents))

    def matvec(self, x):
        x = np.asarray(x, dtype=np.float64)
        y = np.zeros_like(x)
        A, B = self.A, self.B
        for k, (ja, jb) in enumerate(self.blocks):
            C = self.block(x, k)
            if C.size == 0:
                continue
            y[self.off[k]:self.off[k + 1]] = (A.H[ja] @ C + C @ B.H[jb]).T.ravel()
        for bl, ka, ents in self.table:
            T = None
            for kb, hb, w in ents:
                t = w * (self.rho_b_z[kb] @ self.block(x, hb).T).T
                T = t if T is None else T + t
            y[self.off[bl]:self.off[bl + 1]] += np.asarray(self.rho_a_z[ka] @ T).T.ravel()
        return y
