"""The compressed pn interaction of NuTRLZ: the .dop file of NuDiop.

NuDiop (src/NuDiop/NuDiop.f90) takes the multipole pn interaction V_lam(a; b) of the
.oph file -- a = proton orbit pair (s1, s3), b = neutron orbit pair (s2, s4) -- and, for
every (lam, parity) with parity the pairs' parity p1*p3 = p2*p4, diagonalises the square
matrix M[a, b] over the pairs that occur (the neutron pair of row i is the proton pair of
row i shifted by the number of proton shells, NuDiop.f90:126-140):

    M = sum_e e u_e u_e^T.

It keeps the eigenvalues with e / sqrt(lam+1) beyond the cut (> cut for positive e,
< -cut for negative e; NuDiop.f90:212-227) and, of each kept eigenvector, the components
with |u| > cutm (NuDiop.f90:232-247).  NuTRLZ then folds them into combined one-body
operators (NuCoreXZ.f90:1613-1887):

    proton  (e, lam, parity):  sum_a e * renorm * u_e(a) * rho_a
    neutron (e, lam, parity):  sum_b u_e(b) * rho_b,

and its pn table pairs the proton and neutron operators of the same e with the Racah weight
alone (NuCoreXZ.f90:1475-1611).  With no cut the compressed product is the exact one.

File layout (list-directed text, as NuDiop writes it): max_lmo; then for lam = 0, 2, ..
max_lmo and parity = -1, +1: "lam parity", the number of kept eigenvalues, and for each
eigenvalue (ascending): e, the number of kept components, and one line
"s1 s3 s2 s4 u" per component (proton shells 1..norb, neutron shells norb+1..2 norb).

The eigen-decomposition here is numpy's (not Numerical Recipes' tred2/tqli).
"""
import numpy as np


def diop(vlam, space, cut=0.0, cutm=0.0):
    """Returns [(lam2, parity, [(e, [(s1, s3, s2, s4, u), ...]), ...]), ...] in file order."""
    norb = space.norb
    par = space.parity
    max_lmo = max((k[4] for k in vlam), default=0)
    out = []
    for lam in range(0, max_lmo + 1, 2):
        for pt in (-1, 1):
            # M[(o1,o3), (o2,o4)]: ops with pair parities p1*p3 = p2*p4 = pt
            ent = {}
            for (o1, o3, o2, o4, lm), v in vlam.items():
                if lm != lam or par[o1] * par[o3] != pt or par[o2] * par[o4] != pt:
                    continue
                ent[((o1, o3), (o2, o4))] = ent.get(((o1, o3), (o2, o4)), 0.0) + v
            rows = sorted({a for (a, b), v in ent.items() if v != 0.0})
            cols = sorted({b for (a, b), v in ent.items() if v != 0.0})
            if not rows:
                out.append((lam, pt, []))
                continue
            if rows != cols:
                raise ValueError(f"lam {lam} parity {pt}: the pn multipole matrix is not square over its pairs")
            idx = {p: i for i, p in enumerate(rows)}
            M = np.zeros((len(rows), len(rows)))
            for (a, b), v in ent.items():
                if a in idx and b in idx:
                    M[idx[a], idx[b]] += v
            if np.abs(M - M.T).max() > 1e-9 * max(np.abs(M).max(), 1.0):
                raise ValueError(f"lam {lam} parity {pt}: the pn multipole matrix is not symmetric")
            e, U = np.linalg.eigh(0.5 * (M + M.T))
            rt = np.sqrt(lam + 1.0)
            kept = []
            for i in range(len(e)):
                if not ((e[i] / rt > cut and e[i] > 0.0) or (e[i] / rt < -cut and e[i] < 0.0)):
                    continue
                comps = []
                for j, (o1, o3) in enumerate(rows):
                    u = U[j, i]
                    if abs(u) > cutm:
                        comps.append((o1 + 1, o3 + 1, norb + o1 + 1, norb + o3 + 1, float(u)))
                kept.append((float(e[i]), comps))
            out.append((lam, pt, kept))
    return out


def write_dop(path, entries):
    max_lmo = max((lam for lam, _, _ in entries), default=0)
    with open(path, "w") as f:
        f.write(f"{max_lmo:4d}\n")
        for lam, pt, kept in entries:
            f.write(f"{lam:4d}{pt:4d}\n")
            f.write(f"{len(kept):4d}\n")
            for e, comps in kept:
                f.write(f"{e:11.7f}\n")
                f.write(f"{len(comps):6d}\n")
                for s1, s3, s2, s4, u in comps:
                    f.write(f"{s1:4d}{s3:4d}{s2:4d}{s4:4d}{u:11.7f}\n")


def read_dop(path):
    """The .dop file back as the structure diop() returns (list-directed: whitespace tokens)."""
    tok = open(path).read().split()
    p = 0

    def nxt():
        nonlocal p
        p += 1
        return tok[p - 1]

    max_lmo = int(nxt())
    out = []
    for _ in range(2 * (max_lmo // 2 + 1)):
        lam, pt = int(nxt()), int(nxt())
        kept = []
        for _ in range(int(nxt())):
            e = float(nxt())
            comps = []
            for _ in range(int(nxt())):
                comps.append((int(nxt()), int(nxt()), int(nxt()), int(nxt()), float(nxt())))
            kept.append((e, comps))
        out.append((lam, pt, kept))
    return out
