"""Proton-neutron interaction in multipole (particle-hole) form.

Restates the formula of the reference's NuOp (src/NuOp/NuOp.f90:355-360):

    V_lam(s1 s3; s2 s4) = sum_{J,T} V_JT(j1 j2; j3 j4) (J+1) sqrt(lam+1)
                          (-1)^((j1+j4-J-lam)/2) W(j1 j2 j3 j4; J lam) d12 d34 / 2

with particles 1,3 of the "a" species and 2,4 of the "b" species, d12 = sqrt(2)
when orbits 1 and 2 coincide (likewise d34), lam from max(|j1-j3|,|j2-j4|) to
min(j1+j3, j2+j4) in steps of 1 (NuOp.f90:300-307), and T restricted to J+T odd
for coinciding orbits (NuOp.f90:318-331; enforced here by the absence of such
TBMEs).  Keys are the reference's 8-byte ``opn`` strings
(s1, s3, s2, s4, 2*lam, 0, 0, 0) with global shell numbers (NuOp.f90:273-320).
"""
import numpy as np

from .angmom import racah_w


def multipole_pn(inter):
    """Returns dict (o1, o3, o2, o4, lam2) -> V_lam with orbit indices (0-based)."""
    sp = inter.space
    j2 = sp.j2
    out = {}
    for o1 in range(sp.norb):
        for o2 in range(sp.norb):
            d12 = np.sqrt(2.0) if o1 == o2 else 1.0
            for o3 in range(sp.norb):
                for o4 in range(sp.norb):
                    d34 = np.sqrt(2.0) if o3 == o4 else 1.0
                    j1, jb, j3, j4 = j2[o1], j2[o2], j2[o3], j2[o4]
                    lmn = max(abs(j1 - j3), abs(jb - j4))
                    lmx = min(j1 + j3, jb + j4)
                    for lam in range(lmx, lmn - 1, -2):
                        s = 0.0
                        for J2 in range(max(abs(j1 - jb), abs(j3 - j4)), min(j1 + jb, j3 + j4) + 1, 2):
                            for T in (0, 1):
                                V = inter.V(o1, o2, o3, o4, J2, T)
                                if V == 0.0:
                                    continue
                                ph = -1.0 if ((j1 + j4 - J2 - lam) // 2) % 2 else 1.0
                                s += (V * (J2 + 1) * np.sqrt(lam + 1.0) * ph
                                      * racah_w(j1, jb, j3, j4, J2, lam) * d12 * d34 / 2.0)
                        out[(o1, o3, o2, o4, lam)] = s
    return out


def racah_weight(J2al, J2bl, J2ar, J2br, J2, lam2):
    """Recoupling weight of the pn product, as in src/NuLnz/NuCoreX.f90:1114-1126:
    (-1)^((Jal+Jbr-J-lam)/2) W(Jal Jbl Jar Jbr; J lam) sqrt(lam+1)."""
    w = racah_w(J2al, J2bl, J2ar, J2br, J2, lam2)
    if w == 0.0:
        return 0.0
    ph = -1.0 if ((J2al + J2br - J2 - lam2) // 2) % 2 else 1.0
    return ph * w * np.sqrt(lam2 + 1.0)


def op_order(vlam):
    """The order of the pn multipole operators in nsx_problem.op_keys (sorted labels)."""
    return sorted(vlam)


def op_values(vlam, order):
    """Multipole values in a given operator order (0 for labels the dict does not hold)."""
    import numpy as np
    return np.array([vlam.get(k, 0.0) for k in order], dtype=np.float64)
