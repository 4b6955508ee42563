"""Assembly of one J-scheme pn problem from a model space and an interaction.

The vector layout is the reference's (src/NuLnz/NuCoreX.f90:926-1030):
blocks b = (2Ja, 2Jb) with |Ja-Jb| <= J <= Ja+Jb in ascending (2Ja, 2Jb) order
(the SOrder string order of char(2Ja)//char(2Jb)); inside a block the
coefficients form a d_a(Ja) x d_b(Jb) column-major matrix whose rows run over
proton partitions in order (nJT states each) and whose columns run over neutron
partitions in order.  Both parities are stored; ``lcoef`` marks the entries of
the requested parity.
"""
import numpy as np

from .angmom import triangle
from .species import Species
from .pnint import multipole_pn


class JProblem:
    def __init__(self, space, inter, nprot, nneut, J2, parity, renorm=1.0, lam_max=None):
        self.space = space
        self.inter = inter
        self.J2 = J2
        self.parity = parity
        self.renorm = renorm
        self.A = Species(space.j2, space.parity, space.spe, nprot, shell_offset=0)
        self.rhoA = self.A.densities(lam_max)
        self.segA = self.A.hamiltonian_segments(inter, renorm)
        if nneut == nprot:
            # same orbits and interaction for both species: share the work, shift the shell numbers
            import copy
            self.B = copy.copy(self.A)
            self.B.shell_offset = space.norb
            self.rhoB, self.segB = self.rhoA, self.segA
        else:
            self.B = Species(space.j2, space.parity, space.spe, nneut, shell_offset=space.norb)
            self.rhoB = self.B.densities(lam_max)
            self.segB = self.B.hamiltonian_segments(inter, renorm)
        self.vlam = multipole_pn(inter)
        self._blocks()

    @classmethod
    def from_workload(cls, w, inter=None, **kw):
        from .space import gaussian_interaction
        if inter is None:
            inter = gaussian_interaction(w.space, w.seed)
        return cls(w.space, inter, w.nprot, w.nneut, w.J2, w.parity, **kw)

    def _blocks(self):
        A, B, J2 = self.A, self.B, self.J2
        blocks = []
        for ja in range(A.minJ2, A.maxJ2 + 1, 2):
            lo = max(abs(ja - J2), B.minJ2)
            hi = min(ja + J2, B.maxJ2)
            lo += (lo - B.minJ2) % 2
            for jb in range(lo, hi + 1, 2):
                blocks.append((ja, jb))
        blocks.sort()
        self.blocks = blocks
        self.block_index = {b: i for i, b in enumerate(blocks)}
        self.dims = [(A.dimJ(ja), B.dimJ(jb)) for ja, jb in blocks]
        self.offsets = np.cumsum([0] + [da * db for da, db in self.dims])
        self.no_state = int(self.offsets[-1])
        # parity mask
        lc = np.zeros(self.no_state, dtype=bool)
        for k, (ja, jb) in enumerate(blocks):
            pa = np.concatenate([[A.part_parity[ip]] * A.njt(ip, ja) for ip in range(len(A.parts))] or [[]])
            pb = np.concatenate([[B.part_parity[ip]] * B.njt(ip, jb) for ip in range(len(B.parts))] or [[]])
            if len(pa) and len(pb):
                m = (pa[:, None] * pb[None, :]) == self.parity
                lc[self.offsets[k]:self.offsets[k + 1]] = m.T.ravel()   # column-major
        self.lcoef = lc

    # -- dense helpers used by the oracle checks ----------------------------------
    @staticmethod
    def part_offsets(S, J2):
        o = [0]
        for ip in range(len(S.parts)):
            o.append(o[-1] + S.njt(ip, J2))
        return o

    def dense_rho(self, S, rho, key):
        J2l, J2r = key[0], key[1]
        ol, orr = self.part_offsets(S, J2l), self.part_offsets(S, J2r)
        M = np.zeros((ol[-1], orr[-1]))
        for (ipl, ipr), blk in rho[key].items():
            M[ol[ipl]:ol[ipl + 1], orr[ipr]:orr[ipr + 1]] = blk
        return M

    def dense_like(self, S, segs, J2):
        o = self.part_offsets(S, J2)
        H = np.zeros((o[-1], o[-1]))
        for ipl, ipr, M in segs.get(J2, []):
            H[o[ipl]:o[ipl + 1], o[ipr]:o[ipr + 1]] = M
            if ipl != ipr:
                H[o[ipr]:o[ipr + 1], o[ipl]:o[ipl + 1]] = M.T
        return H
