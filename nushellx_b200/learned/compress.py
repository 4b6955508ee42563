"""Proton x neutron sub-blocks of a J-scheme vector and the compression of ground states.

Layout (the reference's, src/NuLnz/NuCoreX.f90:926-1030): block k = (2Ja, 2Jb) holds a
d_a x d_b column-major matrix whose rows run over proton partitions P (nJT(P, Ja) rows
each) and columns over neutron partitions Q.  Sub-block (k, P, Q) is the nJT(P, Ja) x
nJT(Q, Jb) piece of it; only pieces of the requested parity are kept (the others are
zero in every eigenvector).

Compression: K sub-blocks are kept, each with a unit shape u_s, and a ground state g is
represented by its projections w_s = <g|s, u_s>; the vector sum_s w_s u_s restores g up to
what lies outside the kept pieces and the change of shape within them.  Two ways to choose
them: from one reference state g_ref (its K heaviest sub-blocks, u_s = g_ref|s / |g_ref|s|),
or from a training set of ground states (the K sub-blocks of largest mean weight; u_s the
dominant left singular vector of the training restrictions g_v|s, which does not depend on
the arbitrary overall sign of each g_v).  The overall sign of a compressed state is fixed
on the first kept sub-block, in the order of decreasing mean weight, that holds at least a
tenth of its largest projection: that projection is made positive.
"""
import numpy as np


class SubBlocks:
    def __init__(self, P):
        """P: a JProblem (gen.problem) -- only its block list and partition sizes are used."""
        desc = []
        A, B = P.A, P.B
        for k, (ja, jb) in enumerate(P.blocks):
            oa, ob = P.part_offsets(A, ja), P.part_offsets(B, jb)
            da = oa[-1]
            for q in range(len(B.parts)):
                nq = ob[q + 1] - ob[q]
                if nq == 0:
                    continue
                for p in range(len(A.parts)):
                    npp = oa[p + 1] - oa[p]
                    if npp == 0:
                        continue
                    if P.parity and A.part_parity[p] * B.part_parity[q] != P.parity:
                        continue
                    desc.append((int(P.offsets[k]) + oa[p] + da * ob[q], da, npp, nq))
        self.desc = np.array(desc, dtype=np.int64).reshape(-1, 4)   # offset of (0,0), ld, rows, cols
        self.dim = int(P.no_state)
        self.index, self.start = element_index(self.desc)

    def __len__(self):
        return len(self.desc)

    def norms(self, v):
        v = np.asarray(v, dtype=np.float64)
        return np.sqrt(np.add.reduceat(v[self.index] ** 2, self.start[:-1]))


def element_index(desc):
    """Vector indices of the elements of the sub-blocks in desc (rows fastest), and the
    start of each sub-block in that list."""
    sizes = desc[:, 2] * desc[:, 3]
    start = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    idx = np.empty(int(start[-1]), dtype=np.int64)
    for s, (off, ld, nr, nc) in enumerate(desc):
        i = np.arange(nr, dtype=np.int64)[:, None]
        j = np.arange(nc, dtype=np.int64)[None, :]
        idx[start[s]:start[s + 1]] = (off + i + ld * j).ravel(order="F")
    return idx, start


class Compressor:
    def __init__(self, desc, shapes, dim, rank=None):
        """desc: [K, 4] kept sub-blocks (offset, ld, rows, cols); shapes: their unit shapes,
        concatenated (rows fastest); dim: vector length; rank: the order of the kept
        sub-blocks by decreasing weight (used for the sign convention; default: as given)."""
        self.desc = np.asarray(desc, dtype=np.int64).reshape(-1, 4)
        self.shapes = np.asarray(shapes, dtype=np.float64)
        self.dim = int(dim)
        self.index, self.start = element_index(self.desc)
        assert len(self.shapes) == len(self.index)
        self.lengths = np.diff(self.start)
        self.rank = np.arange(len(self.desc)) if rank is None else np.asarray(rank, dtype=np.int64)

    @classmethod
    def from_training(cls, sub, G, K=256):
        """G: training ground states [n, dim] (a torch tensor on the GPU or a numpy array)."""
        import torch
        Gt = torch.as_tensor(G)
        e_elem = torch.zeros(Gt.shape[1], dtype=torch.float64, device=Gt.device)
        for c in range(0, Gt.shape[0], 32):
            e_elem += (Gt[c:c + 32].double() ** 2).sum(0)
        e_elem = (e_elem / Gt.shape[0]).cpu().numpy()
        e = np.add.reduceat(e_elem[sub.index], sub.start[:-1])   # mean weight per sub-block
        order = np.argsort(-e, kind="stable")[:K]           # by decreasing mean weight
        keep = np.sort(order)                                # stored in vector order
        rank = np.searchsorted(keep, order)                  # positions of the ranked blocks in keep
        desc = sub.desc[keep]
        sidx, sstart = element_index(desc)
        shapes = np.zeros(len(sidx))
        for s in range(len(desc)):
            cols = torch.as_tensor(sidx[sstart[s]:sstart[s + 1]], device=Gt.device)
            M = Gt[:, cols].double().T                       # [n_s, n]
            if M.shape[0] == 1:
                u = torch.ones(1, dtype=torch.float64, device=Gt.device)
            else:
                U, S, _ = torch.linalg.svd(M, full_matrices=False)
                u = U[:, 0]
            shapes[sstart[s]:sstart[s + 1]] = u.cpu().numpy()
        return cls(desc, shapes, sub.dim, rank)

    @classmethod
    def from_reference(cls, sub, g_ref, K=256):
        n = sub.norms(g_ref)
        keep = np.sort(np.argsort(-n, kind="stable")[:K])      # K largest, in vector order
        desc = sub.desc[keep]
        idx, start = element_index(desc)
        u = np.asarray(g_ref, dtype=np.float64)[idx]
        u /= np.repeat(n[keep], np.diff(start))
        return cls(desc, u, sub.dim, np.searchsorted(keep, np.argsort(-n, kind="stable")[:K]))

    @property
    def K(self):
        return len(self.desc)

    def compress(self, g):
        gs = np.asarray(g, dtype=np.float64)[self.index]
        w = np.add.reduceat(gs * self.shapes, self.start[:-1])
        big = np.abs(w[self.rank]) >= 0.1 * np.abs(w).max()
        lead = self.rank[int(np.argmax(big))]
        return w if w[lead] >= 0 else -w

    def decompress(self, w):
        x = np.zeros(self.dim)
        x[self.index] = self.shapes * np.repeat(np.asarray(w, dtype=np.float64), self.lengths)
        return x
