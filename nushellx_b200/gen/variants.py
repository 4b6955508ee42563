"""Interaction variants TBME = base + sum_i lam_i * P_i of one J-scheme problem.

The densities, the block structure and hence the solver's plan do not depend on the
interaction; the pn multipole values and the like-particle .mat segments do, linearly.
``InteractionFamily`` therefore evaluates them once for the base interaction and once
for each perturbation P_i (seeded Gaussian TBMEs drawn like the base, N(0,1)/sqrt(N_TBME)),
and a variant's operands are a linear combination of those arrays; a solver handle takes
them through ``Solver.set_interaction`` (nsx_set_interaction) without re-planning.
"""
import numpy as np

from .space import gaussian_interaction
from .pnint import multipole_pn, op_order, op_values
from .writer import segment_arrays


class InteractionFamily:
    def __init__(self, P, nperturb=8, seed0=1000):
        """P: the base JProblem; perturbation i uses the Gaussian seed seed0 + i."""
        self.P = P
        self.order = op_order(P.vlam)
        self.perturb = [gaussian_interaction(P.space, seed0 + i) for i in range(nperturb)]
        self.op0 = op_values(P.vlam, self.order)
        self.a0 = segment_arrays(P.A, P.segA)["vals"]
        self.b0 = segment_arrays(P.B, P.segB)["vals"]
        same = P.segB is P.segA
        self.dop, self.da, self.db = [], [], []
        for Pi in self.perturb:
            full = P.inter.plus(Pi)
            self.dop.append(op_values(multipole_pn(Pi), self.order))
            sa = segment_arrays(P.A, P.A.hamiltonian_segments(full, P.renorm))["vals"]
            self.da.append(sa - self.a0)
            if same:
                self.db.append(self.da[-1])
            else:
                sb = segment_arrays(P.B, P.B.hamiltonian_segments(full, P.renorm))["vals"]
                self.db.append(sb - self.b0)

    @property
    def nperturb(self):
        return len(self.perturb)

    def arrays(self, lam):
        """(op_vals, a_seg_vals, b_seg_vals) of the variant base + sum_i lam_i P_i."""
        lam = np.asarray(lam, dtype=np.float64)
        assert lam.shape == (self.nperturb,)
        op = self.op0 + sum(l * d for l, d in zip(lam, self.dop))
        a = self.a0 + sum(l * d for l, d in zip(lam, self.da))
        b = self.b0 + sum(l * d for l, d in zip(lam, self.db))
        return op, a, b

    def interaction(self, lam):
        """The variant's interaction itself (for the oracle and for direct checks)."""
        inter = self.P.inter
        for l, Pi in zip(lam, self.perturb):
            inter = inter.plus(Pi, float(l))
        return inter


def sample_lambdas(n, nperturb=8, seed=7, scale=0.3):
    """n variants, each lam ~ U[-scale, scale]^nperturb, seeded."""
    return np.random.default_rng(seed).uniform(-scale, scale, size=(n, nperturb))
