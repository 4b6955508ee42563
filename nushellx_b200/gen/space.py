"""Model spaces, seeded synthetic interactions and the five benchmark workloads.

A model space is a list of orbits (2j, parity) shared by protons and neutrons
(the pn formalism of NuShellX: proton shells are numbered 1..norb and neutron
shells norb+1..2norb, as in src/NuOp/NuOp.f90:236-262 and the TrdChar shell
helpers of src/NuCommonX/NuCommonX.f90:70-140).

The interaction is a set of isospin-formalism two-body matrix elements
V_JT(ab;cd) between normalised antisymmetric two-particle states, drawn from a
seeded N(0,1) distribution scaled by 1/sqrt(N_TBME) and symmetrised, plus
single-particle energies.  Matrix elements with a > b (or c > d) follow from
the exchange phase |ba;JT> = (-1)^(ja+jb-J-T) |ab;JT>.
"""
from dataclasses import dataclass, field
from itertools import combinations_with_replacement
import numpy as np

from .angmom import triangle


@dataclass
class ModelSpace:
    j2: list            # 2j per orbit
    parity: list        # +1 / -1 per orbit
    spe: list           # single-particle energies (MeV), same for p and n

    @property
    def norb(self):
        return len(self.j2)


@dataclass
class Interaction:
    space: ModelSpace
    tbme: dict = field(default_factory=dict)   # canonical (a,b,c,d,J2,T) -> V, a<=b, c<=d, (a,b)<=(c,d)

    def V(self, a, b, c, d, J2, T):
        """V_JT(ab;cd) for any orbit order (exchange phases applied)."""
        ph = 1.0
        j2 = self.space.j2
        if a > b:
            a, b = b, a
            ph *= (-1) ** (((j2[a] + j2[b]) // 2 - J2 // 2 - T) % 2)
        if c > d:
            c, d = d, c
            ph *= (-1) ** (((j2[c] + j2[d]) // 2 - J2 // 2 - T) % 2)
        if (a, b) > (c, d):
            a, b, c, d = c, d, a, b
        return ph * self.tbme.get((a, b, c, d, J2, T), 0.0)

    def scaled(self, s):
        return Interaction(self.space, {k: s * v for k, v in self.tbme.items()})

    def plus(self, other, s=1.0):
        keys = set(self.tbme) | set(other.tbme)
        return Interaction(self.space, {k: self.tbme.get(k, 0.0) + s * other.tbme.get(k, 0.0) for k in sorted(keys)})


def tbme_keys(space):
    """All isospin-formalism TBME labels (a<=b, c<=d, (a,b)<=(c,d), J, T) allowed by
    the Pauli principle (J+T odd for a==b of half-integer j), angular momentum and parity."""
    j2, par = space.j2, space.parity
    pairs = list(combinations_with_replacement(range(space.norb), 2))
    keys = []
    for i, (a, b) in enumerate(pairs):
        for (c, d) in pairs[i:]:
            if par[a] * par[b] != par[c] * par[d]:
                continue
            for J2 in range(0, 2 * max(j2) + 1, 2):
                if not (triangle(j2[a], j2[b], J2) and triangle(j2[c], j2[d], J2)):
                    continue
                for T in (0, 1):
                    if (a == b or c == d) and (J2 // 2 + T) % 2 == 0:
                        continue
                    keys.append((a, b, c, d, J2, T))
    return keys


def gaussian_interaction(space, seed):
    """Seeded isospin-conserving Gaussian TBMEs, N(0,1)/sqrt(N_TBME) MeV, symmetric."""
    keys = tbme_keys(space)
    rng = np.random.default_rng(seed)
    vals = rng.standard_normal(len(keys)) / np.sqrt(len(keys))
    return Interaction(space, dict(zip(keys, vals.tolist())))


# ---------------------------------------------------------------------------
# The five workloads.  Orbit order and SPEs as stated for each configuration.
SD = ModelSpace(j2=[5, 1, 3], parity=[1, 1, 1], spe=[-3.9, -3.2, 1.6])
FP = ModelSpace(j2=[7, 3, 5, 1], parity=[-1, -1, -1, -1], spe=[0.0, 2.0, 6.5, 4.0])
F5PG9 = ModelSpace(j2=[5, 3, 1, 9], parity=[-1, -1, -1, 1], spe=[-9.3, -9.8, -8.7, -6.3])


@dataclass
class Workload:
    name: str
    space: ModelSpace
    nprot: int
    nneut: int
    J2: int
    parity: int
    seed: int = 2024


WORKLOADS = {
    "sd_2p2n_0": Workload("sd_2p2n_0", SD, 2, 2, 0, 1),
    "sd_2p2n_2": Workload("sd_2p2n_2", SD, 2, 2, 4, 1),
    "fp_4p4n_0": Workload("fp_4p4n_0", FP, 4, 4, 0, 1),
    "fp_6p6n_0": Workload("fp_6p6n_0", FP, 6, 6, 0, 1),
    "f5pg9_6p10n_0": Workload("f5pg9_6p10n_0", F5PG9, 6, 10, 0, 1),
    "f5pg9_6p10n_2": Workload("f5pg9_6p10n_2", F5PG9, 6, 10, 4, 1),
}
