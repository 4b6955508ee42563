"""NuTRLZ's compressed pn interaction (the .dop file of NuDiop, src/NuDiop/NuDiop.f90; folded
into combined operators as src/NuTRLZ/NuCoreXZ.f90:1613-1887 does).

CPU: the .dop writer/reader round trip, the identity that with no cut the compressed product
is the exact one (oracle against oracle, to the 7 decimals of the text file), the C++
reader's errors and the in-memory entry point.  GPU: H.v of a handle built with the .dop
(nsx_load_files_z) against the compressed-interaction oracle (1e-12 FP64, 2e-5 FP32) with and
without a cut."""
import os
import numpy as np
import pytest

from conftest import make_problem

FP64_TOL, FP32_TOL = 1e-12, 2e-5
CASES = ["sd_2p2n_2", "fp_4p4n_0"]


def _files(name, cut, d):
    from nushellx_b200.gen.writer import write_problem
    tag = f"{name}_{int(cut[0] * 1000)}_{int(cut[1] * 1000)}"
    return write_problem(make_problem(name), os.path.join(d, tag), name, dop_cut=cut)


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_dop_round_trip_and_exact_without_cut(tmp_path):
    from nushellx_b200.gen.dop import diop, write_dop, read_dop
    from oracle.jscheme import Oracle, OracleZ
    P = make_problem("sd_2p2n_2")
    d = diop(P.vlam, P.space)
    write_dop(str(tmp_path / "x.dop"), d)
    r = read_dop(str(tmp_path / "x.dop"))
    assert [(l, p, len(k)) for l, p, k in r] == [(l, p, len(k)) for l, p, k in d]
    for (_, _, k1), (_, _, k2) in zip(d, r):
        for (e1, c1), (e2, c2) in zip(k1, k2):
            assert abs(e1 - e2) < 1e-7 and len(c1) == len(c2)
    man = _files("sd_2p2n_2", (0.0, 0.0), str(tmp_path))
    O, OZ = Oracle(man), OracleZ(man, man["dop"])
    x = np.random.default_rng(3).standard_normal(O.dim)
    assert _rel(OZ.matvec(x), O.matvec(x)) < 1e-7     # the file's 7 decimals
    man2 = _files("sd_2p2n_2", (0.05, 0.01), str(tmp_path))
    assert _rel(OracleZ(man2, man2["dop"]).matvec(x), O.matvec(x)) > 1e-5   # a cut changes H


def test_dop_reader_errors(tmp_path):
    from nushellx_b200.nsx import Solver, NsxError
    man = _files("sd_2p2n_0", (0.0, 0.0), str(tmp_path))
    S = Solver.from_files(man, device=-1, dop=man["dop"])   # plan only: the rewrite and the plan
    assert S.dim == 46 and S.plan_info()["group_sources_max"] > 0
    S.close()
    bad = str(tmp_path / "bad.dop")
    open(bad, "w").write(open(man["dop"]).read()[:40])
    with pytest.raises(NsxError, match="NSX_E_IO"):
        Solver.from_files(man, device=-1, dop=bad)
    with pytest.raises(NsxError, match="NSX_E_IO"):
        Solver.from_files(man, device=-1, dop=str(tmp_path / "missing.dop"))


def test_in_memory_compressed_problem_plans_like_the_files(tmp_path):
    """nsx_create_z (arrays) and nsx_load_files_z (files) give the same plan."""
    from nushellx_b200.gen.dop import diop
    from nushellx_b200.nsx import Solver
    P = make_problem("sd_2p2n_2")
    man = _files("sd_2p2n_2", (0.05, 0.01), str(tmp_path))
    a = Solver.from_files(man, device=-1, dop=man["dop"]).plan_info()
    b = Solver.from_problem_z(P, diop(P.vlam, P.space, 0.05, 0.01), device=-1).plan_info()
    assert a == b


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("cut", [(0.0, 0.0), (0.05, 0.01)])
def test_compressed_matvec_matches_oracle(name, cut, tmp_path):
    from nushellx_b200.build import build
    from nushellx_b200.nsx import Solver, NSX_FP64, NSX_FP32
    from oracle.jscheme import OracleZ
    build()
    man = _files(name, cut, str(tmp_path))
    OZ = OracleZ(man, man["dop"])
    S = Solver.from_files(man, dop=man["dop"])
    x = np.random.default_rng(11).standard_normal(S.dim)
    y = OZ.matvec(x)
    assert _rel(S.matvec_host(x, NSX_FP64), y) < FP64_TOL
    assert _rel(S.matvec_host(x, NSX_FP32), y) < FP32_TOL
    S.close()
