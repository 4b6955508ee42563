"""<psi_i|H|psi_j> between eigenvectors: NuXpct's matrix (src/NuXpct/NuCoreXE.f90:1417-1471),
the reference's own check of a solve -- diagonal, with the eigenvalues on the diagonal -- from
host vectors and through its files (.xvc in, .ovl / .ovx out)."""
import os
import struct
import numpy as np
import pytest

from conftest import make_problem

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _lib():
    from nushellx_b200.build import build
    build()


def _records(path):
    data, p, out = open(path, "rb").read(), 0, []
    while p < len(data):
        (n,) = struct.unpack_from("<i", data, p)
        out.append(data[p + 4:p + 4 + n])
        p += 8 + n
    return out


def test_expectation_matrix_of_eigenvectors_is_diagonal(tmp_path):
    from nushellx_b200.nsx import Solver, NSX_FP64, NSX_FP32
    from test_generator import dense_jscheme
    P = make_problem("sd_2p2n_2")
    H = dense_jscheme(P)
    S = Solver.from_problem(P)
    ev, vecs, _ = S.solve(nev=6, tol=1e-9, precision=NSX_FP64, want_vectors=True)
    M = S.expectation_matrix(vecs)
    assert np.allclose(M, vecs @ H @ vecs.T, atol=1e-10)
    assert np.abs(np.diag(M) - ev).max() < 1e-8
    assert np.abs(M - np.diag(np.diag(M))).max() < 1e-8
    M32 = S.expectation_matrix(vecs, NSX_FP32)
    assert np.abs(M32 - M).max() < 1e-4
    # the file form: NuVec's .xvc in, .ovl / .ovx out
    prefix = str(tmp_path / "sd")
    S.write_results(prefix, ev, vecs)
    S.xpct_files(prefix + ".xvc", prefix + "H")
    recs = _records(prefix + "H.ovx")
    nlev = struct.unpack("<i", recs[0])[0]
    assert nlev == 6
    Mf = np.array([np.frombuffer(r, dtype="<f4") for r in recs[1:]]).T   # matrixc(i, j), column j per record
    assert np.abs(np.diag(Mf) - ev).max() < 1e-4
    assert np.abs(Mf - np.diag(np.diag(Mf))).max() < 1e-4
    assert os.path.getsize(prefix + "H.ovl") > 0
    S.close()
