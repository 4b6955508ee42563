"""H.v on the GPU through the C ABI against the FP64 oracle (parity tests proper).

Tolerances: the FP64 form must agree with the oracle to 1e-12 relative (max
norm, relative to max|y|); the FP32 form to 2e-5 relative (single-precision
accumulation over at most a few thousand terms per output element).
"""
import os
import numpy as np
import pytest

from conftest import make_problem, custom_problem, write_files

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FP32_TOL = 2e-5


@pytest.fixture(scope="module", autouse=True)
def _lib():
    from nushellx_b200.build import build
    build()


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _fp32_variants(S):
    """The FP32 variants the handle can take (the fused one only with groups of <= 16 sources)."""
    from nushellx_b200.nsx import NSX_FP32_FUSED, NSX_FP32_TC, NSX_FP32_SIMT
    return ([NSX_FP32_FUSED] if S.plan_info()["fused_fp32"] else []) + [NSX_FP32_TC, NSX_FP32_SIMT]


def check_fp32_variants(S, x, y_ref):
    """Every FP32 variant against the oracle, then the automatic choice (one of them)."""
    from nushellx_b200.nsx import NSX_FP32, NSX_FP32_AUTO
    for p in _fp32_variants(S):
        S.set_fp32_path(p)
        y32 = S.matvec_host(x, NSX_FP32)
        assert S.plan_info()["fp32_path"] == p
        assert _rel(y32, y_ref) < FP32_TOL, (p, _rel(y32, y_ref))
    S.set_fp32_path(NSX_FP32_AUTO)
    y32 = S.matvec_host(x, NSX_FP32)
    assert S.plan_info()["fp32_path"] in _fp32_variants(S)
    assert _rel(y32, y_ref) < FP32_TOL, _rel(y32, y_ref)


@pytest.mark.parametrize("name", ["sd_2p2n_0", "sd_2p2n_2", "fp_4p4n_0"])
def test_matvec_from_files_matches_oracle(name, files_dir):
    from oracle.jscheme import Oracle
    from nushellx_b200.nsx import Solver, NSX_FP64, NSX_FP32
    P = make_problem(name)
    man = write_files(P, os.path.join(files_dir, name), name)
    O = Oracle(man)
    S = Solver.from_files(man)
    assert S.dim == O.dim
    assert np.array_equal(S.lcoef, O.lcoef)
    rng = np.random.default_rng(7)
    for trial in range(2):
        x = rng.standard_normal(S.dim)
        y_ref = O.matvec(x)
        y64 = S.matvec_host(x, NSX_FP64)
        assert _rel(y64, y_ref) < FP64_TOL, _rel(y64, y_ref)
        check_fp32_variants(S, x, y_ref)
    S.close()


def test_matvec_in_memory_problem_matches_dense_h():
    """nsx_create path (FP64 operator data, no file rounding) against the dense J-scheme H."""
    from nushellx_b200.nsx import Solver, NSX_FP64
    from test_generator import dense_jscheme
    P = make_problem("sd_2p2n_2")
    H = dense_jscheme(P)
    S = Solver.from_problem(P)
    X = np.random.default_rng(3).standard_normal((3, S.dim))
    for x in X:
        assert _rel(S.matvec_host(x, NSX_FP64), H @ x) < FP64_TOL


def test_matvec_mixed_parity_odd_nucleons():
    from nushellx_b200.nsx import Solver, NSX_FP64, NSX_FP32
    from test_generator import dense_jscheme
    P = custom_problem("F5PG9", 2, 1, 3, -1, 9)
    H = dense_jscheme(P)
    S = Solver.from_problem(P)
    x = np.random.default_rng(5).standard_normal(S.dim)
    assert _rel(S.matvec_host(x, NSX_FP64), H @ x) < FP64_TOL
    assert _rel(S.matvec_host(x, NSX_FP32), H @ x) < FP32_TOL


def test_matvec_unit_vectors_and_linearity():
    """Edge inputs: zero vector, unit vectors (the reference's dense-H hook, NuCoreX.f90:1370-1401), linearity."""
    from nushellx_b200.nsx import Solver, NSX_FP64
    from test_generator import dense_jscheme
    P = make_problem("sd_2p2n_0")
    H = dense_jscheme(P)
    S = Solver.from_problem(P)
    assert np.all(S.matvec_host(np.zeros(S.dim), NSX_FP64) == 0.0)
    Hg = np.array([S.matvec_host(e, NSX_FP64) for e in np.eye(S.dim)]).T
    assert np.abs(Hg - H).max() < 1e-12 * np.abs(H).max()
    assert np.abs(Hg - Hg.T).max() < 1e-12 * np.abs(H).max()
    rng = np.random.default_rng(1)
    x, y = rng.standard_normal((2, S.dim))
    lhs = S.matvec_host(2.0 * x - 3.0 * y, NSX_FP64)
    rhs = 2.0 * S.matvec_host(x, NSX_FP64) - 3.0 * S.matvec_host(y, NSX_FP64)
    assert _rel(lhs, rhs) < 1e-12


def test_matvec_device_pointers_and_bad_arguments():
    import torch
    from nushellx_b200.nsx import Solver, NSX_FP64, NsxError
    P = make_problem("sd_2p2n_0")
    S = Solver.from_problem(P)
    x = torch.randn(S.dim, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    S.matvec(x.data_ptr(), y.data_ptr(), NSX_FP64, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert _rel(y.cpu().numpy(), S.matvec_host(x.cpu().numpy(), NSX_FP64)) < 1e-14
    with pytest.raises(NsxError):
        S.matvec(x.data_ptr(), x.data_ptr(), NSX_FP64)      # aliasing
    with pytest.raises(NsxError):
        S.matvec(x.data_ptr(), y.data_ptr(), 7)             # unknown precision


def test_matvec_benchmark_workload_matches_oracle(files_dir):
    """The benchmarked workload itself (fp 6p+6n, J=0+, dimension 1,777,116): H.v from the
    reference-format files against the FP64 oracle on two random vectors.  It reaches the
    paths the small cases do not: Y tiles of more than one row tile, proton slabs whose stacked
    operand is longer than one pipeline pass, and mixing groups with more than 8 sources."""
    from oracle.jscheme import Oracle
    from nushellx_b200.nsx import Solver, NSX_FP64, NSX_FP32
    name = "fp_6p6n_0"
    P = make_problem(name)
    man = write_files(P, os.path.join(files_dir, name), name)
    O = Oracle(man)
    S = Solver.from_files(man)
    assert S.dim == O.dim == 1777116
    assert np.array_equal(S.lcoef, O.lcoef)
    rng = np.random.default_rng(2024)
    for trial in range(2):
        x = rng.standard_normal(S.dim)
        y_ref = O.matvec(x)
        y64 = S.matvec_host(x, NSX_FP64)
        assert _rel(y64, y_ref) < FP64_TOL, _rel(y64, y_ref)
        if trial == 0:
            check_fp32_variants(S, x, y_ref)
        else:
            y32 = S.matvec_host(x, NSX_FP32)
            assert _rel(y32, y_ref) < FP32_TOL, _rel(y32, y_ref)
    S.close()


# Mid-size cases chosen for the kernel paths they reach (asserted from the plan):
#  fp 6p+2n J=0+: proton blocks of 3 Y row tiles, FP64 slabs split in up to 17 K pieces,
#                 proton partitions of up to 49 states (all four tensor-core N classes), the
#                 fused FP32 neutron/mixing stage, k_a_tc slabs cut into K pieces (atomic sums);
#  fp 5p+3n J=1+: mixing groups of 32 sources (FP32 takes k_y + k_z, FP64 the 32-source k_z),
#                 N classes 16 and 32.
PATH_CASES = {"fp_6p2n_0": ("FP", 6, 2, 0, 1, 5), "fp_5p3n_2": ("FP", 5, 3, 2, 1, 5)}


def check_paths(name, info):
    if name == "fp_6p2n_0":
        assert info["y_row_tiles_max"] >= 2 and info["slab_splits_max"] >= 2, info
        assert info["fused_fp32"] == 1 and all(n > 0 for n in info["tc_tiles"]), info
        assert info["tc_chunks_max"] > 8 and info["slab_nl_max"] > 48 and info["tc_pieces"] > 0, info
    else:
        assert info["group_sources_max"] > 16 and info["fused_fp32"] == 0, info
        assert info["tc_tiles"][1] > 0 and info["y_row_tiles_max"] >= 2, info


@pytest.mark.parametrize("name", sorted(PATH_CASES))
def test_matvec_kernel_paths_match_oracle(name, files_dir):
    from oracle.jscheme import Oracle
    from nushellx_b200.nsx import Solver, NSX_FP64, NSX_FP32
    P = custom_problem(*PATH_CASES[name])
    man = write_files(P, os.path.join(files_dir, name), name)
    O = Oracle(man)
    S = Solver.from_files(man)
    check_paths(name, S.plan_info())
    rng = np.random.default_rng(17)
    for trial in range(2):
        x = rng.standard_normal(S.dim)
        y_ref = O.matvec(x)
        y64 = S.matvec_host(x, NSX_FP64)
        assert _rel(y64, y_ref) < FP64_TOL, _rel(y64, y_ref)
        check_fp32_variants(S, x, y_ref)
    S.close()
