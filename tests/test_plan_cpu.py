"""Plan-only handles (nsx_create / nsx_load_files with device < 0): the host logic of the
library without a GPU -- block list, offsets and parity mask against the generator (in memory
and through the C++ file reader), interaction updates, and the reference's output files read
back as NuVec reads them."""
import os
import numpy as np
import pytest

from conftest import make_problem, write_files


@pytest.fixture(scope="module", autouse=True)
def _lib():
    from nushellx_b200.build import build
    build()


@pytest.mark.parametrize("name", ["sd_2p2n_2", "fp_4p4n_0"])
def test_plan_matches_the_generator(name, files_dir):
    from nushellx_b200.nsx import Solver
    P = make_problem(name)
    for S in (Solver.from_problem(P, device=-1),
              Solver.from_files(write_files(P, os.path.join(files_dir, "plan_" + name), name), device=-1)):
        assert S.dim == P.no_state
        assert [tuple(b[:2]) for b in S.blocks] == [tuple(b) for b in P.blocks]
        assert [tuple(b[2:]) for b in S.blocks] == [tuple(d) for d in P.dims]
        assert np.array_equal(S.offsets, P.offsets)
        assert np.array_equal(S.lcoef, P.lcoef)
        assert S.flops > 0
        S.close()


def test_plan_only_handle_refuses_device_work():
    from nushellx_b200.nsx import Solver, NsxError, NSX_FP64
    S = Solver.from_problem(make_problem("sd_2p2n_0"), device=-1)
    with pytest.raises(NsxError, match="plan only"):
        S.matvec_host(np.ones(S.dim), NSX_FP64)
    with pytest.raises(NsxError, match="plan only"):
        S.solve(nev=2)
    with pytest.raises(NsxError, match="plan only"):
        Solver.batch_solve([S], nev=2)
    S.stats_reset()
    assert S.stats()["launches"] == 0
    S.close()


def test_interaction_update_on_a_plan_only_handle():
    from nushellx_b200.nsx import Solver, NsxError
    from nushellx_b200.gen.variants import InteractionFamily
    P = make_problem("sd_2p2n_2")
    fam = InteractionFamily(P)
    S = Solver.from_problem(P, device=-1)
    S.set_interaction(*fam.arrays(np.full(8, 0.1)))
    op, a, b = fam.arrays(np.zeros(8))
    with pytest.raises(NsxError, match="op_vals holds"):
        S.set_interaction(op[:-1], a, b)
    with pytest.raises(NsxError, match="segment value counts"):
        S.set_interaction(op, a[:-1], b)
    bad = op.copy()
    bad[0] = np.nan
    with pytest.raises(NsxError, match="not finite"):
        S.set_interaction(bad, a, b)
    S.close()


@pytest.mark.parametrize("name", ["sd_2p2n_0", "fp_4p4n_0"])
def test_output_files_round_trip_without_a_gpu(name, tmp_path):
    from nushellx_b200.nsx import Solver
    from test_outputs import read_outputs, read_records
    import struct
    P = make_problem(name)
    S = Solver.from_problem(P, device=-1)
    nev = 5
    rng = np.random.default_rng(3)
    Q, _ = np.linalg.qr(rng.standard_normal((S.dim, nev)) * S.lcoef[:, None])
    vecs = Q.T.copy()
    ev = np.sort(rng.uniform(-5, 5, nev))
    prefix = str(tmp_path / "out")
    S.write_results(prefix, ev, vecs, 123, "synthetic", 0)
    w, psi, lv, par = read_outputs(prefix, S, nev)
    assert np.allclose(w, ev, rtol=1e-6, atol=1e-6)
    for i in range(nev):
        s = np.sign(psi[i] @ vecs[i])
        assert np.abs(s * psi[i] - vecs[i]).max() <= 1e-6 * np.abs(vecs[i]).max()
    assert np.allclose(lv, ev, atol=6e-4) and set(par) == {"+"}
    recs = read_records(prefix + ".xvc")
    assert struct.unpack("<ii", recs[0]) == (S.dim, nev) and len(recs) == nev + 1
    r2 = struct.unpack("<iifiiiiiiii", read_records(prefix + ".abz")[1])
    assert r2[0] == 123
    S.close()


def test_plan_reaches_the_kernel_paths_the_gpu_tests_rely_on():
    """The plan statistics behind the GPU path tests (no GPU needed: plan-only handles)."""
    from conftest import custom_problem
    from nushellx_b200.nsx import Solver
    from test_matvec_gpu import PATH_CASES, check_paths
    for name, case in PATH_CASES.items():
        S = Solver.from_problem(custom_problem(*case), device=-1)
        check_paths(name, S.plan_info())
        S.close()
    info = Solver.from_problem(make_problem("fp_4p4n_0"), device=-1).plan_info()
    assert info["fused_fp32"] == 1 and info["slab_splits_max"] > 1


def test_fp32_variant_requests_are_checked():
    """nsx_set_fp32_path on plan-only handles: unknown variants and the fused variant on a plan
    with a mixing group of more than 16 sources are refused; nothing is chosen before a product."""
    from conftest import custom_problem
    from nushellx_b200.nsx import Solver, NsxError, NSX_FP32_AUTO, NSX_FP32_FUSED, NSX_FP32_TC, NSX_FP32_SIMT
    S = Solver.from_problem(make_problem("fp_4p4n_0"), device=-1)
    for p in (NSX_FP32_AUTO, NSX_FP32_FUSED, NSX_FP32_TC, NSX_FP32_SIMT):
        S.set_fp32_path(p)
    for bad in (-1, 4):
        with pytest.raises(NsxError):
            S.set_fp32_path(bad)
    assert S.plan_info()["fp32_path"] == 0
    T = Solver.from_problem(custom_problem("FP", 5, 3, 2, 1, 5), device=-1)
    assert T.plan_info()["fused_fp32"] == 0
    with pytest.raises(NsxError, match="16 sources"):
        T.set_fp32_path(NSX_FP32_FUSED)
    T.set_fp32_path(NSX_FP32_TC)
    S.close()
    T.close()


def _nuvec_averages(P, S, v):
    """NuVec's per-level sums (src/NuVec/NuVec.f90:210-240) restated in numpy: |c|^2 per
    (proton partition, neutron partition, 2J_a, 2J_b), and the shell occupations they weight."""
    A, B = P.A, P.B
    nJa, nJb = (A.maxJ2 - A.minJ2) // 2 + 1, (B.maxJ2 - B.minJ2) // 2 + 1
    cell = np.zeros((nJb, nJa, len(B.parts), len(A.parts)))
    for k, (J2a, J2b, da, db) in enumerate(S.blocks):
        blk = v[S.offsets[k]:S.offsets[k + 1]].reshape(db, da)     # column-major: row = neutron state
        ra = np.repeat(np.arange(len(A.parts)), [A.njt(p, J2a) for p in range(len(A.parts))])
        rb = np.repeat(np.arange(len(B.parts)), [B.njt(p, J2b) for p in range(len(B.parts))])
        w = blk ** 2
        np.add.at(cell[(J2b - B.minJ2) // 2, (J2a - A.minJ2) // 2], (rb[:, None], ra[None, :]), w)
    wa, wb = cell.sum(axis=(0, 1, 2)), cell.sum(axis=(0, 1, 3))
    occa = np.array(A.parts, dtype=float)
    occb = np.array(B.parts, dtype=float)
    norb = P.space.norb
    ava = np.concatenate([wa @ occa, np.zeros(norb)])
    avb = np.concatenate([np.zeros(norb), wb @ occb])
    return ava, avb, cell


@pytest.mark.parametrize("name", ["sd_2p2n_2", "fp_4p4n_0"])
def test_nuvec_averages_xva_and_lp(name, tmp_path):
    """.xva / .lp for given eigenpairs, without a GPU: each record holds the energy, the shell
    occupations weighted by |c|^2 and the partition-pair percentages (NuVec.f90:199-290),
    equal to the numpy restatement; the percentages add up to 100 and the occupations to the
    nucleon numbers."""
    import struct
    from nushellx_b200.nsx import Solver
    from test_outputs import read_records
    P = make_problem(name)
    S = Solver.from_problem(P, device=-1)
    rng = np.random.default_rng(3)
    nev = 3
    vecs = rng.standard_normal((nev, S.dim)) * S.lcoef
    vecs /= np.linalg.norm(vecs, axis=1)[:, None]
    ev = np.array([-3.0, -1.5, 0.25])
    prefix = str(tmp_path / "av")
    S.write_results(prefix, ev, vecs, 10, "synthetic", 0)
    recs = read_records(prefix + ".xva")
    assert len(recs) == nev
    norb = P.space.norb
    for i in range(nev):
        ava, avb, cell = _nuvec_averages(P, S, vecs[i])
        r = np.frombuffer(recs[i], dtype="<f4")
        assert len(r) == 1 + 4 * norb + cell.size
        assert r[0] == np.float32(ev[i])
        assert np.allclose(r[1:1 + 2 * norb], ava, atol=1e-5) and np.allclose(r[1 + 2 * norb:1 + 4 * norb], avb, atol=1e-5)
        sp = r[1 + 4 * norb:].reshape(cell.shape)     # Fortran order (pa fastest, then pb, Ja, Jb)
        assert np.allclose(sp, cell * 100.0, atol=1e-3)
        assert abs(sp.sum() - 100.0) < 1e-2
        assert abs(ava.sum() - P.A.n) < 1e-6 and abs(avb.sum() - P.B.n) < 1e-6
    lp = open(prefix + ".lp").read()
    assert lp.count(" State ") == nev and "A partitions" in lp and "Positive and Negative Parity" in lp
    S.close()
