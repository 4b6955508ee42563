"""Output-block sharding of H.v on the CPU (no GPU): the split of the blocks into ranks' row
ranges (plan-only shard handles), and the row exchange over torch.distributed with gloo ranks
(world sizes 2 and 3).  Each rank forms the FP64 oracle's product for the blocks it owns only
(the reference's per-block work split, src/NuLnz/NuCoreX.f90:142-220); after the exchange every
rank holds the whole product, bit for bit."""
import itertools
import os
import socket
import sys

import numpy as np
import pytest

from conftest import ROOT, make_problem


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("name,world", [("sd_2p2n_2", 2), ("fp_4p4n_0", 2), ("fp_4p4n_0", 3), ("fp_4p4n_0", 4)])
def test_split_covers_the_rows_once_at_block_boundaries(name, world):
    from nushellx_b200.nsx import Solver, NSX_FP64
    P = make_problem(name)
    full = Solver.from_problem(P, device=-1)
    shards = [Solver.from_problem(P, device=-1, shard=(r, world)) for r in range(world)]
    infos = [S.shard_info() for S in shards]
    rows = infos[0]["rows"]
    for r, inf in enumerate(infos):
        assert inf["rank"] == r and inf["world"] == world
        assert np.array_equal(inf["rows"], rows) and np.array_equal(inf["est_flops"], infos[0]["est_flops"])
    assert rows[0] == 0 and rows[-1] == full.dim and np.all(np.diff(rows) >= 0)
    assert set(rows.tolist()) <= set(full.offsets.tolist())   # cuts fall on block boundaries
    # every pn and like-particle flop of the whole product belongs to exactly one rank; a rank's
    # Y work may repeat another's (both read the same Y matrix)
    f = [S.flops for S in shards]
    assert sum(f) >= full.flops * (1 - 1e-12)
    for S in shards:
        S.stats_reset()
    def fl(S):
        st = S.stats()["stages"]
        return np.array([st[k]["flops"] for k in ("k_like", "k_z", "k_a", "k_y")])
    tot = sum(fl(S) for S in shards)
    fs = fl(full)
    assert np.allclose(tot[:3], fs[:3], rtol=1e-12)
    assert tot[3] >= fs[3] * (1 - 1e-12)
    # the cut minimises the largest range's flops (all contiguous cuts tried)
    bf = full.block_flops()
    assert bf.sum() >= full.flops * (1 - 1e-12)
    est = infos[0]["est_flops"]
    for r in range(world):
        assert est[r] == pytest.approx(bf[np.searchsorted(full.offsets, rows[r]):
                                          np.searchsorted(full.offsets, rows[r + 1])].sum(), rel=1e-12)
    nb = len(bf)
    best = min(max(bf[a:b].sum() for a, b in zip((0,) + c, c + (nb,)))
               for c in itertools.combinations_with_replacement(range(nb + 1), world - 1))
    assert est.max() == pytest.approx(best, rel=1e-12)
    for S in shards + [full]:
        S.close()


def _worker(rank, world, port, name, outdir, q):
    try:
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        sys.path.insert(0, ROOT)
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from datetime import timedelta
        import torch
        import torch.distributed as dist
        from conftest import make_problem, write_files
        from nushellx_b200.nsx import Solver
        from nushellx_b200.sharded import gather_rows
        from oracle.jscheme import Oracle
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
        P = make_problem(name)
        man = write_files(P, os.path.join(outdir, f"r{rank}"), "sh")
        S = Solver.from_problem(P, device=-1, shard=(rank, world))
        info = S.shard_info()
        rows = info["rows"]
        O = Oracle(man)
        assert O.dim == S.dim and np.array_equal(O.off, S.offsets)
        own = [k for k in range(len(O.blocks)) if rows[rank] <= O.off[k] < rows[rank + 1]]
        x = np.random.default_rng(11).standard_normal(O.dim) * O.lcoef
        part = O.matvec(x, out_blocks=own)
        y = torch.full((O.dim,), float("nan"), dtype=torch.float64)
        y[rows[rank]:rows[rank + 1]] = torch.from_numpy(part[rows[rank]:rows[rank + 1]])
        assert np.all(part[:rows[rank]] == 0) and np.all(part[rows[rank + 1]:] == 0)
        gather_rows(y, rows, rank)
        ref = O.matvec(x)
        q.put((rank, bool(torch.equal(y, torch.from_numpy(ref))), float(np.abs(ref).max())))
        S.close()
        dist.destroy_process_group()
    except BaseException as e:
        q.put((rank, repr(e), 0.0))
        raise


@pytest.mark.parametrize("world", [2, 3])
def test_ranks_products_gathered_with_gloo_equal_the_whole_product(world, tmp_path):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, "fp_4p4n_0", str(tmp_path), q)) for r in range(world)]
    for p in ps:
        p.start()
    got = dict((r, (ok, m)) for r, ok, m in (q.get(timeout=600) for _ in ps))
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert all(ok is True for ok, _ in got.values()), got
    assert all(m > 0 for _, m in got.values())


def test_shard_handles_check_their_arguments():
    from nushellx_b200.nsx import Solver, NsxError
    P = make_problem("sd_2p2n_0")
    for bad in [(0, 0), (2, 2), (-1, 2), (0, 2000)]:
        with pytest.raises(NsxError):
            Solver.from_problem(P, device=-1, shard=bad)
    # more ranks than blocks: some ranks own no rows and plan no work
    S = Solver.from_problem(P, device=-1)
    nb, world = len(S.blocks), len(S.blocks) + 2
    empty = 0
    for r in range(world):
        T = Solver.from_problem(P, device=-1, shard=(r, world))
        rows = T.shard_info()["rows"]
        assert rows[0] == 0 and rows[-1] == S.dim
        if rows[r + 1] == rows[r]:
            empty += 1
            assert T.flops == 0.0
        else:
            assert T.flops > 0.0
        T.close()
    assert empty >= 2
    S.close()
