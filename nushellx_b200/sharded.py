"""Output-block sharding of H.v over several GPUs, one process per GPU.

The reference splits one H.v over OpenMP threads by output block and J_ar
(src/NuLnz/NuCoreX.f90:142-220): every thread reads the whole input vector and
writes its own output rows.  Across GPUs the same split holds: nsx_create_shard
gives rank r the output rows of a contiguous range of blocks (cut so that the
ranges' flops are as even as a contiguous cut allows), its product reads the
whole vector and writes its rows, and one all-gather of the ranks' rows per
product gives every rank the whole H.v.  Every rank then runs the same Lanczos
recurrence on the whole vector (the library's solver, unchanged), so the
collective is the only exchange.

This module supplies the all-gather as the handle's exchange (nsx_set_exchange),
over torch.distributed: NCCL for CUDA tensors, gloo for host tensors.  The ranks'
row ranges differ in length; each part is padded to the longest and gathered with
one all_gather.

    S = Solver.from_problem(P, device=local_rank, shard=(rank, world))
    attach_exchange(S)                 # after torch.distributed.init_process_group
    S.solve(nev=10, ...)               # the same eigenpairs on every rank
"""
import torch
import torch.distributed as dist

__all__ = ["gather_rows", "attach_exchange"]


class _DeviceArray:
    """A CUDA array interface over a raw device pointer (no copy)."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def gather_rows(y, rows, rank, group=None, buffers=None):
    """Fills y (a 1-D tensor holding this rank's rows [rows[rank], rows[rank+1]) ) with every
    rank's rows, in place, by one all_gather of parts padded to the longest range.

    rows: first row of every rank (world + 1 entries, the last = len(y)).  buffers: optional
    (send, [recv per rank]) tensors of the padded length, reused between calls."""
    world = len(rows) - 1
    lens = [int(rows[r + 1] - rows[r]) for r in range(world)]
    width = max(max(lens), 1)
    if buffers is None:
        send = torch.zeros(width, dtype=y.dtype, device=y.device)
        recv = [torch.empty(width, dtype=y.dtype, device=y.device) for _ in range(world)]
    else:
        send, recv = buffers
    r0 = int(rows[rank])
    if lens[rank]:
        send[:lens[rank]].copy_(y[r0:r0 + lens[rank]])
    dist.all_gather(recv, send, group=group)
    for r in range(world):
        if r != rank and lens[r]:
            y[int(rows[r]):int(rows[r + 1])].copy_(recv[r][:lens[r]])
    return y


def attach_exchange(S, group=None):
    """Makes every product of the shard handle S whole on every rank: after S's rows are
    computed, gather_rows runs on the product's stream (NCCL over the default process group
    unless `group` is given).  Returns the exchange function (also held by S)."""
    info = S.shard_info()
    rows, rank, world = info["rows"], info["rank"], info["world"]
    if world != (dist.get_world_size(group) if dist.is_initialized() else 1):
        raise ValueError("the handle's shard count differs from the process group's size")
    dev = torch.device("cuda", torch.cuda.current_device())
    width = max(max(int(rows[r + 1] - rows[r]) for r in range(world)), 1)
    bufs = (torch.zeros(width, dtype=torch.float64, device=dev),
            [torch.empty(width, dtype=torch.float64, device=dev) for _ in range(world)])

    def exchange(y_ptr, n, stream_ptr):
        y = torch.as_tensor(_DeviceArray(y_ptr, n), device=dev)
        s = torch.cuda.ExternalStream(stream_ptr, device=dev) if stream_ptr else torch.cuda.default_stream(dev)
        with torch.cuda.stream(s):
            gather_rows(y, rows, rank, group, bufs)

    S.set_exchange(exchange)
    return exchange
