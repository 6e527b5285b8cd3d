"""One all-pairs job spread over the ranks of a process group, one device per
rank (the multi-device form of pairwise::run; the reference splits pairs over
MPI ranks, src/pairwise/needleman/needleman.cpp:31-52).

Every rank computes the same split (msa_nw_part_of_pairs: runs of the
kernels' task list with about equal DP cells), scores its own part into a
zero-filled int32 triangle on its device (msa_nw_all_pairs_part), and one sum
reduce assembles the whole matrix on the root rank, the device that runs
neighbor-joining (a serial chain that runs on one GPU). The sum is exact:
parts are disjoint and every other entry is 0.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import MSA_NW_PERSISTENT, check, lib


def exchange(tri, group=None, root: int = 0):
    """Sums the ranks' partial triangles into `tri` on rank `root` (torch
    tensor, int32); other ranks' tensors are left as the reduction leaves
    them. One rank: nothing to do."""
    import torch.distributed as dist
    if dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.reduce(tri, dst=root, op=dist.ReduceOp.SUM, group=group)
    return tri


def score_part(ctx, seqs: int, table, part: int, nparts: int, out_ptr: int, mode: int = MSA_NW_PERSISTENT,
               on_device: bool = True) -> None:
    """This rank's pairs into the triangle at `out_ptr` (other entries kept)."""
    check(lib().msa_nw_all_pairs_part(ctx.handle, seqs, ctypes.byref(table._t), mode, part, nparts,
                                      ctypes.c_void_p(out_ptr), 1 if on_device else 0), ctx.handle)


def all_pairs(flat: np.ndarray, offs: np.ndarray, lens: np.ndarray, table, mode: int = MSA_NW_PERSISTENT,
              group=None, device: int | None = None):
    """The whole int32 triangle on rank 0's device, scored by all ranks (on
    the other ranks the returned tensor holds no whole matrix)."""
    import torch
    import torch.distributed as dist

    from . import runtime
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    ctx = runtime.context(device)
    n = len(lens)
    flat = np.ascontiguousarray(flat, np.uint8)
    offs = np.ascontiguousarray(offs, np.uint64)
    lens = np.ascontiguousarray(lens, np.uint64)
    u8, u64 = ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_uint64)
    h = ctypes.c_uint64()
    check(lib().msa_seqs_upload(ctx.handle, flat.ctypes.data_as(u8), offs.ctypes.data_as(u64),
                                lens.ctypes.data_as(u64), n, ctypes.byref(h)), ctx.handle)
    try:
        tri = torch.zeros(n * (n - 1) // 2, dtype=torch.int32, device=torch.device("cuda", ctx.device))
        torch.cuda.synchronize(ctx.device)   # the library scores on its own stream
        score_part(ctx, h.value, table, rank, world, tri.data_ptr(), mode)
        torch.cuda.synchronize(ctx.device)
    finally:
        lib().msa_seqs_release(ctx.handle, h.value)
    return exchange(tri, group)
