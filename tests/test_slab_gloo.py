"""Bookkeeping of the slab decomposition on CPU: the block split, the exchange counts
of libspns (spns_slab_block, spns_slab_counts) and the staging layout of its pack
kernels, moved between ranks by real torch.distributed all-to-alls (gloo, world
sizes 2 and 3) -- the reference's FFTW-MPI transposes (src/FFTW_package.cpp:47-56,
src/FFTW_package.h:60-64) on CPU ranks.

The pack layout restated here is the one k_slab_pack (solver_kernels.cuh) writes:
rank block s = [f][n1_s][n2_s][Kz] contiguous, blocks in rank order, split along
axis 1 (ky rows) or 2 (x planes).  The GPU side of the same exchange is checked
against the one-GPU step in tests/test_gpu_slab.py.
"""
import ctypes as C
import os
import socket

import numpy as np
import pytest


def _ranges(n, P):
    from spns_b200.slab import block
    return [block(n, P, r) for r in range(P)]


def pack(full, ranges, axis):
    blocks = []
    for st, cnt in ranges:
        blk = full[:, st:st + cnt] if axis == 1 else full[:, :, st:st + cnt]
        blocks.append(np.ascontiguousarray(blk).ravel())
    return np.concatenate(blocks)


def unpack(stage, shape, ranges, axis):
    out = np.empty(shape, dtype=stage.dtype)
    o = 0
    for st, cnt in ranges:
        bshape = list(shape)
        bshape[axis] = cnt
        n = int(np.prod(bshape))
        blk = stage[o:o + n].reshape(bshape)
        if axis == 1:
            out[:, st:st + cnt] = blk
        else:
            out[:, :, st:st + cnt] = blk
        o += n
    return out


def test_block_split_matches_the_library():
    from spns_b200.hit import lib
    from spns_b200.slab import block
    L = lib()
    for n in (17, 33, 48, 49, 257, 513, 768, 1025, 1536):
        for P in (1, 2, 3, 4, 5, 7, 8):
            tot = 0
            for r in range(P):
                s, c = C.c_int(), C.c_int()
                assert L.spns_slab_block(n, P, r, C.byref(s), C.byref(c)) == 0
                assert (s.value, c.value) == block(n, P, r)
                tot += c.value
            assert tot == n


@pytest.mark.parametrize("P", [2, 3, 4, 8])
def test_exchange_counts_pair_up(P):
    """What rank r sends to s is what s expects from r, in both directions, and the
    totals are the rank's rows (or planes) of every field."""
    from spns_b200.slab import block, exchange_counts
    Ky, Mx, Kz = 33, 48, 17
    for back in (False, True):
        c = [exchange_counts(Ky, Mx, Kz, P, r, 6, back) for r in range(P)]
        for r in range(P):
            for s in range(P):
                assert c[r][0][s] == c[s][1][r]
            ny, nx = block(Ky, P, r)[1], block(Mx, P, r)[1]
            assert sum(c[r][0 if not back else 1]) == 6 * ny * Mx * Kz
            assert sum(c[r][1 if not back else 0]) == 6 * Ky * nx * Kz


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, shape, q):
    import torch
    import torch.distributed as dist
    from spns_b200.slab import exchange_counts
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        Ky, Mx, Kz = shape
        rng = np.random.default_rng(5)
        A = rng.standard_normal((6, Ky, Mx, Kz)) + 1j * rng.standard_normal((6, Ky, Mx, Kz))
        B = rng.standard_normal((3, Ky, Mx, Kz)) + 1j * rng.standard_normal((3, Ky, Mx, Kz))
        yr, xr = _ranges(Ky, world), _ranges(Mx, world)
        (y0, ny), (x0, nx) = yr[rank], xr[rank]
        # ky rows -> x planes (after the inverse x pass: 6 fields)
        send = pack(A[:, y0:y0 + ny], xr, 2)
        sc, rc = exchange_counts(Ky, Mx, Kz, world, rank, 6, False)
        assert sum(sc) == send.size
        recv = torch.empty(2 * sum(rc), dtype=torch.float64)
        dist.all_to_all_single(recv, torch.from_numpy(send.view(np.float64).copy()), [2 * c for c in rc], [2 * c for c in sc])
        got = unpack(recv.numpy().view(np.complex128), (6, Ky, nx, Kz), yr, 1)
        ok1 = bool(np.array_equal(got, A[:, :, x0:x0 + nx]))
        # x planes -> ky rows (after the forward y pass: 3 fields)
        send = pack(B[:, :, x0:x0 + nx], yr, 1)
        sc, rc = exchange_counts(Ky, Mx, Kz, world, rank, 3, True)
        recv = torch.empty(2 * sum(rc), dtype=torch.float64)
        dist.all_to_all_single(recv, torch.from_numpy(send.view(np.float64).copy()), [2 * c for c in rc], [2 * c for c in sc])
        got = unpack(recv.numpy().view(np.complex128), (3, ny, Mx, Kz), xr, 2)
        ok2 = bool(np.array_equal(got, B[:, y0:y0 + ny]))
        # CFL maxima as integer maxima of the bit patterns of non-negative doubles
        mine = np.array([0.5 + rank, 3.0 - rank, 1e-3 * rank, 7.25], dtype=np.float64)
        t = torch.from_numpy(mine.view(np.int64).copy())
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        allv = np.array([[0.5 + r, 3.0 - r, 1e-3 * r, 7.25] for r in range(world)])
        ok3 = bool(np.array_equal(t.numpy().view(np.float64), allv.max(axis=0)))
        q.put((rank, ok1, ok2, ok3))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_transposes_over_gloo(world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, (33, 48, 17), q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ok1, ok2, ok3 in res:
        assert ok1, f"rank {rank}: ky-rows -> x-planes transpose"
        assert ok2, f"rank {rank}: x-planes -> ky-rows transpose"
        assert ok3, f"rank {rank}: CFL maximum"
