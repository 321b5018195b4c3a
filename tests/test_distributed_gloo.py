"""Row-distributed SpMV: the partition by nonzeros, and the exchange (all-gather
of x slices) between world-size-2 gloo ranks on the CPU, with the oracle as
the local product so only the distribution logic is under test.  On a GPU the
same class runs the platform kernel as a one-rank NCCL group."""
import datetime
import os
import socket

import numpy as np
import pytest

from helpers import rand_crs


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_partition_rows_balances_nonzeros():
    from smaxkernels_b200.distributed import partition_rows
    rp, col, val = rand_crs(5000, 30, 1, empty_frac=0.2, long_rows=(4000, 3000))
    for world in (1, 2, 3, 8):
        blocks = partition_rows(rp, world)
        assert blocks[0][0] == 0 and blocks[-1][1] == 5000
        assert all(blocks[i][1] == blocks[i + 1][0] for i in range(world - 1))
        counts = [int(rp[e] - rp[b]) for b, e in blocks]
        assert sum(counts) == len(col)
        # no block exceeds its share by more than the longest row
        assert max(counts) <= len(col) / world + 4000
    # more ranks than rows and an all-empty matrix still give valid blocks
    assert partition_rows(np.array([0, 1, 2]), 4)[-1][1] == 2
    assert partition_rows(np.zeros(7, np.int32), 3)[-1][1] == 6


def _worker(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from oracle.oracle import Oracle
        from smaxkernels_b200.distributed import RowDistributedSpMV, local_block, partition_rows
        rp, col, val = rand_crs(3001, 12, 7, empty_frac=0.1, long_rows=(2500,))
        x = np.random.default_rng(8).uniform(-1, 1, 3001)
        blocks = partition_rows(rp, world)
        lrp, lcol, lval = local_block(rp, col, val, blocks[rank])
        O = Oracle()
        op = RowDistributedSpMV(lrp, lcol, lval, 3001, blocks, rank,
                                local_apply=lambda xf: torch.from_numpy(O.spmv_crs(lrp, lcol, lval, xf.numpy())))
        b, e = blocks[rank]
        for rep in range(2):  # the exchange buffers are reused
            y = op(torch.from_numpy(x[b:e].copy()))
        np.save(os.path.join(out_dir, f"y{rank}.npy"), y.numpy())
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_row_distributed_spmv_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    from oracle.oracle import Oracle
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    y = np.concatenate([np.load(tmp_path / f"y{r}.npy") for r in range(world)])
    rp, col, val = rand_crs(3001, 12, 7, empty_frac=0.1, long_rows=(2500,))
    x = np.random.default_rng(8).uniform(-1, 1, 3001)
    np.testing.assert_array_equal(y, Oracle().spmv_crs(rp, col, val, x))  # same per-row order: exact


def _gpu_worker(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from smaxkernels_b200.distributed import RowDistributedSpMV, local_block, partition_rows
        rp, col, val = rand_crs(20000, 20, 9, long_rows=(9000,))
        x = np.random.default_rng(10).uniform(-1, 1, 20000)
        blocks = partition_rows(rp, world)
        lrp, lcol, lval = local_block(rp, col, val, blocks[rank])
        op = RowDistributedSpMV(lrp, lcol, lval, 20000, blocks, rank, device="cuda")
        b, e = blocks[rank]
        y = op(torch.from_numpy(x[b:e].copy()).cuda())
        torch.cuda.synchronize()
        np.save(os.path.join(out_dir, f"y{rank}.npy"), y.cpu().numpy())
        op.close()
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_row_distributed_spmv_nccl_one_rank(tmp_path):
    import torch.multiprocessing as mp
    from helpers import normwise
    from oracle.oracle import Oracle
    mp.spawn(_gpu_worker, args=(1, _free_port(), str(tmp_path)), nprocs=1, join=True)
    y = np.load(tmp_path / "y0.npy")
    rp, col, val = rand_crs(20000, 20, 9, long_rows=(9000,))
    x = np.random.default_rng(10).uniform(-1, 1, 20000)
    assert normwise(y, Oracle().spmv_crs(rp, col, val, x)) <= 1e-12


def _spmm_spgemm_worker(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from oracle.oracle import Oracle
        from smaxkernels_b200.distributed import (RowDistributedSpGEMM, RowDistributedSpMM, local_block,
                                                  partition_rows)
        O = Oracle()
        rp, col, val = rand_crs(1501, 9, 11, empty_frac=0.1, long_rows=(1200,))
        k = 5
        X = np.random.default_rng(12).uniform(-1, 1, 1501 * k)
        blocks = partition_rows(rp, world)
        lrp, lcol, lval = local_block(rp, col, val, blocks[rank])
        b, e = blocks[rank]
        op = RowDistributedSpMM(lrp, lcol, lval, 1501, k, blocks, rank,
                                local_apply=lambda Xf: torch.from_numpy(O.spmm(lrp, lcol, lval, Xf.numpy(), k)))
        for rep in range(2):
            Y = op(torch.from_numpy(X[b * k:e * k].copy()))
        np.save(os.path.join(out_dir, f"Y{rank}.npy"), Y.numpy())
        # SpGEMM: B = A replicated, no exchange; the parts meet on every rank
        gemm = RowDistributedSpGEMM(lrp, lcol, lval, rp, col, val, 1501,
                                    local_apply=lambda a, c, v: O.spgemm(a, c, v, rp, col, val, 1501))
        parts = [None] * world
        dist.all_gather_object(parts, gemm())
        if rank == 0:
            from smaxkernels_b200.distributed import concat_rows
            crp, ccol, cval = concat_rows(parts)
            np.save(os.path.join(out_dir, "crp.npy"), crp)
            np.save(os.path.join(out_dir, "ccol.npy"), ccol)
            np.save(os.path.join(out_dir, "cval.npy"), cval)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_row_distributed_spmm_and_spgemm_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    from oracle.oracle import Oracle
    world = 2
    mp.spawn(_spmm_spgemm_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    O = Oracle()
    rp, col, val = rand_crs(1501, 9, 11, empty_frac=0.1, long_rows=(1200,))
    k = 5
    X = np.random.default_rng(12).uniform(-1, 1, 1501 * k)
    Y = np.concatenate([np.load(tmp_path / f"Y{r}.npy") for r in range(world)])
    np.testing.assert_array_equal(Y, O.spmm(rp, col, val, X, k))
    crp, ccol, cval = O.spgemm(rp, col, val, rp, col, val, 1501)
    np.testing.assert_array_equal(np.load(tmp_path / "crp.npy"), crp)
    np.testing.assert_array_equal(np.load(tmp_path / "ccol.npy"), ccol)
    np.testing.assert_array_equal(np.load(tmp_path / "cval.npy"), cval)


def _gpu_spmm_spgemm_worker(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from smaxkernels_b200.distributed import (RowDistributedSpGEMM, RowDistributedSpMM, local_block,
                                                  partition_rows)
        rp, col, val = rand_crs(9000, 15, 13, long_rows=(5000,))
        k = 8
        X = np.random.default_rng(14).uniform(-1, 1, 9000 * k)
        blocks = partition_rows(rp, world)
        lrp, lcol, lval = local_block(rp, col, val, blocks[rank])
        b, e = blocks[rank]
        op = RowDistributedSpMM(lrp, lcol, lval, 9000, k, blocks, rank, device="cuda")
        Y = op(torch.from_numpy(X[b * k:e * k].copy()).cuda())
        torch.cuda.synchronize()
        np.save(os.path.join(out_dir, "Y.npy"), Y.cpu().numpy())
        op.close()
        crp, ccol, cval = RowDistributedSpGEMM(lrp, lcol, lval, rp, col, val, 9000)()
        np.save(os.path.join(out_dir, "crp.npy"), crp)
        np.save(os.path.join(out_dir, "ccol.npy"), ccol)
        np.save(os.path.join(out_dir, "cval.npy"), cval)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_row_distributed_spmm_spgemm_nccl_one_rank(tmp_path):
    import torch.multiprocessing as mp
    from helpers import normwise
    from oracle.oracle import Oracle
    mp.spawn(_gpu_spmm_spgemm_worker, args=(1, _free_port(), str(tmp_path)), nprocs=1, join=True)
    O = Oracle()
    rp, col, val = rand_crs(9000, 15, 13, long_rows=(5000,))
    k = 8
    X = np.random.default_rng(14).uniform(-1, 1, 9000 * k)
    assert normwise(np.load(tmp_path / "Y.npy"), O.spmm(rp, col, val, X, k)) <= 1e-12
    crp, ccol, cval = O.spgemm(rp, col, val, rp, col, val, 9000)
    np.testing.assert_array_equal(np.load(tmp_path / "crp.npy"), crp)
    np.testing.assert_array_equal(np.load(tmp_path / "ccol.npy"), ccol)
    assert normwise(np.load(tmp_path / "cval.npy"), cval) <= 1e-12
