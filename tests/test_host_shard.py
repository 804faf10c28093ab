"""The multi-GPU host logic on CPU: two gloo ranks shard the shots of one
sampling run (each rank's shard computed by the oracle's restatement of the
device's Philox procedure at the rank's shard offset), gather the record
planes and take the maximum time; the gathered record equals one run over all
the shots, bit for bit."""
import os
import socket

import numpy as np
import pytest

import oracle
from qcb200 import circuits, ops as O
from qcb200.shard import SHOT_GROUP, shard_offset


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _pack(meas_bool):
    """Bool frames x nbits -> uint32 planes nbits x ceil(frames/32)."""
    b = np.ascontiguousarray(meas_bool.T.astype(np.uint8))
    words = (b.shape[1] + 31) // 32
    pad = np.zeros((b.shape[0], words * 32), np.uint8)
    pad[:, :b.shape[1]] = b
    return np.packbits(pad, axis=1, bitorder="little").view(np.uint32)


def _rank_main(rank, world, port, shots, seed, outdir):
    import torch.distributed as dist
    from qcb200.shard import gather_record_planes, max_over_ranks

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        arr = O.to_array(circuits.rotated_surface_code_memory(3, 3, 0.01))
        qmax, bmax = O.affected_counts(arr)
        off = shard_offset(rank, shots)
        _, meas = oracle.pftrajectories_philox(arr, shots, qmax, bmax, seed, shot_offset=off)
        whole = gather_record_planes(_pack(meas), shots)
        t = max_over_ranks([1.0 + rank, 5.0 - rank])
        if rank == 0:
            np.save(os.path.join(outdir, "whole.npy"), whole)
            np.save(os.path.join(outdir, "t.npy"), np.array(t))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("shots", [2048, 1500])
def test_two_rank_shards_compose_to_one_run(tmp_path, shots):
    import torch.multiprocessing as mp

    world, seed = 2, 0x5EED
    mp.start_processes(_rank_main, args=(world, _free_port(), shots, seed, str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    whole = np.load(tmp_path / "whole.npy")
    assert list(np.load(tmp_path / "t.npy")) == [2.0, 5.0]  # the maximum over the ranks
    arr = O.to_array(circuits.rotated_surface_code_memory(3, 3, 0.01))
    qmax, bmax = O.affected_counts(arr)
    stride = shard_offset(1, shots)
    total = stride * (world - 1) + shots
    _, meas = oracle.pftrajectories_philox(arr, total, qmax, bmax, seed, shot_offset=0)
    ref = _pack(meas)
    for r in range(world):  # each shard's columns (between shards there may be unused shots)
        w0, nw = r * stride // 32, shots // 32
        assert np.array_equal(whole[:, w0:w0 + nw], ref[:, w0:w0 + nw])
    assert stride % SHOT_GROUP == 0
