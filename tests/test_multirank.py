"""Multi-rank counting (z-slab shards + all-reduce of the counts), run as 2 and 3 gloo ranks on
the CPU: every rank cuts its slab with `slab_planes`, counts it (here with the oracle, the checker,
standing in for the per-GPU kernel), and `sharded_field_bpfd` all-reduces; the result on every
rank must equal the oracle's counts of the whole field, exactly.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from mkf_b200.shard import sharded_field_bpfd, slab_cells, slab_planes

CASES = [  # (Z, Y, X), thresholds, masks
    ((9, 13, 40), [0.0, 0.5, -0.25], [4, 3, 7]),
    ((2, 20, 33), [0.1], [4]),          # one cell plane: the second (and third) rank has none
    ((31, 7, 5), [-0.3, 0.3], [6, 1]),
]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _field(shape, seed):
    rng = np.random.default_rng(seed)
    return (rng.integers(-3, 4, size=shape) * 0.25).astype(np.float64)


def _worker(rank, world, port, results):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from oracle import Oracle

        orc = Oracle()

        def counter(slab, t, m, out):
            s = slab.numpy()
            Z, Y, X = s.shape
            out += torch.from_numpy(orc.bpfd_field(s, (X, Y, Z), t, m).astype(np.int64))

        got = []
        for i, (shape, t, m) in enumerate(CASES):
            f = _field(shape, 100 + i)
            z0, z1 = slab_planes(shape[0], world, rank)
            slab = torch.from_numpy(np.ascontiguousarray(f[z0:z1]))
            got.append(sharded_field_bpfd(slab, t, m, counter=counter).numpy().copy())
        results[rank] = got
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_counts_equal_whole_field(oracle, world):
    mgr = mp.get_context("spawn").Manager()
    results = mgr.dict()
    mp.start_processes(_worker, args=(world, _free_port(), results), nprocs=world, start_method="spawn")
    for i, (shape, t, m) in enumerate(CASES):
        f = _field(shape, 100 + i)
        Z, Y, X = shape
        want = oracle.bpfd_field(f, (X, Y, Z), t, m).astype(np.int64)
        for r in range(world):
            assert (results[r][i] == want).all(), (world, r, shape)


def test_slab_partition_covers_every_cell_plane_once():
    for Z in (1, 2, 3, 10, 1025):
        for world in (1, 2, 3, 8):
            spans = [slab_cells(Z, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == max(Z - 1, 0)
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [c1 - c0 for c0, c1 in spans]
            assert max(sizes) - min(sizes) <= 1
            for r in range(world):
                z0, z1 = slab_planes(Z, world, r)
                c0, c1 = spans[r]
                assert (z1 - z0) == ((c1 - c0 + 1) if c1 > c0 else 0)
    with pytest.raises(ValueError):
        slab_cells(10, 2, 2)
