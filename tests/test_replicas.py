"""Multi-process (world size 2, gloo on CPU) test of the replica sharding:
ranks split the particles, score their own block with the oracle, and the
union of the ranks' blocks equals the single-process result; the job rate
uses all ranks' units over the slowest rank's time."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import importlib
    import sys

    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "tests"))
    from conftest import load_package
    load_package()
    synth = importlib.import_module("relion_b200.synth")
    replicas = importlib.import_module("relion_b200.replicas")
    import oracle  # conftest put oracle/ on the path
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        pr = synth.make_problem("tiny", P=5)
        first, count = replicas.particle_range(pr.P, rank, world)
        op = oracle.projector_for(pr)
        blocks = [oracle.diff2_coarse_f64(op, pr.eulers, pr.trans_x, pr.trans_y, pr.fimg_re[p], pr.fimg_im[p],
                                          pr.corr[p]) for p in range(first, first + count)]
        fake_ms = 10.0 + 5.0 * rank  # rank 1 is the slowest
        rate = replicas.job_rate(count * pr.O * pr.T, fake_ms, dist)
        gathered = [None] * world
        dist.all_gather_object(gathered, (first, count, blocks))
        if rank == 0:
            np.save(os.path.join(out_dir, "rate.npy"), np.array([rate, pr.P * pr.O * pr.T / 0.015]))
            full = [None] * pr.P
            for f, c, b in gathered:
                for i in range(c):
                    full[f + i] = b[i]
            np.save(os.path.join(out_dir, "sharded.npy"), np.stack(full))
    finally:
        dist.destroy_process_group()


def test_particle_range_partitions():
    from conftest import load_package
    load_package()
    import importlib
    replicas = importlib.import_module("relion_b200.replicas")
    for P in (0, 1, 5, 256, 1023):
        for world in (1, 2, 3, 8):
            spans = [replicas.particle_range(P, r, world) for r in range(world)]
            assert sum(c for _, c in spans) == P
            pos = 0
            for f, c in spans:
                assert f == pos and c >= 0
                pos += c
            assert max(c for _, c in spans) - min(c for _, c in spans) <= 1
    with pytest.raises(ValueError):
        replicas.particle_range(4, 2, 2)


def test_two_rank_sharding_matches_single_process(tmp_path, oracle):
    import importlib

    import torch.multiprocessing as mp
    from conftest import load_package
    load_package()
    synth = importlib.import_module("relion_b200.synth")
    mp.start_processes(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    sharded = np.load(tmp_path / "sharded.npy")
    pr = synth.make_problem("tiny", P=5)
    op = oracle.projector_for(pr)
    single = np.stack([oracle.diff2_coarse_f64(op, pr.eulers, pr.trans_x, pr.trans_y, pr.fimg_re[p],
                                               pr.fimg_im[p], pr.corr[p]) for p in range(pr.P)])
    np.testing.assert_array_equal(sharded, single)
    rate, expect = np.load(tmp_path / "rate.npy")
    assert rate == pytest.approx(expect)  # all units over the slowest rank's 15 ms
