"""Particles split over two ranks (world size 2, gloo on CPU): the exchange
step of a multi-GPU reconstruction.  Each rank inserts its shard
(bsoft_b200.shard.shard_indices) with the FP64 oracle, the partial sums go
to rank 0 in rank order (gather_partials), and reduce_partial_maps adds
them into rank 0's reconstructor through the same calls a Reconstructor
takes.  The summed accumulators and the finished map must equal the
oracle's single pass over all particles (the reference sums its per-thread
partial maps the same way, mg_reconstruct.cpp:263-324)."""
import datetime
import os
import socket
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CASE = "ctf16_tri_flip"


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class _Accumulators:
    """Stands in for a Reconstructor: accumulators() / add_partial()."""

    def __init__(self, vol, w, N):
        self.N = N
        self.vol = (vol[0::2] + 1j * vol[1::2]).reshape(N, N, N)
        self.w = w.reshape(N, N, N).copy()

    def accumulators(self, half=0):
        return self.vol.copy(), self.w.copy()

    def add_partial(self, vol, weight, half=0):
        self.vol = self.vol + vol
        self.w = self.w + weight


def _worker(rank, world, port, outdir):
    sys.path.insert(0, os.path.dirname(HERE))
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import oracle
        from bsoft_b200.shard import gather_partials, reduce_partial_maps, shard_indices, sum_in_rank_order
        from tests.helpers import load_case
        d = os.path.join(outdir, f"rank{rank}")
        os.makedirs(d, exist_ok=True)
        plan, images, _ = load_case(CASE, d)
        idx = shard_indices(len(plan.params), rank, world)
        vol, w, _, _ = oracle.insert(plan, images[idx], plan.params[idx])
        parts = gather_partials([vol, w])
        fake = _Accumulators(vol, w, plan.map)
        reduce_partial_maps(fake)
        if rank == 0:
            assert len(parts) == world
            tv, tw = sum_in_rank_order(parts)
            np.savez(os.path.join(outdir, "sums.npz"), vol=tv, w=tw, fvol=fake.vol, fw=fake.w)
    finally:
        dist.destroy_process_group()


def test_partial_maps_over_two_ranks(tmp_path):
    import torch.multiprocessing as mp
    sys.path.insert(0, os.path.dirname(HERE))
    import oracle
    from tests.helpers import load_case
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    z = np.load(os.path.join(str(tmp_path), "sums.npz"))
    (tmp_path / "all").mkdir()
    plan, images, _ = load_case(CASE, str(tmp_path / "all"))
    vol, w, _, _ = oracle.insert(plan, images, plan.params)
    # the rank-order sum of the two shards against one pass over all particles
    assert np.linalg.norm(z["vol"] - vol) <= 1e-12 * np.linalg.norm(vol)
    assert np.linalg.norm(z["w"] - w) <= 1e-12 * np.linalg.norm(w)
    # reduce_partial_maps on rank 0 gives the same sums, bit for bit
    N = plan.map
    assert np.array_equal(z["fvol"], (z["vol"][0::2] + 1j * z["vol"][1::2]).reshape(N, N, N))
    assert np.array_equal(z["fw"], z["w"].reshape(N, N, N))
    # and the finished maps agree
    m_split, _ = oracle.finish(plan, z["vol"], z["w"])
    m_all, _ = oracle.finish(plan, vol, w)
    assert np.linalg.norm(m_split - m_all) <= 1e-10 * np.linalg.norm(m_all)


def test_shard_indices_partition():
    sys.path.insert(0, os.path.dirname(HERE))
    from bsoft_b200.shard import shard_indices
    n, world = 103, 4
    allidx = np.sort(np.concatenate([shard_indices(n, r, world) for r in range(world)]))
    assert np.array_equal(allidx, np.arange(n))
    with pytest.raises(ValueError):
        shard_indices(n, 4, 4)
