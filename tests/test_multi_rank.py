"""Multi-rank path on CPU (gloo, world size 2): ensembles sharded over ranks with disjoint seeds,
each rank renders its shard (the O2 oracle stands in for a rank's GPU on this CPU-only test), the
accumulations are summed with one all-reduce and must equal a single-process render of all
ensembles (counts exactly, colour within f32 re-association error); max-over-ranks timing."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT, load_package

pkg = load_package()
from gps_pbvr_web_b200 import multi  # noqa: E402


def test_shard_covers_every_ensemble_once():
    for count in [0, 1, 5, 64, 191]:
        for world in [1, 2, 3, 8]:
            got = []
            for r in range(world):
                first, n = multi.shard(count, world, r)
                got += list(range(first, first + n))
            assert got == list(range(count))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_dir):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle as O
    from _scenes import BG, cam17, scene, to_gpu, verify_scenes
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    g = to_gpu(scene(verify_scenes()[3][1]))
    pkgl = load_package()
    p = pkgl.RenderParams(spp_side=2, background=BG)
    count, first_seed = 9, 40
    seed = multi.rank_first_seed(first_seed, count, world, rank)
    _, n = multi.shard(count, world, rank)
    acc, st, _, _ = O.o2_render_ensembles(g, None, 0, O.radius_lut(), 48, 48, 2, cam17(focal=100.0), p.to_c(), seed, n)
    t = torch.from_numpy(acc.copy())
    multi.reduce_accum(t, dist)
    ms = multi.max_over_ranks(float(10 + rank), dist)
    if rank == 0:
        np.save(os.path.join(out_dir, "acc.npy"), t.numpy())
        np.save(os.path.join(out_dir, "ms.npy"), np.array([ms]))
    dist.barrier()
    dist.destroy_process_group()


def test_gloo_two_ranks_equal_one_process(tmp_path):
    import oracle as O
    from _scenes import BG, cam17, scene, to_gpu, verify_scenes
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    acc = np.load(tmp_path / "acc.npy")
    assert float(np.load(tmp_path / "ms.npy")[0]) == 11.0
    g = to_gpu(scene(verify_scenes()[3][1]))
    p = pkg.RenderParams(spp_side=2, background=BG)
    ref, _, _, _ = O.o2_render_ensembles(g, None, 0, O.radius_lut(), 48, 48, 2, cam17(focal=100.0), p.to_c(), 40, 9)
    assert np.array_equal(acc[:, 3], ref[:, 3])
    assert np.allclose(acc[:, :3], ref[:, :3], rtol=1e-5, atol=1e-5)
