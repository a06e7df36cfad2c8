"""The multi-GPU path's host logic (volume-parallel replicas) on CPU: two
gloo ranks, each correcting its own volumes with the oracle, the timing
protocol (barriers, maximum over ranks) and the whole-job throughput.
No GPU and no collective on the data path, as on the GPUs."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(here, "..", "cuda-n4_b200"))
    sys.path.insert(0, os.path.join(here, "..", "oracle"))
    import torch
    import n4_oracle as O
    from n4b200.phantom import make_phantom
    from n4b200.replicas import Replicas, volume_seeds
    rep = Replicas(world, torch.device("cpu"), backend="gloo", timeout_s=60)
    assert rep.rank == rank
    seeds = volume_seeds(rank, 2)
    rep.barrier()
    lat = []
    for sd in seeds:
        ph = make_phantom((16, 16, 12), seed=sd)
        _, L = O.N4(ph.im, ph.mask, low_value=0, maximumNumberOfLevels=1, maximumNumberOfIterations=[2],
                    ConvergenceThreshold=0.0)
        lat.append(L)
    rep.barrier()
    ms = 10.0 * (rank + 1)                    # a stand-in device time per rank
    mx = rep.max_over_ranks(ms)
    thr = rep.throughput(len(seeds), ms)
    np.savez(os.path.join(out_dir, f"rank{rank}.npz"), seeds=np.array(seeds), lat=np.stack(lat), mx=mx, thr=thr)
    rep.close()


def test_two_gloo_ranks_shard_volumes_and_time_by_the_slowest(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        assert p.exitcode == 0
    r0, r1 = (np.load(tmp_path / f"rank{r}.npz") for r in range(2))
    # disjoint volumes, different corrections
    assert not set(r0["seeds"]) & set(r1["seeds"])
    assert not np.allclose(r0["lat"], r1["lat"])
    # both ranks agree on the slowest rank's time and the whole-job rate
    assert float(r0["mx"]) == float(r1["mx"]) == 20.0
    assert float(r0["thr"]) == float(r1["thr"]) == pytest.approx(2 * 2 / 0.020)


def test_shard_covers_every_item_once():
    from n4b200.replicas import shard
    for n in (0, 1, 7, 48):
        for world in (1, 2, 3, 8):
            got = [i for r in range(world) for i in shard(n, r, world)]
            assert got == list(range(n))
