"""The multi-GPU path on CPU: primaries (or whole events) split over two gloo
ranks, each transporting its share with the oracle on its global substreams,
tallies and counters summed by all_reduce, must reproduce the single-process
run of all primaries."""
import os
import socket

import numpy as np
import pytest

from geantexascalepilot_b200 import sharding


def test_partition_covers_contiguously():
    for n in (0, 1, 7, 64, 1001):
        for world in (1, 2, 3, 8):
            spans = [sharding.partition(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        sharding.partition(10, 2, 2)


def test_partition_events_keeps_events_whole():
    ev = np.repeat(np.arange(9), [3, 0, 2, 5, 1, 1, 0, 4, 2]).astype(np.int32)
    spans = [sharding.partition_events(ev, 9, r, 4) for r in range(4)]
    assert spans[0][0] == 0 and spans[-1][1] == len(ev)
    for (a, b), r in zip(spans, range(4)):
        e0, e1 = sharding.partition(9, r, 4)
        assert np.all((ev[a:b] >= e0) & (ev[a:b] < e1))
    with pytest.raises(ValueError):
        sharding.partition_events(ev[::-1], 9, 0, 2)


def _workload(name):
    from geantexascalepilot_b200 import configs
    if name == "c2":
        cfg, prims, nvol = configs.c2(6)
        prims = (prims[0], np.full(len(prims[0]), 300.0), prims[2], prims[3], None)
    else:
        cfg, prims, nvol = configs.c5(nevents=7, mean=2)
        prims = (prims[0], np.full(len(prims[0]), 200.0), prims[2], prims[3], prims[4])
    return cfg, prims, nvol


def _oracle_run(nvol):
    from oracle_ctypes import Oracle, oracle_config
    import torch
    orc = Oracle()

    def run(cfg, sub):
        types, E, pos, d, ev = sub
        r = orc.transport(oracle_config(cfg, 2), types, E, pos, d, events=ev, nvol=nvol, nevents=cfg.nevents)
        st = {k: r[k] for k in sharding.SUM_KEYS if k in r}
        return torch.from_numpy(r["edep"].copy()), st
    return run


def _rank(rank, world, port, name, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cfg, prims, nvol = _workload(name)
        edep, st = sharding.transport_sharded(cfg, prims, nvol, rank, world, _oracle_run(nvol))
        if rank == 0:
            np.savez(out, edep=edep.numpy(), steps=st["steps"], tracks=st["tracks"], nprim=st["nprim"],
                     escaped=st["escaped"])
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("name", ["c2", "c5"])
def test_two_gloo_ranks_reproduce_one_process(oracle, tmp_path, name):
    import torch.multiprocessing as mp
    out = str(tmp_path / "r0.npz")
    mp.start_processes(_rank, args=(2, _free_port(), name, out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    cfg, prims, nvol = _workload(name)
    edep, st = _oracle_run(nvol)(cfg, prims)
    assert int(got["nprim"]) == len(prims[0])
    assert int(got["steps"]) == st["steps"] and int(got["tracks"]) == st["tracks"]
    np.testing.assert_allclose(got["edep"], edep.numpy(), rtol=1e-12, atol=1e-12 * float(edep.abs().max()))
    assert np.isclose(float(got["escaped"]), st["escaped"], rtol=1e-12, atol=1e-9)
