"""The multi-GPU layout on CPU: two gloo ranks (one process each, as torchrun
launches them) own disjoint members of the sweep and agree on the timing and
unit reductions bench.py uses; no other collective is involved."""
import os
import socket


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from bonzo_b200.parallel import max_over_ranks, rank_seed, sum_over_ranks, sweep_shard
        shard = sweep_shard(8, 0, rank)
        zones = sum(q["N"] ** 2 for q in shard)
        out[rank] = dict(seed=rank_seed(0, rank), sizes=[q["N"] for q in shard],
                         zones=zones, zones_all=sum_over_ranks(zones, dist),
                         ms_max=max_over_ranks(1.0 + rank, dist))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_the_sweep():
    import torch.multiprocessing as mp
    mgr = mp.Manager()
    out = mgr.dict()
    port = _free_port()
    mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
    r0, r1 = out[0], out[1]
    assert r0["seed"] != r1["seed"]
    assert r0["zones_all"] == r1["zones_all"] == r0["zones"] + r1["zones"]
    assert r0["ms_max"] == r1["ms_max"] == 2.0
    # each rank's members are a fixed function of its seed (weak scaling)
    from bonzo_b200.parallel import sweep_shard
    assert [q["N"] for q in sweep_shard(8, 0, 1)] == r1["sizes"]


def test_single_process_reductions_are_identity():
    from bonzo_b200.parallel import max_over_ranks, sum_over_ranks
    assert max_over_ranks(3.5) == 3.5 and sum_over_ranks(7) == 7.0
