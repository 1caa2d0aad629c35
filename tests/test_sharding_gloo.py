"""N>1 replica path on CPU: two gloo ranks shard the protocol like the reference's workers,
compute their blocks with the oracle, and report the max elapsed time."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from dcs245_classical_sampling_b200.sampling import make_protocol
        from dcs245_classical_sampling_b200.sharding import gather_ids, max_over_ranks, shard
        from dcs245_classical_sampling_b200.workloads import build_workload
        from oracle import block_ref, sampler_ref
        w = build_workload("ring16_d20_t24_k8")
        proto = make_protocol(11, 6, w["n"], w["open_vertices"])
        mine = shard(proto["records"], rank, world)
        eng = block_ref.OracleEngine(w["graph"], w["unitaries"], w["n"], w["order"], w["parity_operations"],
                                     w["open_vertices"])
        picks = {}
        for r in mine:
            v, _ = eng.block(np.array([int(c) for c in r["input_data_bits"]], np.uint8))
            picks[r["sample_id"]] = sampler_ref.draw(v, r["draw_uniform"])["A_index"]
        ids = gather_ids(sorted(picks))
        mx = max_over_ranks(1.0 + rank)
        q.put((rank, ids, mx, picks))
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_partition_samples():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ids = out[0][1]
    assert sorted(ids[0] + ids[1]) == list(range(6))
    assert all(i % 2 == 0 for i in ids[0]) and all(i % 2 == 1 for i in ids[1])
    assert all(o[2] == 2.0 for o in out)
    # the same sample drawn by a single process gives the same index
    from dcs245_classical_sampling_b200.sampling import make_protocol
    from dcs245_classical_sampling_b200.workloads import build_workload
    from oracle import block_ref, sampler_ref
    w = build_workload("ring16_d20_t24_k8")
    eng = block_ref.OracleEngine(w["graph"], w["unitaries"], w["n"], w["order"], w["parity_operations"],
                                 w["open_vertices"])
    rec = make_protocol(11, 6, w["n"], w["open_vertices"])["records"][3]
    v, _ = eng.block(np.array([int(c) for c in rec["input_data_bits"]], np.uint8))
    picks = {**out[0][3], **out[1][3]}
    assert picks[3] == sampler_ref.draw(v, rec["draw_uniform"])["A_index"]
