"""World-size-2 test of the data-parallel path on CPU (gloo): point shards shaded independently,
env-map gradient summed with one all-reduce, compared with the unsharded result.  The shading
itself runs in the FP64 oracle (no GPU here); the sharding and the collective are the product's
(diff_envshade_b200.sharding)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, result_path):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from oracle import oracle as orc
        from diff_envshade_b200 import workloads as wl
        from diff_envshade_b200.sharding import shard_inputs, allreduce_env_grad
        inp = wl.make_inputs(101, 8, 16, seed=31, vis_p=0.7, vis_layout="mesh", rotation=True)
        mine = shard_inputs(inp, rank, world)
        f = orc.flags_for("specularvisibility2")
        table = orc.texel_table_f64(8, 16, inp.light2obj_rotmat)
        out = orc.backward(mine, f, mine.grad_shading, mine.grad_diffuse_shading, table=table)
        g_env = torch.from_numpy(out["g_env"])
        allreduce_env_grad(g_env)
        gathered = [None] * world
        dist.all_gather_object(gathered, out["g_normal"])
        if rank == 0:
            np.savez(result_path, g_env=g_env.numpy(), g_normal=np.concatenate(gathered))
    finally:
        dist.destroy_process_group()


def test_two_rank_env_gradient_allreduce(tmp_path):
    from oracle import oracle as orc
    from diff_envshade_b200 import workloads as wl
    path = str(tmp_path / "r.npz")
    mp.start_processes(_worker, args=(2, _free_port(), path), nprocs=2, join=True, start_method="spawn")
    got = np.load(path)
    inp = wl.make_inputs(101, 8, 16, seed=31, vis_p=0.7, vis_layout="mesh", rotation=True)
    f = orc.flags_for("specularvisibility2")
    table = orc.texel_table_f64(8, 16, inp.light2obj_rotmat)
    full = orc.backward(inp, f, inp.grad_shading, inp.grad_diffuse_shading, table=table)
    np.testing.assert_allclose(got["g_env"], full["g_env"], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(got["g_normal"], full["g_normal"], rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("P,world", [(0, 3), (5, 2), (101, 4), (70000, 8)])
def test_shard_ranges_partition_the_points(P, world):
    from diff_envshade_b200.sharding import shard_range
    rs = [shard_range(P, r, world) for r in range(world)]
    assert rs[0][0] == 0 and rs[-1][1] == P
    assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))
    sizes = [e - b for b, e in rs]
    assert max(sizes) - min(sizes) <= 1
