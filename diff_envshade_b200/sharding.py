"""Data-parallel sharding of the shading path over ranks.

Points are independent, so a batch splits across ranks by contiguous point ranges and the forward
and the point gradients need no exchange.  The env-map gradient is a sum over every point; ranks
that shade against one shared env map sum their partial gradients with one all-reduce of its
``3*H*W`` floats (the path's only collective; NCCL on GPUs, gloo in the CPU tests).
"""
import torch.distributed as dist


def shard_range(P, rank, world):
    """Contiguous [begin, end) point range of `rank`; sizes differ by at most one point."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of {world}")
    base, extra = divmod(P, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def allreduce_env_grad(g_env, group=None):
    """Sums the env-map gradient over the ranks of `group` in place and returns it."""
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(g_env, op=dist.ReduceOp.SUM, group=group)
    return g_env


def shard_inputs(inp, rank, world):
    """Point shard of a workloads.ShadeInputs (env map, rotation and mesh tables are shared)."""
    import copy
    b, e = shard_range(inp.P, rank, world)
    out = copy.copy(inp)
    for k in ("normal", "view_dir", "albedo", "specular_albedo", "roughness", "grad_shading",
              "grad_diffuse_shading", "nearest_triangle_id"):
        v = getattr(inp, k)
        if v is not None:
            setattr(out, k, v[b:e].contiguous())
    if inp.barycentric_coord is not None:
        out.barycentric_coord = inp.barycentric_coord[:, b:e].contiguous()
    return out


__all__ = ["shard_range", "allreduce_env_grad", "shard_inputs"]
