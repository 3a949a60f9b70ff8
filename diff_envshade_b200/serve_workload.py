"""The serving workload: Poisson request arrivals against the continuous-batching server, and the
same arrival schedule replayed as serial plain launches.

Workload (seeded): ``n`` requests arriving as a Poisson process at ``rate`` per second; point count
log-uniform in [1k, 500k]; env map 16x32 or 32x64 (50/50); visibility on/off (50/50), on meaning the
points are bound to one of a few resident meshes (random triangles, Dirichlet barycentrics,
Bernoulli(0.7) visibility bits); 70% forward-only, 30% forward + all gradients; point attributes
drawn as for the plain config (unit normals, views in the normal's hemisphere, U[0,1] albedo,
U[0.2,0.9] roughness, U[0,0.1] specular).  Point data comes from a few pre-generated pinned pools
(request i uses a prefix of pool i mod n_pools) so that the host side costs nothing at submit time.

Latency of a request = time its outputs are in host memory - its arrival time.
"""
import gc
import math
import time

import numpy as np
import torch

from . import workloads as wl

MAX_P = 500000


class Pools:
    def __init__(self, n_pools=4, n_out=8, n_meshes=2, seed=4242):
        g = torch.Generator().manual_seed(seed)
        self.points = []
        for i in range(n_pools):
            inp = wl.make_inputs(MAX_P, 4, 8, seed=seed + i)
            tri = torch.randint(0, 200000, (MAX_P,), generator=g)
            e = -torch.log(torch.rand(3, MAX_P, generator=g).clamp_min(1e-12))
            bary = (e / e.sum(0, keepdim=True)).contiguous()
            d = {k: getattr(inp, k).pin_memory() for k in ("normal", "view_dir", "albedo", "specular_albedo",
                                                            "roughness", "grad_shading", "grad_diffuse_shading")}
            d["tri"] = tri.pin_memory()
            d["bary"] = bary.pin_memory()
            self.points.append(d)
        pin = dict(dtype=torch.float32, pin_memory=True)
        self.outputs = []
        for _ in range(n_out):
            o = {"shading": torch.empty(MAX_P, 3, **pin), "diffuse_shading": torch.empty(MAX_P, 3, **pin)}
            for k in ("g_normal", "g_view_dir", "g_albedo", "g_specular_albedo"):
                o[k] = torch.empty(MAX_P, 3, **pin)
            o["g_roughness"] = torch.empty(MAX_P, 1, **pin)
            o["g_envmap"] = torch.empty(3, 32, 64, **pin)
            self.outputs.append(o)
        self.envs = {(16, 32): [torch.exp(torch.randn(3, 16, 32, generator=g)) for _ in range(2)],
                     (32, 64): [torch.exp(torch.randn(3, 32, 64, generator=g)) for _ in range(2)]}
        self.meshes = []
        for _ in range(n_meshes):
            faces = torch.randint(0, 100000, (3, 200000), generator=g).to(torch.int32)
            bits = torch.rand(100000, 64 * 32, generator=g) < 0.7
            self.meshes.append((faces.contiguous(), wl.pack_bits(bits)))


def make_schedule(n=2000, rate=5000.0, seed=7):
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n))
    P = np.exp(rng.uniform(math.log(1000), math.log(MAX_P), size=n)).round().astype(np.int64)
    res = np.where(rng.random(n) < 0.5, 0, 1)          # 0: 16x32, 1: 32x64
    vis = rng.random(n) < 0.5
    backward = rng.random(n) < 0.3
    env_pick = rng.integers(0, 2, size=n)
    mesh_pick = rng.integers(0, 2, size=n)
    return [dict(t=float(arrivals[i]), P=int(P[i]), res=((16, 32), (32, 64))[res[i]], vis=bool(vis[i]),
                 backward=bool(backward[i]), env=int(env_pick[i]), mesh=int(mesh_pick[i])) for i in range(n)]


def prepare_barycentrics(pools, sched):
    """Per-request 3 x P barycentric tensors (visibility requests only), carved out of one pinned
    buffer before the run so that submitting costs no host copies."""
    total = sum(3 * r["P"] for r in sched if r["vis"])
    buf = torch.empty(max(total, 1), dtype=torch.float32, pin_memory=True)
    out, off = [None] * len(sched), 0
    for i, r in enumerate(sched):
        if r["vis"]:
            P = r["P"]
            v = buf[off:off + 3 * P].view(3, P)
            v.copy_(pools.points[i % len(pools.points)]["bary"][:, :P])
            out[i] = v
            off += 3 * P
    return out


def _summarize(lat_s, sched, makespan_s):
    """p50/p99/mean/max latency (ms) over all requests and over the 50k-100k-point 16x32 class, and
    throughput: requests per second and point x texel pairs per second, a request with gradients
    counting its pairs twice (forward and adjoint pass)."""
    lat = np.asarray(lat_s) * 1e3
    pairs = sum(r["P"] * r["res"][0] * r["res"][1] * (2 if r["backward"] else 1) for r in sched)
    cls = [i for i, r in enumerate(sched) if 50000 <= r["P"] <= 100000 and r["res"] == (16, 32)]
    out = {"requests": len(sched), "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
           "mean_ms": float(lat.mean()), "max_ms": float(lat.max()), "makespan_s": makespan_s,
           "throughput_req_per_s": len(sched) / makespan_s,
           "throughput_point_texel_per_s": pairs / makespan_s}
    if cls:
        out["class_50k_100k_16x32"] = {"n": len(cls), "p50_ms": float(np.percentile(lat[cls], 50)),
                                       "p99_ms": float(np.percentile(lat[cls], 99))}
    return out


def run_served(pools, sched, bary, device=0, hbm_budget_bytes=40 << 30, tick_us=50, ticks_in_flight=None,
               trace=False, order_min_points=None, rank_by_size=None):
    from .serving import Server
    srv = Server(device=device, hbm_budget_bytes=hbm_budget_bytes, tick_us=tick_us, ticks_in_flight=ticks_in_flight,
                 order_min_points=order_min_points, rank_by_size=rank_by_size)
    try:
        env_ids = {k: [srv.add_envmap(e) for e in v] for k, v in pools.envs.items()}
        mesh_ids = [srv.add_mesh(f, b) for f, b in pools.meshes]
        torch.cuda.synchronize()
        reqs = [None] * len(sched)
        # no collector pause inside the arrival loop (a full collection stalls submission for tens
        # of milliseconds and turns the Poisson schedule into a burst)
        gc.collect()
        gc.disable()
        t0 = time.perf_counter()
        for i, r in enumerate(sched):
            while time.perf_counter() - t0 < r["t"]:
                pass
            pt = pools.points[i % len(pools.points)]
            P = r["P"]
            outs = {k: (v if k == "g_envmap" else v[:P]) for k, v in pools.outputs[i % len(pools.outputs)].items()}
            if not r["backward"]:
                outs = {k: outs[k] for k in ("shading", "diffuse_shading")}
            else:
                H, W = r["res"]
                outs["g_envmap"] = outs["g_envmap"].view(-1)[:3 * H * W].view(3, H, W)
            reqs[i] = srv.submit(pt["normal"][:P], pt["view_dir"][:P], pt["albedo"][:P], pt["specular_albedo"][:P],
                                 pt["roughness"][:P], env_id=env_ids[r["res"]][r["env"]],
                                 mesh_id=mesh_ids[r["mesh"]] if r["vis"] else -1,
                                 nearest_triangle_id=pt["tri"][:P], barycentric_coord=bary[i],
                                 backward=r["backward"], grad_shading=pt["grad_shading"][:P],
                                 grad_diffuse_shading=pt["grad_diffuse_shading"][:P], outputs=outs)
        srv.drain(120)
        srv.poll(len(sched) + 16)
        stats = srv.stats()
    finally:
        gc.enable()
        srv.close()
    bad = [q.status for q in reqs if q.status != 0]
    if bad:
        raise RuntimeError(f"{len(bad)} served requests failed (status {bad[0]})")
    # latency from the arrival time (submit happened at the arrival, to within the spin loop)
    lat = [(q.done[2] - q.done[0]) * 1e-9 for q in reqs]
    first = min(q.done[0] for q in reqs)
    last = max(q.done[2] for q in reqs)
    out = _summarize(lat, sched, (last - first) * 1e-9)
    cls = [i for i, r in enumerate(sched) if 50000 <= r["P"] <= 100000 and r["res"] == (16, 32)]
    if cls:
        # where the class's time goes: wait for memory, upload, ordering, compute, download (p50 / p99, ms)
        st = [reqs[i].stages for i in cls]
        parts = {"admit": [x["admit"] - x["submit"] for x in st], "upload": [x["uploaded"] - x["admit"] for x in st],
                 "order": [x["ready"] - x["uploaded"] for x in st],
                 "compute": [x["computed"] - x["ready"] for x in st], "download": [x["done"] - x["computed"] for x in st]}
        out["class_50k_100k_16x32"]["stages_ms"] = {
            k: [float(np.percentile(v, 50)) * 1e-6, float(np.percentile(v, 99)) * 1e-6] for k, v in parts.items()}
    if trace:  # per request: points, texels, visibility, backward, then its stage times in ns
        keys = ("submit", "admit", "uploaded", "ready", "computed", "done")
        out["trace"] = [[r["P"], r["res"][0] * r["res"][1], int(r["vis"]), int(r["backward"])] +
                        [q.stages[k] for k in keys] for r, q in zip(sched, reqs)]
    out["ticks"] = stats["ticks"]
    out["items_per_tick"] = stats["items"] / max(stats["ticks"], 1)
    out["peak_arena_gb"] = stats["peak_arena_bytes"] / 2**30
    out["device_error"] = stats["device_error"]
    return out


def run_serial_plain(pools, sched, bary, device=0):
    """The same arrivals served one at a time, in arrival order, by the plain operators: host-to-
    device copy, forward (and backward), device-to-host copy, synchronise."""
    import diff_envshade_b200 as des
    dev = torch.device("cuda", device)
    envs = {k: [e.to(dev) for e in v] for k, v in pools.envs.items()}
    meshes = [(f.to(dev), b.to(dev)) for f, b in pools.meshes]
    R = torch.eye(3, device=dev)
    lat = []
    gc.collect()
    gc.disable()
    t0 = time.perf_counter()
    first = None
    for i, r in enumerate(sched):
        while time.perf_counter() - t0 < r["t"]:
            pass
        start = time.perf_counter()
        first = start if first is None else first
        pt = pools.points[i % len(pools.points)]
        P = r["P"]
        d = {k: pt[k][:P].to(dev, non_blocking=True) for k in ("normal", "view_dir", "albedo", "specular_albedo",
                                                                  "roughness")}
        env = envs[r["res"]][r["env"]]
        base = (d["normal"], d["view_dir"], d["albedo"], d["specular_albedo"], d["roughness"], env, R)
        if r["vis"]:
            f, b = meshes[r["mesh"]]
            v = (f, pt["tri"][:P].to(dev, non_blocking=True), bary[i].to(dev, non_blocking=True), b)
            sh, wh = des.bruteforce_specularvisibility_shader_forward2(*base, *v, True)
        else:
            sh, wh = des.bruteforce_specular_shader_forward2(*base, True)
        outs = [sh, wh]
        if r["backward"]:
            gs = pt["grad_shading"][:P].to(dev, non_blocking=True)
            gw = pt["grad_diffuse_shading"][:P].to(dev, non_blocking=True)
            if r["vis"]:
                outs += des.bruteforce_specularvisibility_shader_backward2(gs, gw, *base, *v, True)
            else:
                outs += des.bruteforce_specular_shader_backward2(gs, gw, *base, True)
        host = pools.outputs[i % len(pools.outputs)]
        host["shading"][:P].copy_(outs[0], non_blocking=True)
        host["diffuse_shading"][:P].copy_(outs[1], non_blocking=True)
        if r["backward"]:
            for k, o in zip(("g_normal", "g_view_dir", "g_albedo", "g_specular_albedo", "g_roughness"), outs[2:7]):
                host[k][:P].copy_(o, non_blocking=True)
        torch.cuda.synchronize(dev)
        lat.append(time.perf_counter() - t0 - r["t"])
    gc.enable()
    makespan = time.perf_counter() - first
    return _summarize(lat, sched, makespan)


def run(n=2000, rate=5000.0, tick_us=50, serial=True, hbm_budget_bytes=40 << 30, seed=7, ticks_in_flight=None):
    """Both arms on one arrival schedule; returns {"served": ..., "serial_plain": ...}."""
    pools = Pools()
    sched = make_schedule(n=n, rate=rate, seed=seed)
    bary = prepare_barycentrics(pools, sched)
    res = {"workload": f"{n} requests, Poisson {rate:.0f}/s, P log-uniform [1k, 500k], 16x32|32x64 env, "
                       "visibility 50%, backward 30%", "tick_us": tick_us, "ticks_in_flight": ticks_in_flight}
    res["served"] = run_served(pools, sched, bary, hbm_budget_bytes=hbm_budget_bytes, tick_us=tick_us,
                               ticks_in_flight=ticks_in_flight)
    if serial:
        res["serial_plain"] = run_serial_plain(pools, sched, bary)
    return res


def run_single(P, vis=False, backward=False, reps=2, H=16, W=32, tick_us=50, seed=4242, where="host",
               order_min_points=None):
    """One request shape submitted `reps` times, one after the other, to an otherwise idle server:
    each one's compute time (ready -> last tile done, ms) and the ticks it took.  For timing and
    profiling the batch kernel on a single kind of tile.  where="host": inputs and outputs in
    pinned host memory (read and written in place over the host link); "device": inputs in device
    memory (read in place, no host link).  order_min_points: the server's ordering threshold (an
    ordered request is uploaded first)."""
    from .serving import Server
    g = torch.Generator().manual_seed(seed)
    inp = wl.make_inputs(P, 4, 8, seed=seed)
    pin = {k: getattr(inp, k).pin_memory() for k in ("normal", "view_dir", "albedo", "specular_albedo", "roughness",
                                                      "grad_shading", "grad_diffuse_shading")}
    if where == "device":
        pin = {k: v.cuda() for k, v in pin.items()}
    kw = {}
    with Server(device=0, hbm_budget_bytes=4 << 30, tick_us=tick_us, order_min_points=order_min_points) as srv:
        env_id = srv.add_envmap(torch.exp(torch.randn(3, H, W, generator=g)))
        if vis:
            faces = torch.randint(0, 100000, (3, 200000), generator=g).to(torch.int32)
            bits = wl.pack_bits(torch.rand(100000, (H * W + 31) // 32 * 32, generator=g) < 0.7)
            e = -torch.log(torch.rand(3, P, generator=g).clamp_min(1e-12))
            kw = dict(mesh_id=srv.add_mesh(faces, bits),
                      nearest_triangle_id=torch.randint(0, 200000, (P,), generator=g).pin_memory(),
                      barycentric_coord=(e / e.sum(0, keepdim=True)).contiguous().pin_memory())
            if where == "device":
                kw["nearest_triangle_id"] = kw["nearest_triangle_id"].cuda()
                kw["barycentric_coord"] = kw["barycentric_coord"].cuda()
        times = []
        for _ in range(reps):
            r = srv.submit(pin["normal"], pin["view_dir"], pin["albedo"], pin["specular_albedo"], pin["roughness"],
                           env_id=env_id, backward=backward, grad_shading=pin["grad_shading"],
                           grad_diffuse_shading=pin["grad_diffuse_shading"], **kw)
            srv.drain(60)
            srv.poll()
            if r.status != 0:
                raise RuntimeError(f"request failed (status {r.status})")
            times.append((r.stages["computed"] - r.stages["ready"]) * 1e-6)
        st = srv.stats()
    return {"points": P, "texels": H * W, "visibility": vis, "backward": backward, "inputs": where,
            "order_min_points": order_min_points, "compute_ms": times, "ticks": st["ticks"],
            "device_error": st["device_error"]}


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=2000)
    ap.add_argument("--rate", type=float, default=5000.0)
    ap.add_argument("--tick-us", type=int, default=50)
    ap.add_argument("--seed", type=int, default=7, help="seed of the arrival schedule")
    ap.add_argument("--ticks-in-flight", type=int, default=None)
    ap.add_argument("--no-serial", action="store_true")
    ap.add_argument("--single", type=int, default=0, help="time one request of this many points instead")
    ap.add_argument("--vis", action="store_true", help="(--single) with visibility")
    ap.add_argument("--backward", action="store_true", help="(--single) with gradients")
    ap.add_argument("--reps", type=int, default=2, help="(--single) submissions, one after the other")
    ap.add_argument("--device-inputs", action="store_true", help="(--single) inputs in device memory")
    ap.add_argument("--order-min-points", type=int, default=None, help="(--single) the ordering threshold")
    a = ap.parse_args()
    if a.single > 0:
        print(json.dumps(run_single(a.single, vis=a.vis, backward=a.backward, reps=a.reps, tick_us=a.tick_us,
                                    where="device" if a.device_inputs else "host",
                                    order_min_points=a.order_min_points)))
    else:
        print(json.dumps(run(n=a.n, rate=a.rate, tick_us=a.tick_us, serial=not a.no_serial,
                             ticks_in_flight=a.ticks_in_flight, seed=a.seed)))
