"""Benchmark: forward + backward point*texel throughput of the visibility-masked env-map shader.

Workload (per rank): 70,000 points x 16x32 env map with 512 packed visibility bits per point
(Bernoulli(0.7)), specular on, one forward (bruteforce_specularvisibility_shader_forward2) and
one backward (..._backward2) per step.  Metric = points * texels / (t_fwd + t_bwd).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl {b200,reference}]

Timing: W untimed warm-up steps; then K steps, each bracketed by CUDA events on the launching
stream; a 256 MiB buffer larger than the 126 MB L2 is rewritten between timed steps (outside the
events), and the normals are marked modified before every step (as an optimizer update would), so
the only ordering reused is the one the step's own forward computed for its backward.  The K steps
are run twice: launched eagerly op by op (per-kernel times from events around each main kernel),
then as replays of a CUDA graph of the same two operator calls, which runs every kernel of the step
without the host's per-call launch overhead; `value` is the graph-replay step time.  Multi-GPU (torchrun): every rank shades its own 70k points (weak scaling) and the
env-map gradients are summed over ranks with one NCCL all-reduce (the path's only exchange);
the reported time is the max over ranks.

At N = 1 the line also carries a serving leg ("serving"): 2000 requests (Poisson 5k/s, 1k-500k
points, 16x32 or 32x64 env, visibility on/off, 30% with gradients) through the continuous-batching
server against the same arrivals served one at a time by the plain operators (--no-serve skips it);
a relight leg ("relight"): 262,144 points x 64 env maps x 16x32 on the tensor cores against 64
plain FP32 passes (--no-relight skips it); and the same fwd+bwd step with the visibility of each
point interpolated over a random triangle ("mesh_layout") -- the headline workload gives every
point its own visibility row (barycentrics (1, 0, 0)), as a per-point visibility mask does.

``--impl reference`` times the CPU restatement of the reference's sum (the reference has no
CPU path of its own) on the host cores, on a bounded sample of the same workload.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fwd+bwd point*texel/s (70k pts, 16x32 env, 512-bit visibility)"
UNIT = "point*texel/s"
CONFIG_NAME = "vis-70k"

# Algorithmic FP32-pipe instructions per (point, texel) pair with visibility (FMA = 1), with texel
# tables and per-point constants hoisted: forward = visibility 8 + n.l 3 + Lambert 6 + GGX 40;
# fused adjoint = recompute 45 + Lambert adjoint 12 + GGX adjoint 84 + env-map accumulation 7.
INSTR_FWD_VIS = 57
INSTR_BWD_VIS = 148
FP32_LANES_PER_SM = 128


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving leg")
    ap.add_argument("--no-relight", action="store_true", help="skip the K-env-map relight leg")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """Samples SM clocks, power and clock-event (throttle) reasons through NVML from a background
    thread every ~2 ms while the timed region runs (read-only queries)."""

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self._stop = threading.Event()
        self.t = None

    def start(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            visible = os.environ.get("CUDA_VISIBLE_DEVICES")
            idx = int(visible.split(",")[self.gpu]) if visible and visible.split(",")[0].isdigit() else self.gpu
            self.h = pynvml.nvmlDeviceGetHandleByIndex(idx)
            self.nv = pynvml
        except Exception:
            self.h = None
            return
        self.max_mhz = self.nv.nvmlDeviceGetMaxClockInfo(self.h, self.nv.NVML_CLOCK_SM)
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()

    def _run(self):
        nv = self.nv
        while not self._stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                self.rows.append((sm, reasons))
            except Exception:
                pass
            time.sleep(0.002)

    def stop(self):
        if self.t is None:
            return None
        self._stop.set()
        self.t.join(timeout=2)
        if not self.rows:
            return None
        nv = self.nv
        names = {nv.nvmlClocksEventReasonHwSlowdown: "hw_slowdown",
                 nv.nvmlClocksEventReasonHwThermalSlowdown: "hw_thermal_slowdown",
                 nv.nvmlClocksEventReasonSwThermalSlowdown: "sw_thermal_slowdown",
                 nv.nvmlClocksEventReasonSwPowerCap: "sw_power_cap",
                 nv.nvmlClocksEventReasonHwPowerBrakeSlowdown: "hw_power_brake_slowdown"}
        reasons = sorted({n for _, r in self.rows for bit, n in names.items() if r & bit})
        return {"sm_mhz": float(np.median([s for s, _ in self.rows])), "sm_max_mhz": float(self.max_mhz),
                "reasons": reasons, "samples": len(self.rows), "source": "NVML, 2 ms polling"}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def committed_traffic():
    """DRAM bytes per launch of the adjoint kernel from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "bwd_kernel_vis70k_ncu.txt")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


# ------------------------------------------------------------------------------------------------
# CPU leg (oracle port): reference arm and cpu_baseline
# ------------------------------------------------------------------------------------------------

def cpu_port_throughput(inp, target_s=8.0, max_points=None):
    """FP32 oracle (C++ transcription of the reference sum) fwd+bwd on all host threads over a
    bounded sample of the workload's points; returns (point*texel/s, sample description, threads)."""
    from oracle import oracle as orc
    threads = os.cpu_count() or 1
    flags = orc.flags_for("specularvisibility2")
    HW = inp.HW
    gs = inp.grad_shading.numpy()
    gw = inp.grad_diffuse_shading.numpy()
    n = 512
    total_pairs, total_t, npts = 0, 0.0, 0
    while True:
        pts = np.arange(n) % inp.P
        t0 = time.perf_counter()
        orc.forward(inp, flags, dtype=np.float32, nthreads=threads, points=pts)
        orc.backward(inp, flags, gs, gw, dtype=np.float32, nthreads=threads, points=pts)
        dt = time.perf_counter() - t0
        total_pairs += n * HW
        total_t += dt
        npts += n
        if total_t >= target_s or (max_points and npts >= max_points):
            break
        n = int(min(max(n * 2, 512), inp.P))
    desc = (f"{npts} points x {HW} texels fwd+bwd (FP32 oracle, visibility), {threads} threads, "
            f"{total_t:.1f} s")
    return total_pairs / total_t, desc, threads


def load_workloads():
    """The seeded input generators (diff_envshade_b200/workloads.py, which needs only numpy and
    torch), loaded from their file so that the package -- and with it the native extension -- is
    not imported: the reference arm maps no library of this build."""
    import importlib.util
    path = os.path.join(ROOT, "diff_envshade_b200", "workloads.py")
    spec = importlib.util.spec_from_file_location("_des_bench_workloads", path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod  # dataclasses resolve the module by name
    spec.loader.exec_module(mod)
    return mod


def bench_config(P, H, W, nbits, world):
    """The `config` object of both arms' JSON lines (one definition, so they always agree)."""
    return {"workload": f"{CONFIG_NAME}: {P} points x {H}x{W} env, {nbits}-bit visibility, specular on, fwd+bwd",
            "points_per_rank": P, "texels": H * W, "parallelism": f"dp{world}" if world > 1 else "single",
            "l2": "256 MiB buffer rewritten between timed steps (outside the timed events)"}


def run_reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    wl = load_workloads()
    c = wl.CONFIGS[CONFIG_NAME]
    # rank 0's inputs of the GPU arm (same seed, same draws)
    inp = wl.make_inputs(c["P"], c["H"], c["W"], c["seed"], sigma=c["sigma"], rough=c["rough"], vis_p=c["vis_p"])
    # each step is a bounded sample; the whole arm stays within about two minutes
    per_step_s = min(2.0, max(0.05, 120.0 / max(args.steps + args.warmup, 1)))
    vals = []
    desc = threads = None
    for i in range(args.warmup + args.steps):
        v, desc, threads = cpu_port_throughput(inp, target_s=per_step_s)
        if i >= args.warmup:
            vals.append(v)
    value = float(np.mean(vals))
    pairs = inp.P * inp.HW
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": pairs / value * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded normals/views/materials, lognormal env, Bernoulli(0.7) bits)",
        "config": bench_config(inp.P, c["H"], c["W"], inp.visibility.shape[0] * 32, args.gpus),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": desc + "; the reference has no CPU path: C++ FP32 restatement of its sum "
                                          "(oracle port), each step a bounded sample of the workload's points"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------------------------------------
# GPU arm
# ------------------------------------------------------------------------------------------------

def bf16_peak():
    """Dense bf16 tensor peak (TFLOP/s) for a kernel timed alone: the burst figure of
    MEASURED_PEAKS.json, else this pool's earlier measurement."""
    peaks = measured_peaks()
    for k in ("bf16_tflops", "bf16_tflops_burst"):
        if k in peaks:
            return float(peaks[k]), f"{k} of MEASURED_PEAKS.json (measured)"
    return 1590.0, "fallback 1.59 PFLOP/s (earlier measurement on this pool; MEASURED_PEAKS.json absent)"


def relight_leg(des, wl, dev, flush, peak_tinst, steps=10, warmup=3):
    """K-env-map relighting (262,144 points x 64 maps x 16x32, 512-bit visibility) on tcgen05:
    the whole op (table, ordering, radiance tiles, tensor-core pass) and its tensor-core kernel alone,
    timed with CUDA events with the L2 flushed between passes; against 64 plain FP32 forward passes."""
    c = wl.CONFIGS["multienv-262k"]
    inp = wl.make_inputs(c["P"], c["H"], c["W"], c["seed"], sigma=c["sigma"], rough=c["rough"], vis_p=c["vis_p"],
                         env_count=c["K"])
    d = inp.to(dev)
    P, H, W, K = c["P"], c["H"], c["W"], c["K"]
    HW = H * W
    vis = (d.face_vertex_list, d.nearest_triangle_id, d.barycentric_coord, d.visibility)
    base = (d.normal, d.view_dir, d.albedo, d.specular_albedo, d.roughness)

    def fused():
        return des.relight_multienv(*base, d.envmap, d.light2obj_rotmat, *vis, True, True)

    def plain():
        return torch.stack([des.bruteforce_specularvisibility_shader_forward2(
            *base, d.envmap[k], d.light2obj_rotmat, *vis, True)[0] for k in range(K)], dim=1)

    for _ in range(warmup):
        fused()
    torch.cuda.synchronize()
    op_ms, kern_ms = [], []
    for i in range(steps):
        flush.fill_(float(i))
        e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        for x in e[2:]:
            x.record()  # torch creates events lazily
        des.set_timing_events(e[2].cuda_event, e[3].cuda_event)
        e[0].record()
        out = fused()
        e[1].record()
        des.set_timing_events(0, 0)
        torch.cuda.synchronize()
        op_ms.append(e[0].elapsed_time(e[1]))
        kern_ms.append(e[2].elapsed_time(e[3]))
    ref = plain()
    torch.cuda.synchronize()
    p_ms = []
    for i in range(3):
        flush.fill_(float(i))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        plain()
        b.record()
        torch.cuda.synchronize()
        p_ms.append(a.elapsed_time(b))
    scale = float(ref.abs().max())
    err = float(((out - ref).abs() / (ref.abs() + 1e-3 * scale)).max())
    op, kern, pl = float(np.median(op_ms)), float(np.median(kern_ms)), float(np.median(p_ms))
    build_tinst = P * HW * INSTR_FWD_VIS / (kern * 1e-3) / 1e12
    flops_alg = 2.0 * P * HW * 3 * K  # one [P x HW] x [HW x 3K] product per pass
    flops_exec = 3 * flops_alg        # BF16 hi*hi + lo*hi + hi*lo
    peak_tc, peak_src = bf16_peak()
    return {
        "workload": f"multienv-262k: {P} points x {K} env maps x {H}x{W}, 512-bit visibility, BF16 hi/lo on tcgen05",
        "ms_per_pass": op, "kernel_ms": kern, "value": P * HW * K / (op * 1e-3), "unit": "point*texel*map/s",
        "weight_build": {"bound": "fp32", "work": f"{INSTR_FWD_VIS} FP32-pipe instr per point*texel pair",
                         "achieved": build_tinst, "peak": peak_tinst, "unit": "T FP32-pipe instr/s",
                         "frac": build_tinst / peak_tinst},
        "tensor": {"achieved": flops_exec / (kern * 1e-3) / 1e12, "algorithmic": flops_alg / (kern * 1e-3) / 1e12,
                   "peak": peak_tc, "unit": "TFLOP/s", "frac": flops_exec / (kern * 1e-3) / 1e12 / peak_tc,
                   "peak_source": peak_src},
        "max_rel_err_vs_plain_fp32": err,
        "error_note": "per element |d| / (|plain| + 1e-3 max|plain|) against 64 plain FP32 forward passes; the FP64 "
                      "oracle comparison is tests/test_gpu_relight.py",
        "plain_64x_ms": pl, "speedup_vs_plain": pl / op,
        "l2": "256 MiB buffer rewritten between timed passes (outside the timed events)",
    }


def mesh_layout_step(des, wl, dev, flush, steps=10, warmup=3):
    """The same fwd+bwd step with visibility interpolated over random triangles (three vertex words
    per point and texel) instead of one visibility row per point."""
    c = wl.CONFIGS[CONFIG_NAME]
    d = wl.make_inputs(c["P"], c["H"], c["W"], c["seed"], sigma=c["sigma"], rough=c["rough"], vis_p=c["vis_p"],
                       vis_layout="mesh").to(dev)
    vis = (d.face_vertex_list, d.nearest_triangle_id, d.barycentric_coord, d.visibility)

    def step():
        torch.autograd.graph.increment_version(d.normal)
        des.bruteforce_specularvisibility_shader_forward2(d.normal, d.view_dir, d.albedo, d.specular_albedo,
                                                          d.roughness, d.envmap, d.light2obj_rotmat, *vis, True)
        des.bruteforce_specularvisibility_shader_backward2(d.grad_shading, d.grad_diffuse_shading, d.normal,
                                                           d.view_dir, d.albedo, d.specular_albedo, d.roughness,
                                                           d.envmap, d.light2obj_rotmat, *vis, True)

    for _ in range(warmup):
        step()
    ms = []
    for i in range(steps):
        flush.fill_(float(i))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        step()
        b.record()
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
    m = float(np.mean(ms))
    return {"ms_per_step": m, "value": c["P"] * c["H"] * c["W"] / (m * 1e-3), "unit": UNIT,
            "layout": "random triangles over P/2 vertices, Dirichlet barycentrics (three words per point and slot)"}

def main():
    args = parse()
    if args.impl == "reference":
        return run_reference_arm(args)

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
        pg = dist
    import diff_envshade_b200 as des
    from diff_envshade_b200 import workloads as wl
    from diff_envshade_b200.sharding import allreduce_env_grad

    c = wl.CONFIGS[CONFIG_NAME]
    inp_host = wl.make_inputs(c["P"], c["H"], c["W"], c["seed"] + 1000 * rank, sigma=c["sigma"], rough=c["rough"],
                              vis_p=c["vis_p"])
    d = inp_host.to(dev)
    P, HW = d.P, d.HW
    vis = (d.face_vertex_list, d.nearest_triangle_id, d.barycentric_coord, d.visibility)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def step():
        torch.autograd.graph.increment_version(d.normal)
        sh, wh = des.bruteforce_specularvisibility_shader_forward2(
            d.normal, d.view_dir, d.albedo, d.specular_albedo, d.roughness, d.envmap, d.light2obj_rotmat, *vis, True)
        g = des.bruteforce_specularvisibility_shader_backward2(
            d.grad_shading, d.grad_diffuse_shading, d.normal, d.view_dir, d.albedo, d.specular_albedo, d.roughness,
            d.envmap, d.light2obj_rotmat, *vis, True)
        allreduce_env_grad(g[5])
        return sh, wh, g

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    K = args.steps
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    kf = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    kb = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    for pair in kf + kb:  # torch creates events lazily: record once so the raw handles exist
        for e in pair:
            e.record()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    if pg is not None:
        pg.barrier()
    torch.cuda.synchronize()
    launches0 = des.kernel_launches()
    for i in range(K):
        flush.fill_(float(i))
        # a training step changes the points every step (the optimizer update): mark the normals as
        # modified so that no step can reuse an earlier step's point ordering -- only the backward
        # reuses the ordering its own forward computed
        torch.autograd.graph.increment_version(d.normal)
        ev[i][0].record()
        des.set_timing_events(kf[i][0].cuda_event, kf[i][1].cuda_event)
        sh, wh = des.bruteforce_specularvisibility_shader_forward2(
            d.normal, d.view_dir, d.albedo, d.specular_albedo, d.roughness, d.envmap, d.light2obj_rotmat, *vis, True)
        des.set_timing_events(kb[i][0].cuda_event, kb[i][1].cuda_event)
        g = des.bruteforce_specularvisibility_shader_backward2(
            d.grad_shading, d.grad_diffuse_shading, d.normal, d.view_dir, d.albedo, d.specular_albedo, d.roughness,
            d.envmap, d.light2obj_rotmat, *vis, True)
        des.set_timing_events(0, 0)
        allreduce_env_grad(g[5])
        ev[i][1].record()
    eager_launches = des.kernel_launches() - launches0
    torch.cuda.synchronize()
    if pg is not None:
        pg.barrier()
    eager_ms = float(np.sum([a.elapsed_time(b) for a, b in ev]))
    fwd_ms = [a.elapsed_time(b) for a, b in kf]
    bwd_ms = [a.elapsed_time(b) for a, b in kb]

    # The same step replayed as a CUDA graph of the two operator calls: every replay runs all of the
    # step's kernels (texel tables, point ordering, forward, adjoint, env-gradient reduction), with
    # the host's per-call launch overhead taken out -- on a shared host that overhead can exceed the
    # GPU time of the step and would otherwise be measured as GPU idle time.  This is the step time
    # the metric reports; the eagerly launched loop above gives the per-kernel times and is
    # reported beside it.
    def ops():
        torch.autograd.graph.increment_version(d.normal)
        des.bruteforce_specularvisibility_shader_forward2(
            d.normal, d.view_dir, d.albedo, d.specular_albedo, d.roughness, d.envmap, d.light2obj_rotmat, *vis, True)
        return des.bruteforce_specularvisibility_shader_backward2(
            d.grad_shading, d.grad_diffuse_shading, d.normal, d.view_dir, d.albedo, d.specular_albedo, d.roughness,
            d.envmap, d.light2obj_rotmat, *vis, True)

    side = torch.cuda.Stream(dev)
    side.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(side):
        for _ in range(2):
            ops()
    torch.cuda.current_stream(dev).wait_stream(side)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    l0 = des.kernel_launches()
    with torch.cuda.graph(graph):
        g_graph = ops()
    launches_per_step = des.kernel_launches() - l0
    for _ in range(args.warmup):
        graph.replay()
    gev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    torch.cuda.synchronize()
    if pg is not None:
        pg.barrier()
    torch.cuda.synchronize()
    for i in range(K):
        flush.fill_(float(i))
        gev[i][0].record()
        graph.replay()
        allreduce_env_grad(g_graph[5])
        gev[i][1].record()
    torch.cuda.synchronize()
    if pg is not None:
        pg.barrier()
    clocks = sampler.stop()
    total_ms = float(np.sum([a.elapsed_time(b) for a, b in gev]))
    if pg is not None:
        t = torch.tensor([total_ms, eager_ms], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        total_ms, eager_ms = float(t[0].item()), float(t[1].item())
    ms_per_step = total_ms / K
    value = world * P * HW / (ms_per_step * 1e-3)
    launches = launches_per_step * K
    del graph

    # ---- end-to-end through the reference-facing operators (the forward2 / backward2 pair a user of
    # the reference calls), host buffers, copies inside the timed region.  Every step copies all of
    # its inputs from pinned host memory and all of its outputs back.  The steps are pipelined the
    # way a caller with a stream of batches runs them: step i+1's inputs are uploaded on a copy
    # stream and step i-1's outputs downloaded on another while step i computes (double-buffered
    # device inputs, ordered by events).  The serial form (copy in, compute, copy out, one step after
    # the other) and the same pipeline through the autograd Functions are reported beside it.
    e2e = None
    if not args.no_e2e:
        hp = inp_host.pin()
        names = ["normal", "view_dir", "albedo", "specular_albedo", "roughness", "envmap", "light2obj_rotmat",
                 "face_vertex_list", "nearest_triangle_id", "barycentric_coord", "visibility", "grad_shading",
                 "grad_diffuse_shading"]
        leaves = ("normal", "view_dir", "albedo", "specular_albedo", "roughness", "envmap")
        h2d = sum(getattr(hp, k).numel() * getattr(hp, k).element_size() for k in names)
        main = torch.cuda.current_stream(dev)
        s_up, s_down = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
        # the step's inputs in one pinned block (each at a 256-byte offset), so a step's upload is one
        # copy; on the device, two such blocks whose views are the operator's input tensors
        offs, o = {}, 0
        for k in names:
            offs[k] = o
            o += (getattr(hp, k).numel() * getattr(hp, k).element_size() + 255) // 256 * 256
        host_block = torch.empty(o, dtype=torch.uint8, pin_memory=True)

        def views(block):
            out = {}
            for k in names:
                src = getattr(hp, k)
                nb = src.numel() * src.element_size()
                out[k] = block[offs[k]:offs[k] + nb].view(src.dtype).view(src.shape)
            return out

        for k, v in views(host_block).items():
            v.copy_(getattr(hp, k))
        dev_blocks = [torch.empty(o, dtype=torch.uint8, device=dev) for _ in range(2)]
        bufs = [views(b) for b in dev_blocks]
        ev_in = [torch.cuda.Event() for _ in range(2)]
        ev_free = [torch.cuda.Event() for _ in range(2)]
        ev_out = [torch.cuda.Event() for _ in range(2)]
        ev_down = [torch.cuda.Event() for _ in range(2)]
        stage, out_host = None, None

        def compute_ops(t):
            # the reference-facing operator pair, called as a user of the reference calls it
            vis_t = (t["face_vertex_list"], t["nearest_triangle_id"], t["barycentric_coord"], t["visibility"])
            base = (t["normal"], t["view_dir"], t["albedo"], t["specular_albedo"], t["roughness"], t["envmap"],
                    t["light2obj_rotmat"])
            sh, wh = des.bruteforce_specularvisibility_shader_forward2(*base, *vis_t, True)
            g = des.bruteforce_specularvisibility_shader_backward2(t["grad_shading"], t["grad_diffuse_shading"],
                                                                   *base, *vis_t, True)
            allreduce_env_grad(g[5])
            return [sh, wh] + list(g)

        def compute_autograd(t):
            t = dict(t)
            for k in leaves:
                t[k] = t[k].detach().requires_grad_(True)
            sh, wh = des.shade(t["normal"], t["view_dir"], t["albedo"], t["specular_albedo"], t["roughness"],
                               t["envmap"], t["light2obj_rotmat"],
                               visibility=(t["face_vertex_list"], t["nearest_triangle_id"], t["barycentric_coord"],
                                           t["visibility"]))
            torch.autograd.backward([sh, wh], [t["grad_shading"], t["grad_diffuse_shading"]])
            allreduce_env_grad(t["envmap"].grad)
            return [sh.detach(), wh.detach()] + [t[k].grad for k in leaves]

        compute_fn = [compute_ops]

        def compute(t):
            return compute_fn[0](t)

        def upload(i):
            b = i % 2
            s_up.wait_event(ev_free[b])  # step i-2 is done with this block
            with torch.cuda.stream(s_up):
                dev_blocks[b].copy_(host_block, non_blocking=True)
            ev_in[b].record(s_up)

        def pipelined_step(i, last):
            nonlocal stage, out_host
            if not last:
                upload(i + 1)
            b = i % 2
            main.wait_event(ev_in[b])
            outs = compute(bufs[b])
            ev_free[b].record(main)
            if stage is None:
                n_out = sum(x.numel() for x in outs)
                stage = [torch.empty(n_out, dtype=torch.float32, device=dev) for _ in range(2)]
                out_host = torch.empty(n_out, dtype=torch.float32, pin_memory=True)
            main.wait_event(ev_down[b])  # step i-2's download has left this staging block
            torch.cat([x.reshape(-1) for x in outs], out=stage[b])
            ev_out[b].record(main)
            s_down.wait_event(ev_out[b])
            with torch.cuda.stream(s_down):
                out_host.copy_(stage[b], non_blocking=True)
            ev_down[b].record(s_down)
            return stage[b].numel() * stage[b].element_size()

        def run_pipelined(n):
            start, end = torch.cuda.Event(), torch.cuda.Event()
            for e in ev_free + ev_down:
                e.record(main)
            start.record(main)
            s_up.wait_event(start)
            upload(0)
            d = 0
            for i in range(n):
                d = pipelined_step(i, i == n - 1)
            end.record(s_down)
            main.wait_event(end)  # the last download is inside the region
            return d

        serial_host = None

        def serial_step():
            nonlocal serial_host
            t = {k: getattr(hp, k).to(dev, non_blocking=True) for k in names}
            outs = compute(t)
            if serial_host is None:
                serial_host = [torch.empty(x.shape, dtype=x.dtype, pin_memory=True) for x in outs]
            for x, h in zip(outs, serial_host):
                h.copy_(x, non_blocking=True)
            return sum(x.numel() * x.element_size() for x in outs)

        def timed(fn):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            if pg is not None:
                pg.barrier()
            torch.cuda.synchronize()
            e0.record()
            r = fn()
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            if pg is not None:
                t = torch.tensor([ms], device=dev)
                pg.all_reduce(t, op=pg.ReduceOp.MAX)
                ms = float(t.item())
            return ms, r

        # each pipelined form is timed over K steps three times (the two forms alternating) and the
        # median is reported: the host link and the host's threads are shared with other jobs, and
        # one stall of the copy engines or of the calling thread moves a single short run
        for _ in range(args.warmup):
            serial_step()
        serial_ms, _ = timed(lambda: [serial_step() for _ in range(K)][-1])
        ops_runs, auto_runs, d2h = [], [], 0
        for rep in range(3):
            compute_fn[0] = compute_ops
            run_pipelined(args.warmup)
            ms, d2h = timed(lambda: run_pipelined(K))
            ops_runs.append(ms)
            compute_fn[0] = compute_autograd
            run_pipelined(args.warmup)
            ms, _ = timed(lambda: run_pipelined(K))
            auto_runs.append(ms)
        e2e_ms, e2e_auto_ms = float(np.median(ops_runs)), float(np.median(auto_runs))

        def copies_only(n):
            # the same uploads and downloads with no compute, each direction on its own stream: the
            # host link's bound for the pipelined steps
            start, e_up, e_down = torch.cuda.Event(), torch.cuda.Event(), torch.cuda.Event()
            start.record(main)
            s_up.wait_event(start)
            s_down.wait_event(start)
            for i in range(n):
                with torch.cuda.stream(s_up):
                    dev_blocks[i % 2].copy_(host_block, non_blocking=True)
                with torch.cuda.stream(s_down):
                    out_host.copy_(stage[i % 2], non_blocking=True)
            e_up.record(s_up)
            e_down.record(s_down)
            main.wait_event(e_up)
            main.wait_event(e_down)

        copies_only(args.warmup)
        copy_ms, _ = timed(lambda: copies_only(K))
        e2e = {"value": world * P * HW / (e2e_ms / K * 1e-3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_ms / K,
               "serial_ms_per_step": serial_ms / K,
               "runs_ms_per_step": [round(x / K, 4) for x in ops_runs],
               "copies_only_ms_per_step": copy_ms / K,
               "l2": "not flushed between steps: every step's inputs arrive afresh over the host link",
               "api": "the reference-facing operators bruteforce_specularvisibility_shader_forward2 and "
                      "_backward2 (every step uploads all of its inputs from one pinned host block and "
                      "downloads every output into pinned host memory; step i+1's upload and step i's "
                      "download overlap compute on two copy streams)",
               "autograd": {"value": world * P * HW / (e2e_auto_ms / K * 1e-3), "ms_per_step": e2e_auto_ms / K,
                            "runs_ms_per_step": [round(x / K, 4) for x in auto_runs],
                            "api": "the same pipeline through diff_envshade_b200.shade + "
                                   "torch.autograd.backward"}}

    # ---- roofline of the dominant kernel (fused adjoint) and of the forward kernel
    peaks = measured_peaks()
    if "sm_max_mhz" in peaks:
        sm_max, clock_src = float(peaks["sm_max_mhz"]), "sm_max_mhz of MEASURED_PEAKS.json"
    elif clocks and clocks.get("sm_max_mhz"):
        sm_max, clock_src = float(clocks["sm_max_mhz"]), "NVML max SM clock; MEASURED_PEAKS.json absent"
    else:
        sm_max, clock_src = 1965.0, "nominal B200 max SM clock; no measured clock"
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    peak_tinst = sms * FP32_LANES_PER_SM * sm_max * 1e6 / 1e12
    bwd_avg = float(np.mean(bwd_ms)) * 1e-3
    fwd_avg = float(np.mean(fwd_ms)) * 1e-3
    ach_bwd = P * HW * INSTR_BWD_VIS / bwd_avg / 1e12
    ach_fwd = P * HW * INSTR_FWD_VIS / fwd_avg / 1e12
    roofline = {
        "bound": "fp32", "kernel": "des_bwd_kernel<diffuse,specular,visibility> (fused adjoint)",
        "achieved": ach_bwd, "peak": peak_tinst, "unit": "T FP32-pipe instr/s", "frac": ach_bwd / peak_tinst,
        "traffic": committed_traffic(),
        "peak_source": f"derived: {sms} SMs x {FP32_LANES_PER_SM} FP32 lanes x {sm_max:.0f} MHz "
                       f"({clock_src}; no measured FP32 peak exists)",
        "work": f"{INSTR_BWD_VIS} FP32-pipe instr per point*texel pair x {P}x{HW} pairs per launch",
        "kernel_ms": bwd_avg * 1e3,
        "forward": {"kernel_ms": fwd_avg * 1e3, "achieved": ach_fwd, "frac": ach_fwd / peak_tinst,
                    "work": f"{INSTR_FWD_VIS} instr/pair"},
    }

    relight = mesh = None
    if rank == 0 and world == 1:
        mesh = mesh_layout_step(des, wl, dev, flush)
        if not args.no_relight:
            relight = relight_leg(des, wl, dev, flush, peak_tinst)

    serving = None
    if rank == 0 and world == 1 and not args.no_serve:
        # served p50/p99 against serial plain launches on one arrival schedule (2000 requests, Poisson 5k/s)
        from diff_envshade_b200 import serve_workload
        serving = serve_workload.run(n=2000, rate=5000.0, tick_us=50)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, desc, threads = cpu_port_throughput(inp_host, target_s=10.0)
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": desc}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": args.warmup,
            "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded normals/views/materials, lognormal env, Bernoulli(0.7) bits)",
            "config": bench_config(P, d.envmap.shape[1], d.envmap.shape[2], d.visibility.shape[0] * 32, world),
            "gpu_launches": launches,
            "timing": f"CUDA-graph replays of the two operator calls ({launches_per_step} kernels per step, as "
                      f"launched eagerly); eagerly launched, the same step took {eager_ms / K:.4f} ms "
                      f"({eager_launches} launches in {K} steps)",
            "eager_ms_per_step": eager_ms / K,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "clocks": clocks,
            "serving": serving,
            "relight": relight,
            "mesh_layout": mesh,
            "fwd_ms": float(np.mean(fwd_ms)), "bwd_ms": float(np.mean(bwd_ms)),
        }
        print(json.dumps(line))
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
