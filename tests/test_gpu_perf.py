"""Speed of the CUDA path against the reference extension's own kernels on the same B200.

Both sides shade the same seeded inputs; forward + backward are timed with CUDA events after
warm-up (median of 20 runs; a 256 MiB buffer is rewritten between runs so neither side starts
from a warm L2).  The bar for the 70,000-point, 16x32, 512-bit-visibility workload and for the
1,048,576-point, 32x64, 2048-bit-visibility workload is at least 3x the reference's fwd+bwd time.  Set DES_PERF_OUT=<file> to also write the numbers as
JSON.
"""
import json
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _time(fn, flush, reps=20, warm=3):
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    ts = []
    for i in range(reps):
        flush.fill_(float(i))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    return float(np.median(ts))


def _ops(mod, d, vis):
    v = (d.face_vertex_list, d.nearest_triangle_id, d.barycentric_coord, d.visibility) if vis else ()
    base = (d.normal, d.view_dir, d.albedo, d.specular_albedo, d.roughness, d.envmap, d.light2obj_rotmat)
    if vis:
        fwd = lambda: mod.bruteforce_specularvisibility_shader_forward2(*base, *v, True)  # noqa: E731
        bwd = lambda: mod.bruteforce_specularvisibility_shader_backward2(  # noqa: E731
            d.grad_shading, d.grad_diffuse_shading, *base, *v, True)
    else:
        fwd = lambda: mod.bruteforce_specular_shader_forward2(*base, True)  # noqa: E731
        bwd = lambda: mod.bruteforce_specular_shader_backward2(d.grad_shading, d.grad_diffuse_shading, *base,  # noqa
                                                               True)
    return fwd, bwd


@pytest.mark.parametrize("name,vis,min_speedup", [("vis-70k", True, 3.0), ("plain-4k", False, 1.0),
                                                    ("vis-1m", True, 3.0)])
def test_faster_than_reference_kernels(reference_ext, name, vis, min_speedup):
    import diff_envshade_b200 as des
    from diff_envshade_b200 import workloads as wl
    d = wl.make_config(name).to("cuda")
    flush = torch.empty(64 * 1024 * 1024, device="cuda")
    res = {}
    for tag, mod in (("reference", reference_ext), ("b200", des)):
        fwd, bwd = _ops(mod, d, vis)
        res[tag] = {"fwd_ms": _time(fwd, flush), "bwd_ms": _time(bwd, flush),
                    "fwd_bwd_ms": _time(lambda: (fwd(), bwd()), flush)}
    pairs = d.P * d.HW
    for r in res.values():
        r["point_texel_per_s"] = pairs / (r["fwd_bwd_ms"] * 1e-3)
    speedup = res["reference"]["fwd_bwd_ms"] / res["b200"]["fwd_bwd_ms"]
    summary = {"workload": name, "points": d.P, "texels": d.HW, "speedup_fwd_bwd": speedup, **res}
    print(json.dumps(summary))
    out = os.environ.get("DES_PERF_OUT")
    if out:
        with open(out, "a") as f:
            f.write(json.dumps(summary) + "\n")
    assert speedup >= min_speedup, summary
