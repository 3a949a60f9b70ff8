"""Multi-env-map relighting on tcgen05 (relight_multienv) against the FP64 oracle and against K runs
of the plain FP32 forward kernel.

Tolerance: BF16 hi+lo split mode -- per element |d| <= 1e-3 (|ref| + 1e-3 max|ref|) against the FP64
oracle (the accuracy bound set for the BF16 form); plain BF16 mode -- the same check at 2e-2, with its
measured error printed.  Set DES_PERF_OUT=<file> to append the measured errors and timings as JSON.
"""
import json
import os

import numpy as np
import pytest
import torch

from conftest import assert_close_fwd

pytestmark = pytest.mark.gpu


def _oracle_multi(inp, envs, vis, table, points=None):
    from oracle import oracle as orc
    flags = orc.flags_for("specularvisibility2" if vis else "specular2")
    outs = []
    for k in range(envs.shape[0]):
        inp.envmap = envs[k]
        sh, _ = orc.forward(inp, flags, table=table, points=points)
        outs.append(sh)
    return np.stack(outs, axis=1)  # [P, K, 3]


def _rel_err(got, ref):
    g, r = np.asarray(got, np.float64), np.asarray(ref, np.float64)
    scale = np.abs(r).max()
    return float((np.abs(g - r) / (np.abs(r) + 1e-3 * scale)).max())


def _relight(des, d, envs, vis, split):
    v = (d.face_vertex_list, d.nearest_triangle_id, d.barycentric_coord, d.visibility) if vis else (None,) * 4
    out = des.relight_multienv(d.normal, d.view_dir, d.albedo, d.specular_albedo, d.roughness, envs,
                               d.light2obj_rotmat, *v, True, split)
    torch.cuda.synchronize()
    return out


@pytest.mark.parametrize("P,H,W,K,vis,split", [
    (1000, 16, 32, 16, True, True),
    (777, 16, 32, 70, True, True),     # two passes (64 + 6 env maps), ragged point count
    (513, 8, 16, 24, False, True),
    (1000, 16, 32, 16, True, False),   # plain BF16
    (1, 16, 32, 1, True, True),        # one point, one env map
    (300, 32, 64, 8, True, True),      # the largest map the kernel takes (2048 texels)
    (129, 16, 16, 3, False, False),    # 256 texels, ragged points, plain BF16
])
def test_relight_against_fp64_oracle(P, H, W, K, vis, split):
    import diff_envshade_b200 as des
    from diff_envshade_b200 import workloads as wl
    inp = wl.make_inputs(P, H, W, seed=300 + K, vis_p=0.7 if vis else None, vis_layout="mesh", rotation=True)
    g = torch.Generator().manual_seed(900 + K)
    envs = torch.exp(torch.randn(K, 3, H, W, generator=g))
    d = inp.to("cuda")
    out = _relight(des, d, envs.cuda(), vis, split).cpu().numpy()
    table = des.texel_table(H, W, d.light2obj_rotmat).cpu().numpy()
    ref = _oracle_multi(inp, envs.numpy(), vis, table)
    err = _rel_err(out, ref)
    print(json.dumps({"relight_vs_fp64": err, "P": P, "K": K, "HW": H * W, "vis": vis, "split": split}))
    assert_close_fwd(out, ref, "relight", rtol=1e-3 if split else 2e-2)


def test_relight_matches_plain_path_at_config_size():
    """262,144 points x 64 env maps x 16x32 with visibility (the multi-env workload): every output
    against 64 runs of the plain FP32 forward kernel, a 256-point subset against the FP64 oracle,
    and the time of the fused pass against the 64 plain passes."""
    import diff_envshade_b200 as des
    from diff_envshade_b200 import workloads as wl
    c = wl.CONFIGS["multienv-262k"]
    inp = wl.make_inputs(c["P"], c["H"], c["W"], c["seed"], sigma=c["sigma"], rough=c["rough"], vis_p=c["vis_p"],
                         env_count=c["K"])
    envs = inp.envmap.cuda()
    d = inp.to("cuda")
    vis = (d.face_vertex_list, d.nearest_triangle_id, d.barycentric_coord, d.visibility)
    base = (d.normal, d.view_dir, d.albedo, d.specular_albedo, d.roughness)

    def fused():
        return des.relight_multienv(*base, envs, d.light2obj_rotmat, *vis, True, True)

    def plain():
        return torch.stack([des.bruteforce_specularvisibility_shader_forward2(
            *base, envs[k], d.light2obj_rotmat, *vis, True)[0] for k in range(envs.shape[0])], dim=1)

    out = fused()
    ref = plain()
    torch.cuda.synchronize()
    assert_close_fwd(out.cpu(), ref.cpu(), "fused-vs-plain", rtol=1e-3)
    # FP64 oracle on a subset
    pts = np.random.default_rng(0).choice(c["P"], 256, replace=False)
    table = des.texel_table(c["H"], c["W"], d.light2obj_rotmat).cpu().numpy()
    host = wl.make_inputs(c["P"], c["H"], c["W"], c["seed"], sigma=c["sigma"], rough=c["rough"], vis_p=c["vis_p"],
                          env_count=c["K"])
    exact = _oracle_multi(host, host.envmap.numpy(), True, table, points=pts)
    err64 = _rel_err(out.cpu().numpy()[pts], exact)
    assert_close_fwd(out.cpu().numpy()[pts], exact, "fused-vs-fp64", rtol=1e-3)

    def timeit(fn, reps=5):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
        return float(np.median(ts))

    t_fused, t_plain = timeit(fused), timeit(plain, reps=3)
    summary = {"workload": "multienv-262k", "fused_ms": t_fused, "plain_64x_ms": t_plain,
               "speedup": t_plain / t_fused, "max_rel_err_vs_fp64_subset": err64,
               "max_rel_err_vs_plain": _rel_err(out.cpu().numpy(), ref.cpu().numpy())}
    print(json.dumps(summary))
    if os.environ.get("DES_PERF_OUT"):
        with open(os.environ["DES_PERF_OUT"], "a") as f:
            f.write(json.dumps(summary) + "\n")
    assert t_plain / t_fused >= 5.0, summary
