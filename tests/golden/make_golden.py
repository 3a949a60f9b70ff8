"""Generate the golden fixtures of the shading path from the reference extension.

Runs on a CUDA machine with the reference extension built by ``oracle/build_ref.py``
(``oracle/_ref/_diff_envshade*.so``) and this package built.  For each case it draws seeded
inputs, runs the reference operator, and stores inputs + reference outputs in
``<out>/<case>.npz``; the texel table this package computes (``texel_table``) is stored
beside them so the CPU oracle can be checked against the reference without a GPU.

It also writes ``table_probe_<H>x<W>.npz``: the reference's white-diffuse output for points
that each see exactly one texel through a one-hot visibility word, with axis-aligned normals
and unit radiance.  That output equals fl(fl(+-l_k / pi) * d_omega) for the texel's rotated
direction component l_k, which pins the texel table bit-for-bit.

With ``--only-etc`` it writes only ``etc_*.npz``: the reference's mesh-side helpers
(get_uv_of_triangle forward/backward, get_nearest_mesh_points forward), extract_bitfield,
sample_envmap and blur_envmap on seeded inputs (the shading fixtures above are left as they are).

Usage:  python tests/golden/make_golden.py --out tests/golden [--only-etc]
"""
import argparse
import glob
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)


def load_reference():
    refdir = os.path.join(ROOT, "oracle", "_ref")
    if not glob.glob(os.path.join(refdir, "_diff_envshade*.so")):
        raise SystemExit("reference extension not built (python oracle/build_ref.py)")
    sys.path.insert(0, refdir)
    import _diff_envshade  # noqa: E402
    return _diff_envshade


# case name -> (op, P, H, W, seed, vis layout or None, enable_diffuse, enable_specular, rotation, rough range)
CASES = {
    "vis2_mesh_16x32": ("specularvisibility2", 256, 16, 32, 11, "mesh", True, True, True, (0.2, 0.9)),
    "vis2_identity_16x32": ("specularvisibility2", 256, 16, 32, 12, "identity", True, True, False, (0.2, 0.9)),
    "vis2_mesh_ragged_5x7_nospec": ("specularvisibility2", 200, 5, 7, 13, "mesh", True, False, True, (0.2, 0.9)),
    "vis2_mesh_32x64_rough": ("specularvisibility2", 128, 32, 64, 14, "mesh", True, True, True, (0.05, 1.0)),
    "spec2_16x32": ("specular2", 256, 16, 32, 21, None, True, True, True, (0.2, 0.9)),
    "spec2_16x32_nospec": ("specular2", 256, 16, 32, 22, None, True, False, False, (0.2, 0.9)),
    "spec2_ragged_9x13": ("specular2", 100, 9, 13, 23, None, True, True, True, (0.2, 0.9)),
    "spec_v1_16x32": ("specular", 256, 16, 32, 31, None, True, True, True, (0.2, 0.9)),
    "spec_v1_specular_only": ("specular", 256, 16, 32, 32, None, False, True, False, (0.2, 0.9)),
    "spec_v1_diffuse_only": ("specular", 256, 16, 32, 33, None, True, False, True, (0.2, 0.9)),
    "clamp_16x32": ("specular_clamp", 256, 16, 32, 41, None, True, True, True, (0.2, 0.9)),
    "clamp_16x32_diffuse_only": ("specular_clamp", 256, 16, 32, 42, None, True, False, False, (0.2, 0.9)),
    "diffuse_16x32": ("diffuse", 256, 16, 32, 51, None, True, False, True, (0.2, 0.9)),
}


def run_reference(ref, op, inp, ed, es):
    d = {k: v.cuda() for k, v in inp.tensors().items()}
    n, v, a, s, r, env, R = (d["normal"], d["view_dir"], d["albedo"], d["specular_albedo"], d["roughness"],
                             d["envmap"], d["light2obj_rotmat"])
    gs, gw = d["grad_shading"], d["grad_diffuse_shading"]
    out = {}
    if op == "specularvisibility2":
        vis = (d["face_vertex_list"], d["nearest_triangle_id"], d["barycentric_coord"], d["visibility"])
        sh, wh = ref.bruteforce_specularvisibility_shader_forward2(n, v, a, s, r, env, R, *vis, es)
        g = ref.bruteforce_specularvisibility_shader_backward2(gs, gw, n, v, a, s, r, env, R, *vis, es)
        out.update(shading=sh, diffuse_shading=wh)
    elif op == "specular2":
        sh, wh = ref.bruteforce_specular_shader_forward2(n, v, a, s, r, env, R, es)
        g = ref.bruteforce_specular_shader_backward2(gs, gw, n, v, a, s, r, env, R, es)
        out.update(shading=sh, diffuse_shading=wh)
    elif op == "specular":
        sh = ref.bruteforce_specular_shader_forward(n, v, a, s, r, env, R, ed, es)
        g = ref.bruteforce_specular_shader_backward(gs, n, v, a, s, r, env, R, ed, es)
        out.update(shading=sh)
    elif op == "specular_clamp":
        sh = ref.bruteforce_specular_shader_clamp_forward(n, v, a, s, r, env, R, ed, es)
        g = ref.bruteforce_specular_shader_clamp_backward(gs, n, v, a, s, r, env, R, ed, es)
        out.update(shading=sh)
    elif op == "diffuse":
        sh = ref.bruteforce_diffuse_shader_forward(n, a, env, R)
        gn, ga, ge = ref.bruteforce_diffuse_shader_backward(gs, n, a, env, R)
        g = [gn, None, ga, None, None, ge]
        out.update(shading=sh)
    else:
        raise ValueError(op)
    names = ["g_normal", "g_view", "g_albedo", "g_spec", "g_rough", "g_env"]
    for k, t in zip(names, g):
        if t is not None:
            out[k] = t
    torch.cuda.synchronize()
    return {k: t.detach().cpu().numpy() for k, t in out.items()}


def table_probe_inputs(H, W, R):
    """P = 6*H*W points: point (t, k) has normal +-e_axis, one-hot visibility on texel t."""
    HW = H * W
    axes = torch.tensor([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], dtype=torch.float32)
    P = 6 * HW
    normal = axes.repeat(HW, 1).contiguous()                    # point index = t*6 + k
    texel = torch.arange(HW).repeat_interleave(6)
    nslots = (HW + 31) // 32
    w = np.zeros((nslots, P), dtype=np.uint32)
    t = texel.numpy()
    w[t // 32, np.arange(P)] = (np.uint32(1) << (t % 32).astype(np.uint32))
    words = torch.from_numpy(w.view(np.int32))
    return dict(
        normal=normal, view_dir=normal.clone(), albedo=torch.ones(P, 3), specular_albedo=torch.zeros(P, 3),
        roughness=torch.full((P, 1), 0.5), envmap=torch.ones(3, H, W), light2obj_rotmat=R.float().contiguous(),
        face_vertex_list=torch.arange(P, dtype=torch.int32).repeat(3, 1).contiguous(),
        nearest_triangle_id=torch.arange(P, dtype=torch.int64),
        barycentric_coord=torch.cat([torch.ones(1, P), torch.zeros(2, P)]).contiguous(),
        visibility=words.contiguous())


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden"))
    ap.add_argument("--only-etc", action="store_true", help="write only the etc_*.npz helper fixtures")
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    ref = load_reference()
    import diff_envshade_b200 as des
    from diff_envshade_b200 import workloads as wl

    write_etc_fixtures(ref, a.out)
    if a.only_etc:
        return

    for name, (op, P, H, W, seed, layout, ed, es, rot, rough) in CASES.items():
        inp = wl.make_inputs(P, H, W, seed, rough=rough, vis_p=(0.7 if layout else None),
                             vis_layout=(layout or "identity"), rotation=rot)
        outs = run_reference(ref, op, inp, ed, es)
        table = des.texel_table(H, W, inp.light2obj_rotmat.cuda()).cpu().numpy()
        arrays = {f"in_{k}": v.numpy() for k, v in inp.tensors().items()}
        arrays.update({f"ref_{k}": v for k, v in outs.items()})
        arrays["table"] = table
        meta = np.array([op, str(P), str(H), str(W), str(seed), str(layout), str(int(ed)), str(int(es))])
        np.savez_compressed(os.path.join(a.out, f"{name}.npz"), meta=meta, **arrays)
        print("wrote", name, {k: v.shape for k, v in outs.items()})

    g = torch.Generator().manual_seed(99)
    for (H, W, rot) in [(16, 32, False), (32, 64, False), (7, 9, True), (16, 32, True)]:
        R = wl.random_rotation(g) if rot else torch.eye(3)
        tag = f"{H}x{W}" + ("_rot" if rot else "")
        arrays = table_probes(ref, H, W, R, one_hot_env=(H * W <= 512))
        arrays["table"] = des.texel_table(H, W, R.float().cuda()).cpu().numpy()
        arrays["R"] = R.numpy()
        np.savez_compressed(os.path.join(a.out, f"table_probe_{tag}.npz"), **arrays)
        print("wrote table probe", tag, sorted(arrays))


def table_probes(ref, H, W, R, one_hot_env):
    """Reference outputs that each reduce to fl(fl(+-l_axis / pi) * d_omega) for single texels.

    ref_white        Forward2 with visibility: point (t, axis) sees only texel t       [6*HW]
    ref_galbedo      Backward2 with visibility, grad_shading = 1: its g_albedo          [6*HW]
    ref_genv         BackwardEnvmap2 with visibility, one axis per call, grad_diffuse = 1 [6, HW]
    ref_white_novis  Forward2 without visibility, one-hot env map per call (small maps) [HW, 6]
    ref_genv_novis   BackwardEnvmap2 without visibility, 6 axis points, grad_diffuse = 1 [HW]
                     (the sum over the positive-cosine points, in point order)
    """
    HW = H * W
    out = {}
    d = {k: v.cuda() for k, v in table_probe_inputs(H, W, R).items()}
    vis = (d["face_vertex_list"], d["nearest_triangle_id"], d["barycentric_coord"], d["visibility"])
    base = (d["normal"], d["view_dir"], d["albedo"], d["specular_albedo"], d["roughness"], d["envmap"],
            d["light2obj_rotmat"])
    _, white = ref.bruteforce_specularvisibility_shader_forward2(*base, *vis, False)
    out["ref_white"] = white[:, 0].cpu().numpy()
    ones = torch.ones_like(d["normal"])
    g = ref.bruteforce_specularvisibility_shader_backward2(ones, torch.zeros_like(ones), *base, *vis, False)
    out["ref_galbedo"] = g[2][:, 0].cpu().numpy()
    genv = []
    for k in range(6):
        sel = torch.arange(k, 6 * HW, 6, device="cuda")  # point t*6+k: texel t, axis k
        sub = {n: d[n][sel].contiguous() for n in ("normal", "view_dir", "albedo", "specular_albedo", "roughness")}
        P = HW
        faces = torch.arange(P, dtype=torch.int32, device="cuda").repeat(3, 1).contiguous()
        tri = torch.arange(P, dtype=torch.int64, device="cuda")
        bary = torch.cat([torch.ones(1, P), torch.zeros(2, P)]).cuda().contiguous()
        bits = d["visibility"][:, sel].contiguous()
        zeros = torch.zeros(P, 3, device="cuda")
        gk = ref.bruteforce_specularvisibility_shader_backward2(
            zeros, torch.ones(P, 3, device="cuda"), sub["normal"], sub["view_dir"], sub["albedo"],
            sub["specular_albedo"], sub["roughness"], d["envmap"], d["light2obj_rotmat"], faces, tri, bary, bits,
            False)
        genv.append(gk[5][0].reshape(-1).cpu().numpy())
    out["ref_genv"] = np.stack(genv)
    # no-visibility kernels: 6 axis points
    n6 = d["normal"][:6].contiguous()
    a6 = torch.ones(6, 3, device="cuda")
    z6 = torch.zeros(6, 3, device="cuda")
    r6 = torch.full((6, 1), 0.5, device="cuda")
    g6 = ref.bruteforce_specular_shader_backward2(z6, torch.ones(6, 3, device="cuda"), n6, n6, a6, z6, r6,
                                                  d["envmap"], d["light2obj_rotmat"], False)
    out["ref_genv_novis"] = g6[5][0].reshape(-1).cpu().numpy()
    if one_hot_env:
        wn = np.zeros((HW, 6), dtype=np.float32)
        for t in range(HW):
            env = torch.zeros(3, H, W, device="cuda")
            env.view(3, -1)[:, t] = 1.0
            _, w = ref.bruteforce_specular_shader_forward2(n6, n6, a6, z6, r6, env, d["light2obj_rotmat"], False)
            wn[t] = w[:, 0].cpu().numpy()
        out["ref_white_novis"] = wn
    torch.cuda.synchronize()
    return out



def write_etc_fixtures(ref, out_dir):
    """Reference outputs of the mesh-side and env-map helpers (etc.cu) on seeded inputs."""
    from diff_envshade_b200 import workloads as wl
    g = torch.Generator().manual_seed(2024)
    # get_uv_of_triangle: random triangles, queries around them (interior, edge and vertex regions)
    P = 1024
    tri = torch.randn(P, 3, 3, generator=g)
    w = torch.rand(P, 3, generator=g) * 1.6 - 0.3
    q = (w[:, :, None] * tri).sum(1) + 0.2 * torch.randn(P, 3, generator=g)
    gb = torch.randn(P, 3, generator=g)
    bary = ref.get_uv_of_triangle_forward(tri.cuda(), q.cuda())
    gq = ref.get_uv_of_triangle_backward(tri.cuda(), q.cuda(), gb.cuda())
    np.savez_compressed(os.path.join(out_dir, "etc_uv_of_triangle.npz"), triangles=tri.numpy(), query_pos=q.numpy(),
                        grad_barycentric_coord=gb.numpy(), ref_barycentric_coord=bary.cpu().numpy(),
                        ref_grad_query_pos=gq.cpu().numpy())
    # get_nearest_mesh_points forward on a jittered sphere (the reference backward reads its own
    # output buffer as the incoming gradient, so only the forward is a usable fixture)
    pos, faces = wl.make_sphere_mesh(16, 32, seed=7)
    head, lst = wl.vertex_adjacency(faces, pos.shape[1])
    qp, idx = wl.make_mesh_queries(pos, 2048, 4, seed=8)
    # the reference kernel traps (ends the CUDA context) when a query has no candidate face or more
    # than 128 distinct ones: check on the CPU that every query has 1..128 before running it
    n, end = head[0].numpy(), head[1].numpy()
    cand = [len({f for v in row for f in lst.numpy()[end[v] - n[v]:end[v]]}) for row in idx.numpy()]
    assert 1 <= min(cand) and max(cand) <= 128, (min(cand), max(cand))
    tri_id, nb = ref.get_nearest_mesh_points_forward(head.cuda(), lst.cuda(), faces.cuda(), pos.cuda(), qp.cuda(),
                                                     idx.cuda())
    np.savez_compressed(os.path.join(out_dir, "etc_nearest_mesh_points.npz"), adjacency_head=head.numpy(),
                        adjacency_list=lst.numpy(), face_vertex_list=faces.numpy(), vertex_pos=pos.numpy(),
                        query_pos=qp.numpy(), idxs=idx.numpy(), ref_nearest_triangle_id=tri_id.cpu().numpy(),
                        ref_barycentric_coord=nb.cpu().numpy())
    # extract_bitfield: ragged bit count, a window of points
    words = torch.randint(-2 ** 31, 2 ** 31 - 1, (16, 300), generator=g, dtype=torch.int64).to(torch.int32)
    bits = ref.extract_bitfield_forward(words.cuda(), 500, 17, 250)
    np.savez_compressed(os.path.join(out_dir, "etc_extract_bitfield.npz"), bitfield=words.numpy(),
                        meta=np.array([500, 17, 250]), ref_out=bits.cpu().numpy())
    # sample_envmap: random directions (not normalised) on a lognormal 3 x 16 x 32 map
    env = torch.exp(torch.randn(3, 16, 32, generator=g))
    dirs = torch.randn(3, 2048, generator=g) * torch.rand(1, 2048, generator=g).add(0.5)
    smp = ref.sample_envmap_forward(dirs.cuda(), env.cuda())
    # blur_envmap: 3 x 16 x 32 -> 8 x 16, 64 samples, alpha 0.3; and 4 channels -> 4 x 8
    blur = ref.blur_envmap_forward(env.cuda(), 8, 16, 64, 0.3)
    env4 = torch.exp(torch.randn(4, 8, 16, generator=g))
    blur4 = ref.blur_envmap_forward(env4.cuda(), 4, 8, 16, 0.7)
    np.savez_compressed(os.path.join(out_dir, "etc_envmap_sampling.npz"), envmap=env.numpy(), query_point=dirs.numpy(),
                        ref_sample=smp.cpu().numpy(), ref_blur=blur.cpu().numpy(), blur_args=np.array([8, 16, 64]),
                        blur_alpha=np.array([0.3], dtype=np.float32), envmap4=env4.numpy(),
                        ref_blur4=blur4.cpu().numpy(), blur4_args=np.array([4, 8, 16]),
                        blur4_alpha=np.array([0.7], dtype=np.float32))
    torch.cuda.synchronize()
    print("wrote etc fixtures")


if __name__ == "__main__":
    main()
