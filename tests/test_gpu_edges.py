"""Edge cases of the shading operators on the GPU, against the FP64 oracle at the suite's
tolerances (conftest.py):

* ragged sizes: 1 point, 33 points (one full tile and one lane), 97 points;
* degenerate geometry in one batch: views along the normal, grazing views (n.v = 0.01), views
  below the surface (n.v < 0; the clamp variant shades those points to zero), normals along the
  coordinate axes, roughness at 0.05 and 1.0, zero diffuse or specular albedo;
* no points at all: empty outputs and a zero env-map gradient.
"""
import numpy as np
import pytest
import torch

from conftest import assert_close_grad
from test_gpu_parity import check_outputs, oracle_outputs, run_op

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def des():
    assert torch.cuda.is_available()
    import diff_envshade_b200
    return diff_envshade_b200


def _unit(x):
    return x / x.norm(dim=-1, keepdim=True)


def edge_inputs(P=97, seed=123, vis=True):
    from diff_envshade_b200 import workloads as wl
    inp = wl.make_inputs(P, 16, 32, seed=seed, vis_p=0.7 if vis else None, vis_layout="mesh", rotation=True)
    g = torch.Generator().manual_seed(seed + 1)
    n, v = inp.normal.clone(), inp.view_dir.clone()
    r, a, s = inp.roughness.clone(), inp.albedo.clone(), inp.specular_albedo.clone()
    m = min(P, 8)
    v[:m] = n[:m]                                                   # view along the normal
    if P > 16:
        t = _unit(torch.linalg.cross(n[8:16], torch.randn(8, 3, generator=g), dim=1))
        v[8:16] = _unit(t + 0.01 * n[8:16])                         # grazing: n.v ~ 0.01
    if P > 22:
        axes = torch.tensor([[1., 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]])
        n[16:22] = axes                                             # normals along the axes
        v[16:22] = _unit(axes + 0.5 * _unit(torch.randn(6, 3, generator=g)))
    if P > 32:
        r[24:28] = 0.05                                             # roughness extremes
        r[28:32] = 1.0
    if P > 36:
        a[32:34] = 0.0                                              # no diffuse / no specular
        s[34:36] = 0.0
    if P > 40:
        v[36:40] = -v[36:40]                                        # view below the surface
    inp.normal, inp.view_dir = n.contiguous(), v.contiguous()
    inp.roughness, inp.albedo, inp.specular_albedo = r.contiguous(), a.contiguous(), s.contiguous()
    return inp


@pytest.mark.parametrize("P", [1, 33, 97])
@pytest.mark.parametrize("op,layout", [("specularvisibility2", "mesh"), ("specular2", None),
                                       ("specular_clamp", None), ("diffuse", None)])
def test_edge_inputs_against_fp64_oracle(des, P, op, layout):
    inp = edge_inputs(P, vis=layout is not None)
    d = inp.to("cuda")
    ed, es = True, op != "diffuse"
    got = run_op(des, op, d, ed, es)
    table = des.texel_table(16, 32, d.light2obj_rotmat).cpu().numpy()
    ref = oracle_outputs(op, inp, ed, es, table)
    ref = {k: v for k, v in ref.items() if k in got}
    check_outputs(got, ref, f"{op}-P{P}")
    if op == "specular_clamp" and P > 40:
        sh = got["shading"].cpu().numpy()
        below = (inp.normal[36:40] * inp.view_dir[36:40]).sum(-1).numpy() <= 0
        assert np.all(sh[36:40][below] == 0.0), "points viewed from below shade to zero with the clamp"


def test_no_points(des):
    """P = 0: empty shading, empty point gradients and an all-zero env-map gradient."""
    inp = edge_inputs(97)
    d = inp.to("cuda")
    e = {k: getattr(d, k)[:0] for k in ("normal", "view_dir", "albedo", "specular_albedo", "roughness",
                                        "grad_shading", "grad_diffuse_shading", "nearest_triangle_id")}
    bary = d.barycentric_coord[:, :0].contiguous()
    vis = (d.face_vertex_list, e["nearest_triangle_id"], bary, d.visibility)
    base = (e["normal"], e["view_dir"], e["albedo"], e["specular_albedo"], e["roughness"], d.envmap,
            d.light2obj_rotmat)
    sh, wh = des.bruteforce_specularvisibility_shader_forward2(*base, *vis, True)
    assert sh.shape == (0, 3) and wh.shape == (0, 3)
    g = des.bruteforce_specularvisibility_shader_backward2(e["grad_shading"], e["grad_diffuse_shading"], *base, *vis,
                                                           True)
    for t in g[:5]:
        assert t.shape[0] == 0
    assert g[5].shape == d.envmap.shape
    assert_close_grad(g[5].cpu(), torch.zeros(d.envmap.shape), "empty:g_envmap")
    torch.cuda.synchronize()


@pytest.mark.parametrize("P", [1000, 20000], ids=["input-order", "ordered"])
def test_single_vertex_path_matches_three_word_path(des, P):
    """A warp whose points each use one visibility row (triangle (p, p, p), barycentrics (1, 0, 0))
    takes the one-word visibility path.  Giving point 0 a genuine three-vertex triangle with the same
    barycentrics (1, 0, 0) keeps every visibility value the same but sends its warp down the general
    three-word path: every output must stay the same bit for bit."""
    from diff_envshade_b200 import workloads as wl
    inp = wl.make_inputs(P, 16, 32, seed=77, vis_p=0.7, vis_layout="identity", rotation=True)
    d = inp.to("cuda")
    alt = inp.to("cuda")
    extra = torch.tensor([[0], [1], [2]], dtype=torch.int32, device="cuda")
    alt.face_vertex_list = torch.cat([d.face_vertex_list, extra], dim=1).contiguous()
    tri = d.nearest_triangle_id.clone()
    tri[0] = P  # the appended face (0, 1, 2)
    alt.nearest_triangle_id = tri
    got = run_op(des, "specularvisibility2", d)
    ref = run_op(des, "specularvisibility2", alt)
    for k in got:
        assert torch.equal(got[k], ref[k]), k
