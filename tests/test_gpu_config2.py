"""The large workload at full size: 1,048,576 points, 32x64 env map (exp(N(0,1.5)) radiance),
2048-bit visibility (64 slots, Bernoulli(0.6)), roughness U[0.05, 1].

The FP64 oracle cannot integrate all 2.1G point*texel pairs inside a test, so the full-size run is
checked through what does not depend on size:

* per-point outputs of 4096 random points against the FP64 oracle on the same texel table (a
  point's outputs depend on that point alone): the suite's forward and gradient bounds
  (conftest.py: forward per element 1e-5 relative; gradients 1e-4 of the tensor scale);
* the point gradients of 256 random points against central finite differences of the FP64 oracle
  forward of L = <g_shading, shading> + <g_diffuse, diffuse_shading>.  The step is h = 1e-4, scaled
  down by min(1, r^4 / 0.01) for normal, view and roughness: the GGX lobe is r^4 wide in n.h, so
  at r = 0.05 a 1e-4 step would jump across it.  The function has kinks (max(n.l, 0)) that finite
  differences straddle, so the bound is looser than the analytic check: per gradient tensor
  max|d| <= 1e-3 max|FD| (oracle against FD on these distributions: 2e-4 on g_normal, below 1e-6
  elsewhere);
* the env-map gradient, a sum over every point, through the adjoint identity: the shading is linear
  in the env map, so <g_s, shading> + <g_d, diffuse_shading> = <g_envmap, envmap> exactly.  With
  positive upstream gradients (no cancellation) both sides, summed in FP64 from the FP32 outputs,
  must agree to 1e-5 relative; dropping one 32-point tile would move the right side by ~3e-5;
* a repeated call is bit-identical, env-map gradient included.
"""
import copy

import numpy as np
import pytest
import torch

from conftest import assert_close_fwd, assert_close_grad

pytestmark = pytest.mark.gpu

FD_H = 1e-4
FD_TOL = 1e-3
ADJ_TOL = 1e-5
GRADS = ("g_normal", "g_view", "g_albedo", "g_spec", "g_rough", "g_env")


@pytest.fixture(scope="module")
def big():
    assert torch.cuda.is_available()
    import diff_envshade_b200 as des
    from diff_envshade_b200 import workloads as wl
    inp = wl.make_config("vis-1m")
    d = inp.to("cuda")
    vis = (d.face_vertex_list, d.nearest_triangle_id, d.barycentric_coord, d.visibility)
    base = (d.normal, d.view_dir, d.albedo, d.specular_albedo, d.roughness, d.envmap, d.light2obj_rotmat)
    sh, wh = des.bruteforce_specularvisibility_shader_forward2(*base, *vis, True)
    g = des.bruteforce_specularvisibility_shader_backward2(d.grad_shading, d.grad_diffuse_shading, *base, *vis, True)
    table = des.texel_table(32, 64, d.light2obj_rotmat).cpu().numpy()
    out = {"shading": sh.cpu(), "diffuse_shading": wh.cpu()}
    for k, t in zip(GRADS, g):
        out[k] = t.cpu()
    return des, inp, d, base, vis, table, out


def test_full_size_points_against_fp64_oracle(big):
    from oracle import oracle as orc
    des, inp, d, base, vis, table, out = big
    pts = np.sort(np.random.default_rng(11).choice(inp.P, 4096, replace=False))
    flags = orc.flags_for("specularvisibility2", True, True)
    sh, wh = orc.forward(inp, flags, table=table, points=pts)
    ref = orc.backward(inp, flags, inp.grad_shading, inp.grad_diffuse_shading, table=table, points=pts)
    assert_close_fwd(out["shading"][pts], sh, "1m:shading")
    assert_close_fwd(out["diffuse_shading"][pts], wh, "1m:diffuse_shading")
    for k in GRADS[:5]:
        assert_close_grad(out[k][pts], ref[k], f"1m:{k}")


def test_full_size_gradients_against_finite_differences(big):
    from oracle import oracle as orc
    des, inp, d, base, vis, table, out = big
    n = 256
    pts = np.sort(np.random.default_rng(12).choice(inp.P, n, replace=False))
    flags = orc.flags_for("specularvisibility2", True, True)
    cols = {k: getattr(inp, k).numpy().astype(np.float64)[pts]
            for k in ("normal", "view_dir", "albedo", "specular_albedo", "roughness")}
    lobe = FD_H * np.minimum(1.0, cols["roughness"][:, 0] ** 4 / 0.01)
    steps = {"normal": lobe, "view_dir": lobe, "roughness": lobe, "albedo": np.full(n, FD_H),
             "specular_albedo": np.full(n, FD_H)}
    plan = [(k, c, s) for k, m in (("normal", 3), ("view_dir", 3), ("albedo", 3), ("specular_albedo", 3),
                                   ("roughness", 1)) for c in range(m) for s in (1.0, -1.0)]
    # one oracle call over len(plan) perturbed copies of the n points
    pert = copy.copy(inp)
    for k, v in cols.items():
        setattr(pert, k, np.concatenate([v] * len(plan)))
    for i, (k, c, s) in enumerate(plan):
        getattr(pert, k)[i * n:(i + 1) * n, c] += s * steps[k]
    pert.nearest_triangle_id = np.concatenate([inp.nearest_triangle_id.numpy()[pts]] * len(plan))
    pert.barycentric_coord = np.concatenate([inp.barycentric_coord.numpy()[:, pts]] * len(plan), axis=1)
    sh, wh = orc.forward(pert, flags, table=table)
    gs = np.tile(inp.grad_shading.numpy().astype(np.float64)[pts], (len(plan), 1))
    gw = np.tile(inp.grad_diffuse_shading.numpy().astype(np.float64)[pts], (len(plan), 1))
    L = (sh * gs).sum(1) + (wh * gw).sum(1)
    names = {"normal": "g_normal", "view_dir": "g_view", "albedo": "g_albedo", "specular_albedo": "g_spec",
             "roughness": "g_rough"}
    fd = {g: np.zeros((n, 1 if g == "g_rough" else 3)) for g in names.values()}
    for i in range(0, len(plan), 2):
        k, c, _ = plan[i]
        fd[names[k]][:, c] = (L[i * n:(i + 1) * n] - L[(i + 1) * n:(i + 2) * n]) / (2 * steps[k])
    for g, f in fd.items():
        got = out[g][pts].numpy().astype(np.float64)
        err = np.abs(got - f).max() / np.abs(f).max()
        assert err <= FD_TOL, f"{g}: max|gpu - FD| / max|FD| = {err:.3e}"


def test_full_size_env_gradient_adjoint_identity(big):
    des, inp, d, base, vis, table, out = big
    g = torch.Generator().manual_seed(13)
    gs = (0.5 + 0.5 * torch.rand(inp.P, 3, generator=g)).cuda()
    gw = (0.5 + 0.5 * torch.rand(inp.P, 3, generator=g)).cuda()
    g_env = des.bruteforce_specularvisibility_shader_backward2(gs, gw, *base, *vis, True)[5]
    sh = out["shading"].cuda().double()
    wh = out["diffuse_shading"].cuda().double()
    lhs = float((gs.double() * sh).sum() + (gw.double() * wh).sum())
    rhs = float((g_env.double() * d.envmap.double()).sum())
    assert lhs > 0
    assert abs(lhs - rhs) <= ADJ_TOL * lhs, f"adjoint identity: {lhs!r} vs {rhs!r} ({abs(lhs - rhs) / lhs:.3e})"


def test_full_size_deterministic(big):
    """A second identical 1M-point call gives bit-identical outputs, env-map gradient included
    (fixed-order FP64 reduction; the normal-direction ordering is a stable sort)."""
    des, inp, d, base, vis, table, out = big
    sh, wh = des.bruteforce_specularvisibility_shader_forward2(*base, *vis, True)
    g = des.bruteforce_specularvisibility_shader_backward2(d.grad_shading, d.grad_diffuse_shading, *base, *vis, True)
    assert torch.equal(sh.cpu(), out["shading"]) and torch.equal(wh.cpu(), out["diffuse_shading"])
    for k, t in zip(GRADS, g):
        assert torch.equal(t.cpu(), out[k]), k
