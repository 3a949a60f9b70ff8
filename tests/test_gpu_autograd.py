"""The torch.autograd.Function wrappers (the drop-in a caller of the reference writes around its
operators) against the FP64 oracle, through ``shade()`` and through each Function.

Cases: both outputs in the loss; only ``shading`` in the loss (the white-diffuse output receives no
gradient, so its incoming gradient is None and counts as zero); ``enable_specular=False``; a
non-identity light rotation; the v1 and clamp families with one term switched off; and
``create_graph=True``, which must raise when the gradient is differentiated again (the backward
operators are native kernels that autograd cannot trace).

Tolerances (conftest.py): forward per element |d| <= 1e-5 (|ref| + 1e-3 max|ref|); gradients per
tensor max|d| <= 1e-4 max|ref| and per element |d| <= 1e-4 (|ref| + 0.1 max|ref|).
"""
import numpy as np
import pytest
import torch

from conftest import assert_close_fwd, assert_close_grad

pytestmark = pytest.mark.gpu

LEAVES = ("normal", "view_dir", "albedo", "specular_albedo", "roughness", "envmap")
GRAD_KEY = {"normal": "g_normal", "view_dir": "g_view", "albedo": "g_albedo", "specular_albedo": "g_spec",
            "roughness": "g_rough", "envmap": "g_env"}


@pytest.fixture(scope="module")
def des():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import diff_envshade_b200
    return diff_envshade_b200


def _leaves(d, names=LEAVES):
    return {k: getattr(d, k).detach().clone().requires_grad_(True) for k in names}


def _oracle(inp, op, ed, es, g_white, table):
    from oracle import oracle as orc
    flags = orc.flags_for(op, ed, es)
    sh, wh = orc.forward(inp, flags, table=table)
    out = orc.backward(inp, flags, inp.grad_shading, g_white, table=table)
    out["shading"], out["diffuse_shading"] = sh, wh
    return out


def _check_grads(x, ref, names, tag):
    for k in names:
        assert x[k].grad is not None, f"{tag}: no gradient for {k}"
        assert_close_grad(x[k].grad.cpu(), ref[GRAD_KEY[k]].reshape(x[k].shape), f"{tag}:{k}")


@pytest.mark.parametrize("vis", [True, False], ids=["visibility", "plain"])
@pytest.mark.parametrize("use_white", [True, False], ids=["both-outputs", "shading-only"])
@pytest.mark.parametrize("enable_specular", [True, False], ids=["specular", "no-specular"])
def test_shade_against_fp64_oracle(des, vis, use_white, enable_specular):
    from diff_envshade_b200 import workloads as wl
    inp = wl.make_inputs(3000, 16, 32, seed=41 + 2 * vis + use_white, vis_p=0.7 if vis else None,
                         vis_layout="mesh", rotation=True)
    d = inp.to("cuda")
    x = _leaves(d)
    sh, wh = des.shade(x["normal"], x["view_dir"], x["albedo"], x["specular_albedo"], x["roughness"], x["envmap"],
                       d.light2obj_rotmat, visibility=d.vis_tuple() if vis else None,
                       enable_specular=enable_specular)
    if use_white:
        torch.autograd.backward([sh, wh], [d.grad_shading, d.grad_diffuse_shading])
    else:
        torch.autograd.backward([sh], [d.grad_shading])  # wh gets no gradient: None -> zeros
    torch.cuda.synchronize()
    table = des.texel_table(16, 32, d.light2obj_rotmat).cpu().numpy()
    op = "specularvisibility2" if vis else "specular2"
    g_white = inp.grad_diffuse_shading if use_white else np.zeros((inp.P, 3))
    ref = _oracle(inp, op, True, enable_specular, g_white, table)
    tag = f"shade[vis={vis},white={use_white},spec={enable_specular}]"
    assert_close_fwd(sh.detach().cpu(), ref["shading"], f"{tag}:shading")
    assert_close_fwd(wh.detach().cpu(), ref["diffuse_shading"], f"{tag}:diffuse_shading")
    names = LEAVES if enable_specular else ("normal", "albedo", "envmap")
    _check_grads(x, ref, names, tag)
    if not enable_specular:  # terms switched off receive zeros, as the reference's backward allocates
        for k in ("view_dir", "specular_albedo", "roughness"):
            assert x[k].grad is not None and float(x[k].grad.abs().max()) == 0.0, k


@pytest.mark.parametrize("fn,op,ed,es", [
    ("SpecularShade", "specular", True, True),
    ("SpecularShade", "specular", False, True),
    ("SpecularShade", "specular", True, False),
    ("SpecularShadeClamp", "specular_clamp", True, True),
    ("DiffuseShade", "diffuse", True, False),
])
def test_v1_functions_against_fp64_oracle(des, fn, op, ed, es):
    from diff_envshade_b200 import workloads as wl
    inp = wl.make_inputs(2000, 8, 16, seed=61, rotation=True)
    d = inp.to("cuda")
    if fn == "DiffuseShade":
        x = _leaves(d, ("normal", "albedo", "envmap"))
        sh = des.DiffuseShade.apply(x["normal"], x["albedo"], x["envmap"], d.light2obj_rotmat)
        names = ("normal", "albedo", "envmap")
    else:
        x = _leaves(d)
        sh = getattr(des, fn).apply(x["normal"], x["view_dir"], x["albedo"], x["specular_albedo"], x["roughness"],
                                    x["envmap"], d.light2obj_rotmat, ed, es)
        names = tuple(k for k in LEAVES if (es or k not in ("view_dir", "specular_albedo", "roughness"))
                      and (ed or k != "albedo"))
    torch.autograd.backward([sh], [d.grad_shading])
    torch.cuda.synchronize()
    table = des.texel_table(8, 16, d.light2obj_rotmat).cpu().numpy()
    ref = _oracle(inp, op, ed, es, None, table)
    assert_close_fwd(sh.detach().cpu(), ref["shading"], f"{fn}:shading")
    _check_grads(x, ref, names, fn)


def test_functions_apply_directly_match_shade(des):
    """SpecularVisibilityShade2.apply and SpecularShade2.apply give the same tensors as shade()."""
    from diff_envshade_b200 import workloads as wl
    d = wl.make_inputs(1500, 16, 32, seed=71, vis_p=0.6, vis_layout="mesh", rotation=True).to("cuda")
    for vis in (True, False):
        a, b = _leaves(d), _leaves(d)
        s1, w1 = des.shade(*[a[k] for k in LEAVES], d.light2obj_rotmat, visibility=d.vis_tuple() if vis else None)
        if vis:
            s2, w2 = des.SpecularVisibilityShade2.apply(*[b[k] for k in LEAVES], d.light2obj_rotmat, *d.vis_tuple(),
                                                        True)
        else:
            s2, w2 = des.SpecularShade2.apply(*[b[k] for k in LEAVES], d.light2obj_rotmat, True)
        torch.autograd.backward([s1, w1], [d.grad_shading, d.grad_diffuse_shading])
        torch.autograd.backward([s2, w2], [d.grad_shading, d.grad_diffuse_shading])
        assert torch.equal(s1, s2) and torch.equal(w1, w2)
        for k in LEAVES:
            assert torch.equal(a[k].grad, b[k].grad), k


def test_double_backward_raises(des):
    """A second derivative through the native backward must raise, not return zeros."""
    from diff_envshade_b200 import workloads as wl
    d = wl.make_inputs(256, 8, 16, seed=81, vis_p=0.7, vis_layout="mesh").to("cuda")
    x = _leaves(d)
    sh, wh = des.shade(*[x[k] for k in LEAVES], d.light2obj_rotmat, visibility=d.vis_tuple())
    # the incoming gradient 2*sh depends on the leaves, so the first-order gradient is itself part
    # of the graph -- differentiating it again must fail loudly
    (g,) = torch.autograd.grad((sh * sh).sum(), [x["normal"]], create_graph=True)
    assert g.requires_grad
    with pytest.raises(RuntimeError, match="once_differentiable"):
        (g.sum() + x["normal"].sum()).backward()
