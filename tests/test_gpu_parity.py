"""GPU parity of the CUDA shading path against the reference extension and the FP64 oracle.

Tolerances (see conftest.py): forward per element rel 1e-5; gradients rel 1e-4 of the
tensor scale; the texel table and the visibility bits are compared bit-for-bit.
"""
import ctypes
import os

import numpy as np
import pytest
import torch

from conftest import assert_close_fwd, assert_close_grad, golden_files
import cabi

pytestmark = pytest.mark.gpu

GRAD_KEYS = ("g_normal", "g_view", "g_albedo", "g_spec", "g_rough", "g_env")


@pytest.fixture(scope="module")
def des():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import diff_envshade_b200
    return diff_envshade_b200


def _dev(inp):
    return inp.to("cuda")


def run_op(mod, op, d, ed=True, es=True):
    """Run operator family `op` of module `mod` (this package or the reference) on device inputs."""
    n, v, a, s, r, env, R = (d.normal, d.view_dir, d.albedo, d.specular_albedo, d.roughness, d.envmap,
                             d.light2obj_rotmat)
    gs, gw = d.grad_shading, d.grad_diffuse_shading
    out = {}
    if op == "specularvisibility2":
        vis = (d.face_vertex_list, d.nearest_triangle_id, d.barycentric_coord, d.visibility)
        out["shading"], out["diffuse_shading"] = mod.bruteforce_specularvisibility_shader_forward2(
            n, v, a, s, r, env, R, *vis, es)
        g = mod.bruteforce_specularvisibility_shader_backward2(gs, gw, n, v, a, s, r, env, R, *vis, es)
    elif op == "specular2":
        out["shading"], out["diffuse_shading"] = mod.bruteforce_specular_shader_forward2(n, v, a, s, r, env, R, es)
        g = mod.bruteforce_specular_shader_backward2(gs, gw, n, v, a, s, r, env, R, es)
    elif op == "specular":
        out["shading"] = mod.bruteforce_specular_shader_forward(n, v, a, s, r, env, R, ed, es)
        g = mod.bruteforce_specular_shader_backward(gs, n, v, a, s, r, env, R, ed, es)
    elif op == "specular_clamp":
        out["shading"] = mod.bruteforce_specular_shader_clamp_forward(n, v, a, s, r, env, R, ed, es)
        g = mod.bruteforce_specular_shader_clamp_backward(gs, n, v, a, s, r, env, R, ed, es)
    elif op == "diffuse":
        out["shading"] = mod.bruteforce_diffuse_shader_forward(n, a, env, R)
        gn, ga, ge = mod.bruteforce_diffuse_shader_backward(gs, n, a, env, R)
        g = [gn, None, ga, None, None, ge]
    else:
        raise ValueError(op)
    for k, t in zip(GRAD_KEYS, g):
        if t is not None:
            out[k] = t
    torch.cuda.synchronize()
    return {k: t.detach().cpu() for k, t in out.items()}


def check_outputs(got, ref, tag, allowance=None):
    allowance = allowance or {}
    for k in ("shading", "diffuse_shading"):
        if k in ref:
            assert_close_fwd(got[k], ref[k], f"{tag}:{k}", allowance=allowance.get(k))
    for k in GRAD_KEYS:
        if k in ref:
            assert_close_grad(got[k], ref[k], f"{tag}:{k}", allowance=allowance.get(k))


def oracle_outputs(op, inp, ed, es, table):
    """FP64 oracle outputs (same texel table) for operator family `op`."""
    from oracle import oracle as orc
    flags = orc.flags_for(op, ed, es)
    sh, wh = orc.forward(inp, flags, table=table)
    gw = inp.grad_diffuse_shading if flags & orc.WHITE else None
    out = orc.backward(inp, flags, inp.grad_shading, gw, table=table)
    out["shading"], out["diffuse_shading"] = sh, wh
    return out


def check_against_reference(got, ref, exact, tag):
    """Ours vs exact (FP64 oracle) at the stated tolerance, and ours vs the reference with the
    reference's own per-element deviation from exact arithmetic as an allowance."""
    check_outputs(got, {k: exact[k] for k in ref}, f"{tag}:vs-fp64")
    allowance = {k: np.abs(np.asarray(ref[k], dtype=np.float64) - exact[k]) for k in ref}
    check_outputs(got, ref, f"{tag}:vs-reference", allowance)


# ------------------------------------------------------------------------------------------------
# texel table: bit-exact with the reference's per-pair getLightDir / getDeltaOmega / rotation
# ------------------------------------------------------------------------------------------------

PROBES = golden_files("table_probe_*.npz")


def _probe_predictions(table):
    """fl(fl(+-l_axis / pi) * d_omega) per (texel, axis) where the cosine is positive, else 0."""
    pi = np.float32(3.141592653589793)
    pred = np.zeros((table.shape[0], 6), dtype=np.float32)
    for k, (axis, sign) in enumerate([(0, 1), (0, -1), (1, 1), (1, -1), (2, 1), (2, -1)]):
        cos = (np.float32(sign) * table[:, axis]).astype(np.float32)
        pred[:, k] = np.where(cos > 0, (cos / pi).astype(np.float32) * table[:, 3], np.float32(0))
    return pred


def _bits_equal(a, b):
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = np.ascontiguousarray(b, dtype=np.float32)
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.skipif(not PROBES, reason="table probe fixtures not generated")
@pytest.mark.parametrize("path", PROBES, ids=[os.path.basename(p)[12:-4] for p in PROBES])
def test_texel_table_bit_exact_with_reference(des, path):
    """The rotated texel table equals, bit for bit, the direction and solid angle every reference
    kernel family evaluates per pair: each probe output below reduces to fl(fl(+-l_k/pi) * d_omega)
    for one texel (see tests/golden/make_golden.py)."""
    z = np.load(path)
    H, W = (int(x) for x in os.path.basename(path)[12:-4].split("_")[0].split("x"))
    HW = H * W
    table = des.texel_table(H, W, torch.from_numpy(z["R"]).float().cuda()).cpu().numpy()
    assert _bits_equal(table, z["table"])
    pred = _probe_predictions(table)
    assert (pred > 0).sum() >= 3 * HW
    assert _bits_equal(pred.reshape(-1), z["ref_white"]), "Forward2 (visibility)"
    assert _bits_equal(pred.reshape(-1), z["ref_galbedo"]), "Backward2 (visibility)"
    assert _bits_equal(pred.T, z["ref_genv"]), "BackwardEnvmap2 (visibility)"
    if "ref_white_novis" in z:
        assert _bits_equal(pred, z["ref_white_novis"]), "Forward2 (no visibility)"
    # this kernel accumulates with a fused multiply-add: acc = fma(fl(cos/pi), d_omega, acc)
    from fractions import Fraction
    pi = np.float32(3.141592653589793)
    acc = [np.float32(0)] * HW
    for t in range(HW):
        a = np.float32(0)
        for k, (axis, sign) in enumerate([(0, 1), (0, -1), (1, 1), (1, -1), (2, 1), (2, -1)]):
            cos = np.float32(np.float32(sign) * table[t, axis])
            if cos > 0:
                q = np.float32(cos / pi)
                a = _round_f32(Fraction(float(q)) * Fraction(float(table[t, 3])) + Fraction(float(a)))
        acc[t] = a
    assert _bits_equal(np.array(acc, dtype=np.float32), z["ref_genv_novis"]), "BackwardEnvmap2 (no visibility)"


def _round_f32(fr):
    """Correctly rounded (nearest, ties to even) float32 of a Fraction."""
    from fractions import Fraction
    f = np.float32(float(fr))
    cands = [f, np.nextafter(f, np.float32(np.inf)), np.nextafter(f, np.float32(-np.inf))]
    return min(cands, key=lambda c: (abs(Fraction(float(c)) - fr), int(np.float32(c).view(np.uint32)) & 1))


# ------------------------------------------------------------------------------------------------
# golden fixtures made by the reference extension
# ------------------------------------------------------------------------------------------------

CASES = golden_files("[!t]*.npz")


def _inputs_from_fixture(z):
    from diff_envshade_b200 import workloads as wl
    t = {k[3:]: torch.from_numpy(z[k]) for k in z.files if k.startswith("in_")}
    inp = wl.ShadeInputs(t["normal"], t["view_dir"], t["albedo"], t["specular_albedo"], t["roughness"],
                         t["envmap"], t["light2obj_rotmat"], t.get("face_vertex_list"), t.get("nearest_triangle_id"),
                         t.get("barycentric_coord"), t.get("visibility"), t["grad_shading"],
                         t["grad_diffuse_shading"])
    return inp


@pytest.mark.skipif(not CASES, reason="golden fixtures not generated")
@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(p)[:-4] for p in CASES])
def test_against_reference_golden(des, path):
    z = np.load(path)
    op, P, H, W, seed, layout, ed, es = z["meta"]
    host = _inputs_from_fixture(z)
    ed, es = bool(int(ed)), bool(int(es))
    got = run_op(des, op, _dev(host), ed, es)
    ref = {k[4:]: z[k] for k in z.files if k.startswith("ref_")}
    exact = oracle_outputs(op, host, ed, es, z["table"])
    check_against_reference(got, ref, exact, os.path.basename(path))


# ------------------------------------------------------------------------------------------------
# live comparisons (reference extension on this GPU, FP64 oracle)
# ------------------------------------------------------------------------------------------------

LIVE = [
    ("plain-4k", "specular2", None),
    ("vis-70k", "specularvisibility2", "identity"),
    ("vis-70k-mesh", "specularvisibility2", "mesh"),
]


@pytest.mark.parametrize("name,op,layout", LIVE)
def test_against_reference_live(des, reference_ext, name, op, layout):
    """Config sizes: 4096 points (no visibility) and 70,000 points x 16x32 with 512 visibility
    bits, forward + backward, on the same inputs through both extensions."""
    from diff_envshade_b200 import workloads as wl
    base = name.replace("-mesh", "")
    c = wl.CONFIGS[base]
    inp = wl.make_inputs(c["P"], c["H"], c["W"], c["seed"], sigma=c["sigma"], rough=c["rough"], vis_p=c["vis_p"],
                         vis_layout=layout or "identity", rotation=True)
    d = _dev(inp)
    got = run_op(des, op, d)
    ref = run_op(reference_ext, op, d)
    table = des.texel_table(c["H"], c["W"], d.light2obj_rotmat).cpu().numpy()
    exact = oracle_outputs(op, inp, True, True, table)
    _record_parity(name, got, ref, exact)
    check_against_reference(got, ref, exact, name)


def _raw_stats(a, b):
    """(max|a - b| / max|b|, max over elements of |a - b| / |b|) with no allowance and no floor
    (elements where both are exactly zero count as equal)."""
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    d = np.abs(a - b)
    scale = np.abs(b).max()
    with np.errstate(divide="ignore", invalid="ignore"):
        rel = np.where(d == 0, 0.0, d / np.abs(b))
    return float(d.max() / scale) if scale > 0 else float(d.max()), float(rel.max())


def _record_parity(name, got, ref, exact):
    """The literal comparison against the reference (no allowance) per output, beside the same
    statistics of the reference and of this build against the FP64 oracle.  Printed, and appended
    as JSON to $DES_PERF_OUT when set."""
    import json
    rows = {}
    for k in ref:
        t_or, e_or = _raw_stats(got[k], ref[k])
        t_rx, e_rx = _raw_stats(ref[k], exact[k])
        t_ox, e_ox = _raw_stats(got[k], exact[k])
        rows[k] = {"ours_vs_ref": [t_or, e_or], "ref_vs_fp64": [t_rx, e_rx], "ours_vs_fp64": [t_ox, e_ox]}
    line = {"parity_case": name, "stats": "[max|d|/max|ref|, max elementwise |d|/|ref|]", "outputs": rows}
    print(json.dumps(line))
    if os.environ.get("DES_PERF_OUT"):
        with open(os.environ["DES_PERF_OUT"], "a") as f:
            f.write(json.dumps(line) + "\n")


@pytest.mark.parametrize("op,ed,es,layout", [
    ("specularvisibility2", True, True, "mesh"),
    ("specularvisibility2", True, False, "mesh"),
    ("specular2", True, True, None),
    ("specular", True, True, None),
    ("specular", False, True, None),
    ("specular_clamp", True, True, None),
    ("diffuse", True, False, None),
])
def test_against_fp64_oracle(des, op, ed, es, layout):
    """Same texel table, FP64 arithmetic in the oracle: this isolates the kernels' FP32 error,
    including the FP64-reduced env-map gradient."""
    from oracle import oracle as orc
    from diff_envshade_b200 import workloads as wl
    inp = wl.make_inputs(3000, 16, 32, seed=77, vis_p=0.7 if layout else None, vis_layout=layout or "identity",
                         rotation=True)
    d = _dev(inp)
    got = run_op(des, op, d, ed, es)
    table = des.texel_table(16, 32, d.light2obj_rotmat).cpu().numpy()
    flags = orc.flags_for(op, ed, es)
    sh, wh = orc.forward(inp, flags, table=table)
    gw = inp.grad_diffuse_shading.numpy() if flags & orc.WHITE else None
    ref = orc.backward(inp, flags, inp.grad_shading.numpy(), gw, table=table)
    ref["shading"] = sh
    if "diffuse_shading" in got:
        ref["diffuse_shading"] = wh
    ref = {k: v for k, v in ref.items() if k in got}
    check_outputs(got, ref, f"{op}-oracle")


def test_deterministic(des):
    from diff_envshade_b200 import workloads as wl
    d = _dev(wl.make_config("vis-70k"))
    a = run_op(des, "specularvisibility2", d)
    b = run_op(des, "specularvisibility2", d)
    for k in a:
        assert torch.equal(a[k], b[k]), k


def test_cabi_direct_matches_torch_ops(des):
    """The C ABI called through ctypes with raw device pointers gives the torch-op results."""
    from diff_envshade_b200 import workloads as wl
    d = _dev(wl.make_inputs(1000, 16, 32, seed=5, vis_p=0.7, vis_layout="mesh", rotation=True))
    want = run_op(des, "specularvisibility2", d)
    L = cabi.lib()
    args = cabi.make_args(d)
    flags = cabi.DES_DIFFUSE | cabi.DES_SPECULAR
    wsb = L.des_shade_workspace_bytes(args.P, args.H, args.W, flags, 1, torch.cuda.current_device())
    ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    sh = torch.empty(1000, 3, device="cuda")
    wh = torch.empty(1000, 3, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.des_shade_forward(ctypes.byref(args), flags, cabi.ptr(sh), cabi.ptr(wh), cabi.ptr(ws), wsb,
                               stream) == cabi.DES_OK
    outs = [torch.empty(1000, 3, device="cuda") for _ in range(4)] + [torch.empty(1000, 1, device="cuda"),
                                                                       torch.empty(3, 16, 32, device="cuda")]
    assert L.des_shade_backward(ctypes.byref(args), flags, cabi.ptr(d.grad_shading), cabi.ptr(d.grad_diffuse_shading),
                                *[cabi.ptr(o) for o in outs], cabi.ptr(ws), wsb, stream) == cabi.DES_OK
    torch.cuda.synchronize()
    assert torch.equal(sh.cpu(), want["shading"]) and torch.equal(wh.cpu(), want["diffuse_shading"])
    for k, o in zip(GRAD_KEYS, outs):
        assert torch.equal(o.cpu(), want[k]), k
    st = ctypes.c_int(-1)
    assert L.des_workspace_status(cabi.ptr(ws), wsb, ctypes.byref(st), stream) == cabi.DES_OK
    assert st.value == cabi.DES_OK


@pytest.mark.parametrize("P,layout", [(70000, "identity"), (40000, "mesh"), (16384, None), (300001, "identity")])
def test_point_ordering_changes_no_result(des, P, layout):
    """Calls with P >= 16384 shade the points ordered by normal direction and skip texels below all
    32 lanes' horizons; DES_INPUT_ORDER turns that off.  (300,001 points: 4096-point ranking chunks
    of several passes and a ragged last chunk.)  Per-point outputs must be bit-identical
    (each point's arithmetic is the same and a skipped texel adds exact zeros); the env-map
    gradient differs only in FP64 summation order (gradient bound of conftest.py)."""
    from diff_envshade_b200 import workloads as wl
    inp = wl.make_inputs(P, 16, 32, seed=P + 3, vis_p=0.7 if layout else None, vis_layout=layout or "identity",
                         rotation=True)
    d = _dev(inp)
    L = cabi.lib()
    args = cabi.make_args(d)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    dev = torch.cuda.current_device()
    res = {}
    for order in (0, cabi.DES_INPUT_ORDER, cabi.DES_COMPACT):
        flags = cabi.DES_DIFFUSE | cabi.DES_SPECULAR | order
        wsf = L.des_shade_workspace_bytes(args.P, args.H, args.W, flags, 0, dev)
        wsb = L.des_shade_workspace_bytes(args.P, args.H, args.W, flags, 1, dev)
        ws = torch.empty(max(wsf, wsb), dtype=torch.uint8, device="cuda")
        sh, wh = torch.empty(P, 3, device="cuda"), torch.empty(P, 3, device="cuda")
        assert L.des_shade_forward(ctypes.byref(args), flags, cabi.ptr(sh), cabi.ptr(wh), cabi.ptr(ws), wsf,
                                   stream) == cabi.DES_OK
        outs = [torch.empty(P, 3, device="cuda") for _ in range(4)] + [torch.empty(P, 1, device="cuda"),
                                                                        torch.empty(3, 16, 32, device="cuda")]
        assert L.des_shade_backward(ctypes.byref(args), flags, cabi.ptr(d.grad_shading),
                                    cabi.ptr(d.grad_diffuse_shading), *[cabi.ptr(o) for o in outs], cabi.ptr(ws),
                                    wsb, stream) == cabi.DES_OK
        res[order] = [sh, wh] + outs
    both = cabi.DES_DIFFUSE | cabi.DES_SPECULAR
    assert L.des_shade_workspace_bytes(args.P, args.H, args.W, both, 1, dev) > \
        L.des_shade_workspace_bytes(args.P, args.H, args.W, both | cabi.DES_INPUT_ORDER, 1, dev)
    assert L.des_shade_workspace_bytes(args.P, args.H, args.W, both | cabi.DES_COMPACT, 1, dev) <= \
        L.des_shade_workspace_bytes(args.P, args.H, args.W, both | cabi.DES_INPUT_ORDER, 1, dev)
    torch.cuda.synchronize()
    for other in (cabi.DES_INPUT_ORDER, cabi.DES_COMPACT):
        for name, a, b in zip(("shading", "diffuse_shading") + GRAD_KEYS, res[0], res[other]):
            if name == "g_env" or (other == cabi.DES_COMPACT and name.startswith("g_")):
                # compact: the adjoint splits each point's texel sum over a different number of warps
                assert_close_grad(a.cpu(), b.cpu(), f"plan {other}:{name}")
            else:
                assert torch.equal(a, b), f"default plan and plan {other} differ in {name}"


def test_backward_reuses_its_forwards_ordering(des):
    """The torch ops keep one workspace per device: a backward that follows its forward on the same
    normals, env map and rotation skips the ordering and texel-table kernels (2 launches instead of
    4); modifying the normals (their version counter) makes the next call order the points again, and
    a backward after a backward rebuilds the table."""
    from diff_envshade_b200 import workloads as wl
    d = _dev(wl.make_inputs(70000, 16, 32, seed=91, vis_p=0.7, rotation=True))
    base = (d.normal, d.view_dir, d.albedo, d.specular_albedo, d.roughness, d.envmap, d.light2obj_rotmat)
    vis = (d.face_vertex_list, d.nearest_triangle_id, d.barycentric_coord, d.visibility)
    gs, gw = d.grad_shading, d.grad_diffuse_shading
    n0 = des.kernel_launches()
    des.bruteforce_specularvisibility_shader_forward2(*base, *vis, True)
    n1 = des.kernel_launches()
    g = des.bruteforce_specularvisibility_shader_backward2(gs, gw, *base, *vis, True)
    n2 = des.kernel_launches()
    assert n1 - n0 == 3 and n2 - n1 == 2, (n1 - n0, n2 - n1)  # fwd: prep, place, shade; bwd: shade, reduce
    torch.autograd.graph.increment_version(d.normal)
    g2 = des.bruteforce_specularvisibility_shader_backward2(gs, gw, *base, *vis, True)
    n3 = des.kernel_launches()
    assert n3 - n2 == 4  # ordered again: prep, place, shade, reduce
    for a, b in zip(g[:5], g2[:5]):
        assert torch.equal(a, b)
    assert_close_grad(g[5].cpu(), g2[5].cpu(), "reuse:g_env")


def test_stale_ordering_changes_no_result(des):
    """DES_REUSE_ORDER with an ordering computed for other normals (same P): per-point outputs are
    bit-identical to a fresh call, the env-map gradient within the gradient bound."""
    from diff_envshade_b200 import workloads as wl
    P = 50000
    A = _dev(wl.make_inputs(P, 16, 32, seed=92, vis_p=0.7))
    B = _dev(wl.make_inputs(P, 16, 32, seed=93, vis_p=0.7))
    L = cabi.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    flags = cabi.DES_DIFFUSE | cabi.DES_SPECULAR
    dev = torch.cuda.current_device()
    argsA, argsB = cabi.make_args(A), cabi.make_args(B)
    wsb = max(L.des_shade_workspace_bytes(P, 16, 32, flags, k, dev) for k in (0, 1))
    ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    shA = torch.empty(P, 3, device="cuda")
    assert L.des_shade_forward(ctypes.byref(argsA), flags, cabi.ptr(shA), None, cabi.ptr(ws), wsb, stream) == 0

    def backward(extra, wsx):
        outs = [torch.empty(P, 3, device="cuda") for _ in range(4)] + [torch.empty(P, 1, device="cuda"),
                                                                        torch.empty(3, 16, 32, device="cuda")]
        st = L.des_shade_backward(ctypes.byref(argsB), flags | extra, cabi.ptr(B.grad_shading),
                                  cabi.ptr(B.grad_diffuse_shading), *[cabi.ptr(o) for o in outs], cabi.ptr(wsx), wsb,
                                  stream)
        assert st == 0
        return outs

    stale = backward(cabi.DES_REUSE_ORDER, ws)  # ordering of A's normals applied to B
    fresh = backward(0, torch.empty(wsb, dtype=torch.uint8, device="cuda"))
    torch.cuda.synchronize()
    for a, b in zip(stale[:5], fresh[:5]):
        assert torch.equal(a, b)
    assert_close_grad(stale[5].cpu(), fresh[5].cpu(), "stale:g_env")


@pytest.mark.parametrize("P", [1000, 20000], ids=["input-order", "ordered"])
def test_adjoint_reusing_forward_table(des, P):
    """An adjoint that reuses the texel table (and ordering) its forward left in the workspace
    (DES_REUSE_TABLE | DES_REUSE_ORDER) gives the outputs of an adjoint computed from scratch: per-point
    gradients bit for bit, the env-map gradient within the gradient bound."""
    from diff_envshade_b200 import workloads as wl
    d = _dev(wl.make_inputs(P, 16, 32, seed=91, vis_p=0.7, vis_layout="mesh", rotation=True))
    L = cabi.lib()
    flags = cabi.DES_DIFFUSE | cabi.DES_SPECULAR
    args = cabi.make_args(d)
    dev = torch.cuda.current_device()
    wsb = max(L.des_shade_workspace_bytes(P, 16, 32, flags, 0, dev), L.des_shade_workspace_bytes(P, 16, 32, flags, 1, dev))
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def adjoint(ws, f):
        outs = [torch.empty(P, 3, device="cuda") for _ in range(4)] + [torch.empty(P, 1, device="cuda"),
                                                                        torch.empty(3, 16, 32, device="cuda")]
        st = L.des_shade_backward(ctypes.byref(args), f, cabi.ptr(d.grad_shading), cabi.ptr(d.grad_diffuse_shading),
                                  *[cabi.ptr(o) for o in outs], cabi.ptr(ws), wsb, stream)
        assert st == cabi.DES_OK
        return outs

    ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    sh, wh = torch.empty(P, 3, device="cuda"), torch.empty(P, 3, device="cuda")
    assert L.des_shade_forward(ctypes.byref(args), flags, cabi.ptr(sh), cabi.ptr(wh), cabi.ptr(ws), wsb,
                               stream) == cabi.DES_OK
    reused = adjoint(ws, flags | cabi.DES_REUSE_ORDER | cabi.DES_REUSE_TABLE)
    fresh = adjoint(torch.zeros(wsb, dtype=torch.uint8, device="cuda"), flags)
    torch.cuda.synchronize()
    for name, a, b in zip(GRAD_KEYS[:5], reused, fresh):
        assert torch.equal(a, b), name
    assert_close_grad(reused[5].cpu(), fresh[5].cpu(), "g_env")
