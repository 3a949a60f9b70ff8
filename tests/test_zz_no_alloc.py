"""des_shade_backward_noalloc: the fused adjoint for callers that cannot allocate device memory.

Some callers (a real-time renderer's frame loop, a host framework that owns every device byte)
cannot hand this library a workspace.  The no-allocation entry point keeps its scratch in a static
device array instead.  These tests call it through the C ABI and check it against the regular entry
point (des_shade_backward with a caller-provided workspace) on two calls in a row with different
inputs -- the array keeps the previous call's contents, so the second call proves nothing stale
leaks -- and check that a problem too large for the array is refused before any launch.

This file is named to be collected last, and it passes both on its own in a fresh process and
after the rest of the suite.  Tolerances are the suite's (conftest.py).
"""
import ctypes

import pytest
import torch

import cabi
from conftest import assert_close_grad

pytestmark = pytest.mark.gpu

GRAD_NAMES = ("g_normal", "g_view", "g_albedo", "g_spec", "g_rough", "g_env")


def _lib():
    L = cabi.lib()
    f = L.des_shade_backward_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.POINTER(cabi.ShadeArgs), ctypes.c_uint, ctypes.c_void_p, ctypes.c_void_p] + \
        [ctypes.c_void_p] * 6 + [ctypes.c_void_p]
    return L


def _outputs(P, H, W):
    return [torch.empty(P, 3, device="cuda") for _ in range(4)] + [torch.empty(P, 1, device="cuda"),
                                                                    torch.empty(3, H, W, device="cuda")]


def _with_workspace(L, args, flags, d, stream):
    wsb = L.des_shade_workspace_bytes(args.P, args.H, args.W, flags, 1, torch.cuda.current_device())
    ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    outs = _outputs(args.P, args.H, args.W)
    st = L.des_shade_backward(ctypes.byref(args), flags, cabi.ptr(d.grad_shading), cabi.ptr(d.grad_diffuse_shading),
                              *[cabi.ptr(o) for o in outs], cabi.ptr(ws), wsb, stream)
    assert st == cabi.DES_OK, L.des_status_string(st)
    return outs


def _noalloc(L, args, flags, d, stream):
    outs = _outputs(args.P, args.H, args.W)
    st = L.des_shade_backward_noalloc(ctypes.byref(args), flags, cabi.ptr(d.grad_shading),
                                      cabi.ptr(d.grad_diffuse_shading), *[cabi.ptr(o) for o in outs], stream)
    assert st == cabi.DES_OK, L.des_status_string(st)
    return outs


def test_noalloc_backward_matches_workspace_entry_point_twice():
    assert torch.cuda.is_available()
    from diff_envshade_b200 import workloads as wl
    L = _lib()
    flags = cabi.DES_DIFFUSE | cabi.DES_SPECULAR
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    cases = [wl.make_inputs(70000, 16, 32, seed=801, vis_p=0.7, vis_layout="identity", rotation=True),
             wl.make_inputs(5000, 16, 32, seed=802, vis_p=0.6, vis_layout="mesh", rotation=True)]
    for inp in cases:  # two calls in a row, different inputs
        d = inp.to("cuda")
        args = cabi.make_args(d)
        want = _with_workspace(L, args, flags, d, stream)
        got = _noalloc(L, args, flags, d, stream)
        torch.cuda.synchronize()
        for name, g, w in zip(GRAD_NAMES, got, want):
            assert_close_grad(g.cpu(), w.cpu(), f"noalloc:{name}")


SCRATCH = 4 << 20  # DES_SHADE_NOALLOC_SCRATCH_BYTES


def _plan_bytes(L, P, H, W, flags):
    return L.des_shade_workspace_bytes(P, H, W, flags, 1, torch.cuda.current_device())


def test_noalloc_ordered_plan_ignores_reuse_flag():
    """A small map whose ordered plan fits the array (8x8 texels, 20,000 points: the points are
    ordered by normal direction inside the array).  DES_REUSE_ORDER is passed on purpose: no forward
    ever left an ordering in the array, so the entry point must order the points itself -- twice in
    a row with different point counts, so a stale permutation would lose points the second time."""
    from diff_envshade_b200 import workloads as wl
    L = _lib()
    flags = cabi.DES_DIFFUSE | cabi.DES_SPECULAR
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for P, seed in ((20000, 811), (17000, 812)):
        assert _plan_bytes(L, P, 8, 8, flags) <= SCRATCH  # the default (ordered) plan fits
        d = wl.make_inputs(P, 8, 8, seed=seed, vis_p=0.7, vis_layout="mesh", rotation=True).to("cuda")
        args = cabi.make_args(d)
        want = _with_workspace(L, args, flags, d, stream)
        got = _noalloc(L, args, flags | cabi.DES_REUSE_ORDER, d, stream)
        torch.cuda.synchronize()
        for name, g, w in zip(GRAD_NAMES, got, want):
            assert_close_grad(g.cpu(), w.cpu(), f"noalloc-ordered:{name}")


def test_noalloc_input_order_fallback():
    """Sizes whose ordered plan does not fit the array but whose input-order plan does (8x16 texels,
    300,000 points on a 148-SM B200): the call shades in input order with the default CTA width."""
    from diff_envshade_b200 import workloads as wl
    L = _lib()
    flags = cabi.DES_DIFFUSE | cabi.DES_SPECULAR
    P, H, W = 300000, 8, 16
    ordered, unordered = _plan_bytes(L, P, H, W, flags), _plan_bytes(L, P, H, W, flags | cabi.DES_INPUT_ORDER)
    if not (ordered > SCRATCH >= unordered):
        pytest.skip(f"plan sizes on this device do not isolate the input-order fallback ({ordered}, {unordered})")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    d = wl.make_inputs(P, H, W, seed=821, vis_p=0.6, vis_layout="identity", rotation=True).to("cuda")
    args = cabi.make_args(d)
    want = _with_workspace(L, args, flags, d, stream)
    got = _noalloc(L, args, flags, d, stream)
    torch.cuda.synchronize()
    for name, g, w in zip(GRAD_NAMES, got, want):
        assert_close_grad(g.cpu(), w.cpu(), f"noalloc-input-order:{name}")


def test_noalloc_refuses_problems_larger_than_its_scratch():
    L = _lib()
    flags = cabi.DES_DIFFUSE | cabi.DES_SPECULAR
    a = cabi.ShadeArgs()
    a.P, a.H, a.W, a.C = 1 << 20, 32, 64, 3
    need = L.des_shade_workspace_bytes(a.P, a.H, a.W, flags, 1, torch.cuda.current_device())
    assert need > 4 << 20
    dummy = ctypes.c_void_p(0x1000)  # never dereferenced: the size check fails before any launch
    for f in ("normal", "view_dir", "albedo", "specular_albedo", "roughness", "envmap", "light2obj_rotmat"):
        setattr(a, f, dummy)
    st = L.des_shade_backward_noalloc(ctypes.byref(a), flags, dummy, None, *([dummy] * 6), None)
    assert st == cabi.DES_ERR_WORKSPACE
