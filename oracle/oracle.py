"""ctypes front-end of the CPU oracle (envshade_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()`` as the checker,
and by ``bench.py``'s CPU-baseline leg.  The product package never imports this module.

The oracle restates the reference's sum and adjoint (bruteforce_shader.cu:124-227, 231-2683)
in FP64 (the checker) or FP32 (the CPU baseline), multithreaded with std::thread.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "envshade_oracle.cpp")
SRCS = [SRC, os.path.join(HERE, "mesh_oracle.cpp")]
LIB = os.path.join(HERE, "libdes_oracle.so")

DIFFUSE, SPECULAR, CLAMP, WHITE, V1ORDER = 1, 2, 4, 8, 16

# flags of each reference operator family (the oracle's kV1Order selects the v1 term order)
OP_FLAGS = {
    "diffuse": DIFFUSE | V1ORDER,
    "specular": V1ORDER,          # | DIFFUSE / SPECULAR from enable_* arguments
    "specular_clamp": V1ORDER | CLAMP,
    "specular2": DIFFUSE | WHITE,  # | SPECULAR when enabled
    "specularvisibility2": DIFFUSE | WHITE,
}


def build(force=False):
    if not force and os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(s) for s in SRCS):
        return LIB
    tmp = LIB + ".tmp"
    subprocess.check_call(["g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-pthread", *SRCS, "-o", tmp])
    os.replace(tmp, LIB)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB)
        P = ctypes.c_void_p
        for suf in ("f64", "f32"):
            f = getattr(L, f"des_oracle_forward_{suf}")
            f.restype = ctypes.c_int
            f.argtypes = [ctypes.c_int64, ctypes.c_int, ctypes.c_int] + [P] * 7 + [ctypes.c_int, ctypes.c_int] + \
                [P] * 4 + [ctypes.c_uint, P, P, ctypes.c_int]
            b = getattr(L, f"des_oracle_backward_{suf}")
            b.restype = ctypes.c_int
            b.argtypes = [ctypes.c_int64, ctypes.c_int, ctypes.c_int] + [P] * 7 + [ctypes.c_int, ctypes.c_int] + \
                [P] * 4 + [ctypes.c_uint] + [P] * 8 + [ctypes.c_int]
        L.des_oracle_texel_table_f64.restype = None
        L.des_oracle_texel_table_f64.argtypes = [ctypes.c_int, ctypes.c_int, P, P]
        i64 = ctypes.c_int64
        L.des_oracle_uv_of_triangle_f64.restype = None
        L.des_oracle_uv_of_triangle_f64.argtypes = [i64, P, P, P]
        L.des_oracle_uv_of_triangle_backward_f64.restype = None
        L.des_oracle_uv_of_triangle_backward_f64.argtypes = [i64, P, P, P, P]
        for suf in ("f64", "f32"):
            f = getattr(L, f"des_oracle_nearest_mesh_points_{suf}")
            f.restype = i64
            f.argtypes = [i64] * 5 + [P] * 8
        L.des_oracle_nearest_mesh_points_backward_f64.restype = None
        L.des_oracle_nearest_mesh_points_backward_f64.argtypes = [i64, i64, i64] + [P] * 6
        L.des_oracle_extract_bitfield.restype = None
        L.des_oracle_extract_bitfield.argtypes = [i64] * 4 + [P, P]
        L.des_oracle_sample_envmap_f64.restype = None
        L.des_oracle_sample_envmap_f64.argtypes = [i64, ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P, P]
        _lib = L
    return _lib


def _np(x, dtype):
    if x is None:
        return None
    if hasattr(x, "detach"):
        x = x.detach().cpu().numpy()
    return np.ascontiguousarray(np.asarray(x), dtype=dtype)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def texel_table_f64(H, W, R=None):
    """Exact-trigonometry texel table [H*W, 4] = (rotated x, y, z, d_omega), in memory order."""
    R = np.eye(3) if R is None else _np(R, np.float64)
    out = np.zeros((H * W, 4), dtype=np.float64)
    lib().des_oracle_texel_table_f64(H, W, _ptr(np.ascontiguousarray(R, dtype=np.float64)), _ptr(out))
    return out


class _Prepared:
    def __init__(self, inp, table, dtype):
        self.dtype = dtype
        self.P = inp.normal.shape[0]
        self.H, self.W = inp.envmap.shape[-2], inp.envmap.shape[-1]
        self.normal = _np(inp.normal, dtype)
        self.view = _np(inp.view_dir, dtype)
        self.albedo = _np(inp.albedo, dtype)
        self.spec = _np(inp.specular_albedo, dtype)
        self.rough = _np(inp.roughness, dtype)
        self.env = _np(inp.envmap, dtype)
        if table is None:
            table = texel_table_f64(self.H, self.W, inp.light2obj_rotmat)
        self.table = _np(table, dtype)
        if getattr(inp, "visibility", None) is not None:
            self.faces = _np(inp.face_vertex_list, np.int32)
            self.tri = _np(inp.nearest_triangle_id, np.int64)
            self.bary = _np(inp.barycentric_coord, dtype)
            self.vis = _np(inp.visibility, np.int32).view(np.uint32)
            self.N_face, self.N_vertex = self.faces.shape[1], self.vis.shape[1]
        else:
            self.faces = self.tri = self.bary = self.vis = None
            self.N_face = self.N_vertex = 0

    def common(self):
        return [self.P, self.H, self.W, _ptr(self.normal), _ptr(self.view), _ptr(self.albedo), _ptr(self.spec),
                _ptr(self.rough), _ptr(self.env), _ptr(self.table), self.N_face, self.N_vertex, _ptr(self.faces),
                _ptr(self.tri), _ptr(self.bary), _ptr(self.vis)]


def forward(inp, flags, table=None, dtype=np.float64, nthreads=0, points=None):
    """Returns (shading, diffuse_shading) as [P, 3] arrays (diffuse_shading zeros unless WHITE).

    ``inp`` has the attributes of workloads.ShadeInputs; ``table`` is an optional [H*W, 4] texel
    table (e.g. the one the GPU built); ``points`` optionally restricts to a subset of indices.
    """
    inp = _subset(inp, points)
    pr = _Prepared(inp, table, dtype)
    sh = np.zeros((pr.P, 3), dtype=dtype)
    wh = np.zeros((pr.P, 3), dtype=dtype)
    fn = lib().des_oracle_forward_f64 if dtype == np.float64 else lib().des_oracle_forward_f32
    st = fn(*pr.common(), flags, _ptr(sh), _ptr(wh), nthreads)
    if st != 0:
        raise RuntimeError(f"oracle forward failed ({st})")
    return sh, wh


def backward(inp, flags, grad_shading, grad_white=None, table=None, dtype=np.float64, nthreads=0, points=None):
    """Returns dict of g_normal, g_view, g_albedo, g_spec [P,3], g_rough [P,1], g_env [3,H,W]."""
    inp = _subset(inp, points)
    if points is not None:
        grad_shading = _np(grad_shading, dtype)[points]
        grad_white = None if grad_white is None else _np(grad_white, dtype)[points]
    pr = _Prepared(inp, table, dtype)
    gs = _np(grad_shading, dtype)
    gw = _np(grad_white, dtype)
    out = {k: np.zeros((pr.P, 3), dtype=dtype) for k in ("g_normal", "g_view", "g_albedo", "g_spec")}
    out["g_rough"] = np.zeros((pr.P, 1), dtype=dtype)
    out["g_env"] = np.zeros((3, pr.H, pr.W), dtype=dtype)
    fn = lib().des_oracle_backward_f64 if dtype == np.float64 else lib().des_oracle_backward_f32
    st = fn(*pr.common(), flags, _ptr(gs), _ptr(gw), _ptr(out["g_normal"]), _ptr(out["g_view"]),
            _ptr(out["g_albedo"]), _ptr(out["g_spec"]), _ptr(out["g_rough"]), _ptr(out["g_env"]), nthreads)
    if st != 0:
        raise RuntimeError(f"oracle backward failed ({st})")
    return out


def _subset(inp, points):
    if points is None:
        return inp
    import copy
    idx = np.asarray(points)
    out = copy.copy(inp)
    for k in ("normal", "view_dir", "albedo", "specular_albedo", "roughness"):
        setattr(out, k, _np(getattr(inp, k), np.float64)[idx])
    if getattr(inp, "visibility", None) is not None:
        out.nearest_triangle_id = _np(inp.nearest_triangle_id, np.int64)[idx]
        out.barycentric_coord = _np(inp.barycentric_coord, np.float64)[:, idx]
    return out


def flags_for(op, enable_diffuse=True, enable_specular=True):
    f = OP_FLAGS[op]
    if op in ("specular", "specular_clamp"):
        f |= (DIFFUSE if enable_diffuse else 0) | (SPECULAR if enable_specular else 0)
    elif enable_specular and op != "diffuse":
        f |= SPECULAR
    return f


# ---- mesh-side helpers and env-map sampling (mesh_oracle.cpp; reference etc.cu) ----

def uv_of_triangle(triangles, query_pos):
    """[P, 3, 3] triangles, [P, 3] queries -> [P, 3] barycentric (1 - s - t, s, t), FP64."""
    tri = _np(triangles, np.float64).reshape(-1, 9)
    q = _np(query_pos, np.float64).reshape(-1, 3)
    out = np.zeros((q.shape[0], 3))
    lib().des_oracle_uv_of_triangle_f64(q.shape[0], _ptr(tri), _ptr(q), _ptr(out))
    return out


def uv_of_triangle_backward(triangles, query_pos, grad_bary):
    tri = _np(triangles, np.float64).reshape(-1, 9)
    q = _np(query_pos, np.float64).reshape(-1, 3)
    g = _np(grad_bary, np.float64).reshape(-1, 3)
    out = np.zeros_like(q)
    lib().des_oracle_uv_of_triangle_backward_f64(q.shape[0], _ptr(tri), _ptr(q), _ptr(g), _ptr(out))
    return out


def nearest_mesh_points(adjacency_head, adjacency_list, faces, vertex_pos, query_pos, idxs, dtype=np.float64):
    """Returns (triangle id [P] int64, barycentric [3, P], number of queries without a face)."""
    head = _np(adjacency_head, np.int32)
    lst = _np(adjacency_list, np.int32)
    f = _np(faces, np.int32)
    vp = _np(vertex_pos, dtype)
    q = _np(query_pos, dtype)
    ix = _np(idxs, np.int64)
    P, K = q.shape[1], ix.shape[1]
    tri = np.zeros(P, dtype=np.int64)
    bary = np.zeros((3, P), dtype=dtype)
    fn = lib().des_oracle_nearest_mesh_points_f64 if dtype == np.float64 else lib().des_oracle_nearest_mesh_points_f32
    missing = fn(head.shape[1], f.shape[1], P, K, lst.size, _ptr(head), _ptr(lst), _ptr(f), _ptr(vp), _ptr(q),
                 _ptr(ix), _ptr(tri), _ptr(bary))
    return tri, bary, int(missing)


def nearest_mesh_points_backward(faces, vertex_pos, query_pos, tri, grad_bary):
    f = _np(faces, np.int32)
    vp = _np(vertex_pos, np.float64)
    q = _np(query_pos, np.float64)
    t = _np(tri, np.int64)
    g = _np(grad_bary, np.float64)
    out = np.zeros_like(q)
    lib().des_oracle_nearest_mesh_points_backward_f64(vp.shape[1], f.shape[1], q.shape[1], _ptr(f), _ptr(vp), _ptr(q),
                                                      _ptr(t), _ptr(g), _ptr(out))
    return out


def extract_bitfield(bitfield, N_bit, i_start, i_end):
    w = _np(bitfield, np.int32).view(np.uint32)
    out = np.zeros((i_end - i_start, N_bit), dtype=np.float32)
    lib().des_oracle_extract_bitfield(w.shape[1], N_bit, i_start, i_end, _ptr(w), _ptr(out))
    return out


def sample_envmap(query_point, envmap):
    """[3, P] directions, [C, H, W] env -> [C, P] bilinear lat-long samples, FP64."""
    q = _np(query_point, np.float64)
    env = _np(envmap, np.float64)
    C, H, W = env.shape
    out = np.zeros((C, q.shape[1]))
    lib().des_oracle_sample_envmap_f64(q.shape[1], H, W, C, _ptr(q), _ptr(env), _ptr(out))
    return out
