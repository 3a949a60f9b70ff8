"""ctypes view of the C ABI (include/diff_envshade_b200.h) used by the tests.

This is the binding a C-ABI consumer written in Python would use (plain ctypes over the shared
library); the tests call the library through it directly, without the torch extension.
"""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "diff_envshade_b200.h")
LIBPATH = os.path.join(ROOT, "diff_envshade_b200", "libdes_b200.so")

DES_OK, DES_ERR_INVALID_ARGUMENT, DES_ERR_UNSUPPORTED, DES_ERR_WORKSPACE, DES_ERR_CUDA, DES_ERR_BAD_INDEX = range(6)
DES_DIFFUSE, DES_SPECULAR, DES_CLAMP = 1, 2, 4
DES_INPUT_ORDER = 16
DES_COMPACT = 32
DES_REUSE_ORDER = 64
DES_REUSE_TABLE = 128

vp = ctypes.c_void_p


class ShadeArgs(ctypes.Structure):
    _fields_ = [
        ("P", ctypes.c_int64), ("H", ctypes.c_int32), ("W", ctypes.c_int32), ("C", ctypes.c_int32),
        ("normal", vp), ("view_dir", vp), ("albedo", vp), ("specular_albedo", vp), ("roughness", vp),
        ("envmap", vp), ("light2obj_rotmat", vp),
        ("N_face", ctypes.c_int32), ("N_vertex", ctypes.c_int32), ("N_slot", ctypes.c_int32),
        ("face_vertex_list", vp), ("nearest_triangle_id", vp), ("barycentric_coord", vp), ("visibility", vp),
    ]


def declared_functions():
    """Names of every function the public header declares."""
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(des_[a-z0-9_]+)\s*\(", text)))


_lib = None


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIBPATH)
        L.des_status_string.restype = ctypes.c_char_p
        L.des_status_string.argtypes = [ctypes.c_int]
        L.des_abi_version.restype = ctypes.c_int
        L.des_shade_workspace_bytes.restype = ctypes.c_size_t
        L.des_shade_workspace_bytes.argtypes = [ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, ctypes.c_uint,
                                                ctypes.c_int, ctypes.c_int]
        L.des_shade_forward.restype = ctypes.c_int
        L.des_shade_forward.argtypes = [ctypes.POINTER(ShadeArgs), ctypes.c_uint, vp, vp, vp, ctypes.c_size_t, vp]
        L.des_shade_backward.restype = ctypes.c_int
        L.des_shade_backward.argtypes = [ctypes.POINTER(ShadeArgs), ctypes.c_uint, vp, vp] + [vp] * 6 + \
            [vp, ctypes.c_size_t, vp]
        L.des_texel_table.restype = ctypes.c_int
        L.des_texel_table.argtypes = [ctypes.c_int32, ctypes.c_int32, vp, vp, vp]
        L.des_workspace_status.restype = ctypes.c_int
        L.des_workspace_status.argtypes = [vp, ctypes.c_size_t, ctypes.POINTER(ctypes.c_int), vp]
        _lib = L
    return _lib


def ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def make_args(inp, with_vis=True):
    """ShadeArgs over device tensors of a workloads.ShadeInputs (kept alive by the caller)."""
    a = ShadeArgs()
    a.P = inp.normal.shape[0]
    a.C = inp.albedo.shape[1]
    a.H, a.W = inp.envmap.shape[-2], inp.envmap.shape[-1]
    a.normal, a.view_dir, a.albedo = ptr(inp.normal), ptr(inp.view_dir), ptr(inp.albedo)
    a.specular_albedo, a.roughness = ptr(inp.specular_albedo), ptr(inp.roughness)
    a.envmap, a.light2obj_rotmat = ptr(inp.envmap), ptr(inp.light2obj_rotmat)
    if with_vis and inp.visibility is not None:
        a.N_face = inp.face_vertex_list.shape[1]
        a.N_vertex = inp.visibility.shape[1]
        a.N_slot = inp.visibility.shape[0]
        a.face_vertex_list = ptr(inp.face_vertex_list)
        a.nearest_triangle_id = ptr(inp.nearest_triangle_id)
        a.barycentric_coord = ptr(inp.barycentric_coord)
        a.visibility = ptr(inp.visibility)
    return a
