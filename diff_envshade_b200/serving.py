"""Python front end of the serving runtime (des_server_* in include/diff_envshade_b200.h).

The scheduler itself is native (a C++ thread inside libdes_b200.so): this module only binds the C
ABI with ctypes (calls release the GIL) and manages the host tensors a request points at.

    srv = Server(device=0, hbm_budget_bytes=40 << 30, tick_us=50)
    env = srv.add_envmap(envmap_3xHxW, rotation_3x3)
    mesh = srv.add_mesh(face_vertex_list_3xF_int32, visibility_SxV_int32)
    req = srv.submit(normal, view_dir, albedo, specular_albedo, roughness, env_id=env, mesh_id=mesh,
                     nearest_triangle_id=tri, barycentric_coord=bary, backward=True,
                     grad_shading=g, grad_diffuse_shading=gw)
    srv.drain(); srv.poll() -> finished records; req.outputs -> dict of host tensors
"""
import ctypes
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
_vp = ctypes.c_void_p

DES_DIFFUSE, DES_SPECULAR, DES_CLAMP = 1, 2, 4


class _Request(ctypes.Structure):
    _fields_ = [("P", ctypes.c_int64), ("env_id", ctypes.c_int32), ("mesh_id", ctypes.c_int32),
                ("flags", ctypes.c_uint), ("backward", ctypes.c_int32)] + \
               [(n, _vp) for n in ("normal", "view_dir", "albedo", "specular_albedo", "roughness",
                                   "nearest_triangle_id", "barycentric_coord", "grad_shading",
                                   "grad_diffuse_shading", "shading", "diffuse_shading", "g_normal", "g_view_dir",
                                   "g_albedo", "g_specular_albedo", "g_roughness", "g_envmap")]


class _Done(ctypes.Structure):
    _fields_ = [("ticket", ctypes.c_int64), ("t_submit_ns", ctypes.c_int64), ("t_admit_ns", ctypes.c_int64),
                ("t_uploaded_ns", ctypes.c_int64), ("t_ready_ns", ctypes.c_int64), ("t_computed_ns", ctypes.c_int64),
                ("t_done_ns", ctypes.c_int64),
                ("status", ctypes.c_int32), ("pad", ctypes.c_int32)]


class _Stats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_int64), ("completed", ctypes.c_int64), ("ticks", ctypes.c_int64),
                ("items", ctypes.c_int64), ("peak_arena_bytes", ctypes.c_int64), ("device_error", ctypes.c_int32),
                ("pad", ctypes.c_int32)]


_lib = None


def _load():
    global _lib
    if _lib is None:
        import diff_envshade_b200  # noqa: F401  (fails loudly if the native library is missing)
        L = ctypes.CDLL(os.path.join(_HERE, "libdes_b200.so"))
        L.des_status_string.restype = ctypes.c_char_p
        L.des_server_create.argtypes = [ctypes.c_int, ctypes.c_size_t, ctypes.c_int, ctypes.POINTER(_vp)]
        L.des_server_add_envmap.argtypes = [_vp, ctypes.c_int32, ctypes.c_int32, _vp, _vp,
                                            ctypes.POINTER(ctypes.c_int32)]
        L.des_server_add_mesh.argtypes = [_vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _vp, _vp,
                                          ctypes.POINTER(ctypes.c_int32)]
        L.des_server_submit.argtypes = [_vp, ctypes.POINTER(_Request), ctypes.POINTER(ctypes.c_int64)]
        L.des_server_poll.argtypes = [_vp, ctypes.POINTER(_Done), ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.des_server_drain.argtypes = [_vp, ctypes.c_int]
        L.des_server_stats.argtypes = [_vp, ctypes.POINTER(_Stats)]
        L.des_server_destroy.argtypes = [_vp]
        L.des_server_set_ticks_in_flight.argtypes = [_vp, ctypes.c_int]
        L.des_server_set_order_min_points.argtypes = [_vp, ctypes.c_int64]
        L.des_server_set_rank_by_size.argtypes = [_vp, ctypes.c_int]
        for f in ("des_server_create", "des_server_add_envmap", "des_server_add_mesh", "des_server_submit",
                  "des_server_poll", "des_server_drain", "des_server_stats", "des_server_destroy",
                  "des_server_set_ticks_in_flight", "des_server_set_order_min_points", "des_server_set_rank_by_size"):
            getattr(L, f).restype = ctypes.c_int
        _lib = L
    return _lib


def _check(st, what):
    if st != 0:
        raise RuntimeError(f"{what}: {_load().des_status_string(st).decode()}")


def _ptr(t):
    return None if t is None else _vp(t.data_ptr())


def _host(t, dtype, device=None):
    """Contiguous tensor of dtype that the server can read: a CUDA tensor on `device` stays where it
    is, anything else becomes pinned host memory (copies only when needed)."""
    t = t.detach()
    if device is not None and t.is_cuda and t.device.index == device:
        return t.to(dtype).contiguous()
    if t.device.type != "cpu" or t.dtype != dtype or not t.is_contiguous() or not t.is_pinned():
        t = t.to("cpu", dtype).contiguous().pin_memory()
    return t


class Request:
    """Handle of a submitted request: keeps its host tensors alive; outputs are valid once done."""

    def __init__(self, ticket, inputs, outputs, backward):
        self.ticket = ticket
        self._inputs = inputs
        self.outputs = outputs
        self.backward = backward
        self.done = None    # (t_submit_ns, t_admit_ns, t_done_ns) once finished
        self.stages = None  # dict of every stage time (ns since server creation) once finished
        self.status = None  # 0 (DES_OK) once finished successfully, else the des_status code


class Server:
    def __init__(self, device=0, hbm_budget_bytes=40 << 30, tick_us=50, ticks_in_flight=None,
                 order_min_points=None, rank_by_size=None):
        self._L = _load()
        h = _vp()
        _check(self._L.des_server_create(int(device), int(hbm_budget_bytes), int(tick_us), ctypes.byref(h)),
               "des_server_create")
        self._h = h
        if ticks_in_flight is not None:
            _check(self._L.des_server_set_ticks_in_flight(h, int(ticks_in_flight)), "des_server_set_ticks_in_flight")
        if rank_by_size is not None:
            _check(self._L.des_server_set_rank_by_size(h, int(bool(rank_by_size))), "des_server_set_rank_by_size")
        if order_min_points is not None:
            _check(self._L.des_server_set_order_min_points(h, int(order_min_points)),
                   "des_server_set_order_min_points")
        self._device = int(device)
        self._envs = {}
        self._requests = {}

    def add_envmap(self, envmap, light2obj_rotmat=None):
        env = _host(envmap, torch.float32)
        R = _host(torch.eye(3) if light2obj_rotmat is None else light2obj_rotmat, torch.float32)
        H, W = env.shape[-2], env.shape[-1]
        i = ctypes.c_int32()
        _check(self._L.des_server_add_envmap(self._h, H, W, _ptr(env), _ptr(R), ctypes.byref(i)), "add_envmap")
        self._envs[i.value] = (H, W)
        return i.value

    def add_mesh(self, face_vertex_list, visibility):
        f = _host(face_vertex_list, torch.int32)
        v = _host(visibility, torch.int32)
        i = ctypes.c_int32()
        _check(self._L.des_server_add_mesh(self._h, f.shape[1], v.shape[1], v.shape[0], _ptr(f), _ptr(v),
                                           ctypes.byref(i)), "add_mesh")
        return i.value

    def submit(self, normal, view_dir, albedo, specular_albedo, roughness, env_id, mesh_id=-1,
               nearest_triangle_id=None, barycentric_coord=None, backward=False, grad_shading=None,
               grad_diffuse_shading=None, enable_specular=True, outputs=None):
        """Queues one request.  Inputs are pinned host tensors or CUDA tensors on the server's
        device (anything else is copied to pinned memory first); `outputs` optionally supplies output
        tensors to write into (pinned or pageable host tensors, or CUDA tensors on the server's
        device).  Inputs and outputs must stay untouched until the request is done."""
        P = normal.shape[0]
        if env_id not in self._envs:
            _check(1, f"submit: unknown env_id {env_id}")  # DES_ERR_INVALID_ARGUMENT, as the C ABI returns
        H, W = self._envs[env_id]
        dv = self._device
        ins = {k: _host(v, torch.float32, dv) for k, v in (("normal", normal), ("view_dir", view_dir),
                                                            ("albedo", albedo), ("specular_albedo", specular_albedo),
                                                            ("roughness", roughness))}
        if mesh_id >= 0:
            ins["nearest_triangle_id"] = _host(nearest_triangle_id, torch.int64, dv)
            ins["barycentric_coord"] = _host(barycentric_coord, torch.float32, dv)
        if backward:
            ins["grad_shading"] = _host(grad_shading, torch.float32, dv)
            if grad_diffuse_shading is not None:
                ins["grad_diffuse_shading"] = _host(grad_diffuse_shading, torch.float32, dv)
        if outputs is None:
            pin = dict(dtype=torch.float32, pin_memory=True)
            outputs = {"shading": torch.empty(P, 3, **pin), "diffuse_shading": torch.empty(P, 3, **pin)}
            if backward:
                for k in ("g_normal", "g_view_dir", "g_albedo", "g_specular_albedo"):
                    outputs[k] = torch.empty(P, 3, **pin)
                outputs["g_roughness"] = torch.empty(P, 1, **pin)
                outputs["g_envmap"] = torch.empty(3, H, W, **pin)
        q = _Request()
        q.P, q.env_id, q.mesh_id = P, env_id, mesh_id
        q.flags = DES_DIFFUSE | (DES_SPECULAR if enable_specular else 0)
        q.backward = 1 if backward else 0
        for k, v in ins.items():
            setattr(q, k, _ptr(v))
        for k, v in outputs.items():
            setattr(q, k, _ptr(v))
        t = ctypes.c_int64()
        _check(self._L.des_server_submit(self._h, ctypes.byref(q), ctypes.byref(t)), "submit")
        req = Request(t.value, ins, outputs, backward)
        self._requests[t.value] = req
        return req

    def poll(self, max_items=4096):
        buf = (_Done * max_items)()
        n = ctypes.c_int()
        _check(self._L.des_server_poll(self._h, buf, max_items, ctypes.byref(n)), "poll")
        out = []
        for i in range(n.value):
            d = buf[i]
            req = self._requests.pop(d.ticket, None)
            if req is not None:
                req.status = d.status
                req.done = (d.t_submit_ns, d.t_admit_ns, d.t_done_ns)
                req.stages = {"submit": d.t_submit_ns, "admit": d.t_admit_ns, "uploaded": d.t_uploaded_ns,
                              "ready": d.t_ready_ns,
                              "computed": d.t_computed_ns, "done": d.t_done_ns}
                out.append(req)
        return out

    def drain(self, timeout_s=120.0):
        _check(self._L.des_server_drain(self._h, int(timeout_s * 1000)), "drain")

    def stats(self):
        s = _Stats()
        _check(self._L.des_server_stats(self._h, ctypes.byref(s)), "stats")
        return {k: getattr(s, k) for k, _ in _Stats._fields_ if k != "pad"}

    def close(self):
        if getattr(self, "_h", None):
            self._L.des_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
