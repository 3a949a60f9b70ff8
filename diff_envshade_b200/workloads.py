"""Seeded synthetic shading workloads.

The reference measures on no dataset; these generators produce inputs with the shapes and
value distributions of the benchmark configurations:

  normals        unit vectors uniform on the sphere (normalised Gaussians)
  view dirs      unit vectors uniform in the normal's hemisphere (sampled on the sphere, flipped)
  albedo         U[0,1]^3;  roughness U[r_lo, r_hi];  specular albedo U[0,0.1]^3
  env map        3 x H x W, radiance exp(N(0, sigma))
  visibility     each texel bit Bernoulli(p), packed LSB-first, 32 texels per int32 word,
                 words laid out [N_slot][N_vertex] (texel t -> bit t%32 of slot t//32)

Two visibility layouts exist: ``identity`` (one vertex per point, triangle (p,p,p),
barycentrics (1,0,0), so each point's visibility is exactly its own bits) and ``mesh``
(random triangles over P/2 vertices, Dirichlet(1,1,1) barycentrics) which exercises the
barycentric interpolation.  All draws use a CPU ``torch.Generator`` so the same seed gives the
same tensors on every machine.
"""
import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np
import torch

# name -> (P, H, W, env sigma, roughness range, visibility probability or None, K env maps)
CONFIGS = {
    "plain-4k": dict(P=4096, H=16, W=32, sigma=1.0, rough=(0.2, 0.9), vis_p=None, K=1, seed=1234),
    "vis-70k": dict(P=70000, H=16, W=32, sigma=1.0, rough=(0.2, 0.9), vis_p=0.7, K=1, seed=1235),
    "vis-1m": dict(P=1048576, H=32, W=64, sigma=1.5, rough=(0.05, 1.0), vis_p=0.6, K=1, seed=1236),
    "multienv-262k": dict(P=262144, H=16, W=32, sigma=1.0, rough=(0.2, 0.9), vis_p=0.7, K=64, seed=1237),
}


@dataclass
class ShadeInputs:
    normal: torch.Tensor
    view_dir: torch.Tensor
    albedo: torch.Tensor
    specular_albedo: torch.Tensor
    roughness: torch.Tensor
    envmap: torch.Tensor
    light2obj_rotmat: torch.Tensor
    face_vertex_list: Optional[torch.Tensor] = None
    nearest_triangle_id: Optional[torch.Tensor] = None
    barycentric_coord: Optional[torch.Tensor] = None
    visibility: Optional[torch.Tensor] = None
    grad_shading: Optional[torch.Tensor] = None
    grad_diffuse_shading: Optional[torch.Tensor] = None
    meta: dict = field(default_factory=dict)

    @property
    def P(self):
        return self.normal.shape[0]

    @property
    def HW(self):
        return self.envmap.shape[1] * self.envmap.shape[2]

    @property
    def has_vis(self):
        return self.visibility is not None

    def tensors(self):
        return {k: v for k, v in self.__dict__.items() if isinstance(v, torch.Tensor)}

    def to(self, device):
        kw = {k: (v.to(device) if isinstance(v, torch.Tensor) else v) for k, v in self.__dict__.items()}
        return ShadeInputs(**kw)

    def pin(self):
        kw = {k: (v.pin_memory() if isinstance(v, torch.Tensor) else v) for k, v in self.__dict__.items()}
        return ShadeInputs(**kw)

    def vis_tuple(self):
        if not self.has_vis:
            return None
        return (self.face_vertex_list, self.nearest_triangle_id, self.barycentric_coord, self.visibility)


def _unit(x):
    return x / x.norm(dim=-1, keepdim=True).clamp_min(1e-12)


def random_rotation(g):
    q = _unit(torch.randn(4, generator=g, dtype=torch.float64))
    w, x, y, z = q.tolist()
    R = torch.tensor([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                      [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                      [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]], dtype=torch.float64)
    return R.float()


def pack_bits(bits):
    """bits: bool [P, n_texels] -> int32 [ceil(n/32), P] words, texel t = bit t%32 of slot t//32."""
    P, n = bits.shape
    nslots = (n + 31) // 32
    b = bits.numpy()
    if n != nslots * 32:
        b = np.concatenate([b, np.zeros((P, nslots * 32 - n), dtype=bool)], axis=1)
    # little-endian bit order within each byte and byte order within each word: bit t%32 of word t//32
    words = np.packbits(b, axis=1, bitorder="little").view("<u4")  # [P, nslots]
    return torch.from_numpy(np.ascontiguousarray(words.T).view(np.int32))


def random_visibility(g, N_vertex, n_texels, p, rows_per_draw=None):
    """Packed Bernoulli(p) visibility words [ceil(n/32), N_vertex].  Large tables are drawn in blocks
    of vertices so that host memory stays bounded; tables of up to 2^28 bits are one draw."""
    if rows_per_draw is None:
        rows_per_draw = N_vertex if N_vertex * n_texels <= (1 << 28) else max(1, (1 << 25) // n_texels)
    parts = []
    for v0 in range(0, N_vertex, rows_per_draw):
        rows = min(rows_per_draw, N_vertex - v0)
        parts.append(pack_bits(torch.rand(rows, n_texels, generator=g) < p))
    return parts[0] if len(parts) == 1 else torch.cat(parts, dim=1).contiguous()


def unpack_bits(words, n_texels):
    """int32 [N_slot, N] -> bool [N, n_texels] (inverse of pack_bits)."""
    w = words.cpu().numpy().view(np.uint32).astype(np.uint64)  # [S, N]
    bits = ((w[:, None, :] >> np.arange(32, dtype=np.uint64)[None, :, None]) & 1).astype(bool)  # [S, 32, N]
    bits = bits.reshape(-1, w.shape[1])[:n_texels]
    return torch.from_numpy(np.ascontiguousarray(bits.T))


def make_inputs(P, H, W, seed, sigma=1.0, rough=(0.2, 0.9), vis_p=None, vis_layout="identity", rotation=False,
                grads=True, env_count=1):
    g = torch.Generator().manual_seed(seed)
    n = _unit(torch.randn(P, 3, generator=g))
    v = _unit(torch.randn(P, 3, generator=g))
    v = torch.where(((v * n).sum(-1, keepdim=True) < 0), -v, v)
    albedo = torch.rand(P, 3, generator=g)
    rough_t = rough[0] + (rough[1] - rough[0]) * torch.rand(P, 1, generator=g)
    spec = 0.1 * torch.rand(P, 3, generator=g)
    shape = (3, H, W) if env_count == 1 else (env_count, 3, H, W)
    env = torch.exp(sigma * torch.randn(*shape, generator=g))
    R = random_rotation(g) if rotation else torch.eye(3)
    inp = ShadeInputs(n.contiguous(), v.contiguous(), albedo, spec, rough_t, env.contiguous(), R.contiguous())
    inp.meta = dict(P=P, H=H, W=W, seed=seed, sigma=sigma, rough=rough, vis_p=vis_p, vis_layout=vis_layout)
    if vis_p is not None:
        HW = H * W
        if vis_layout == "identity":
            N_vertex = P
            faces = torch.arange(P, dtype=torch.int32).repeat(3, 1).contiguous()
            tri = torch.arange(P, dtype=torch.int64)
            bary = torch.zeros(3, P)
            bary[0] = 1.0
        elif vis_layout == "mesh":
            N_vertex = max(P // 2, 3)
            N_face = max(P, 1)
            faces = torch.randint(0, N_vertex, (3, N_face), generator=g, dtype=torch.int64).to(torch.int32)
            tri = torch.randint(0, N_face, (P,), generator=g, dtype=torch.int64)
            e = -torch.log(torch.rand(3, P, generator=g).clamp_min(1e-12))
            bary = (e / e.sum(0, keepdim=True)).contiguous()
        else:
            raise ValueError(vis_layout)
        inp.face_vertex_list = faces.contiguous()
        inp.nearest_triangle_id = tri.contiguous()
        inp.barycentric_coord = bary.contiguous()
        inp.visibility = random_visibility(g, N_vertex, HW, vis_p)
    if grads:
        inp.grad_shading = torch.randn(P, 3, generator=g)
        inp.grad_diffuse_shading = torch.randn(P, 3, generator=g)
    return inp


def make_config(name, **overrides):
    c = dict(CONFIGS[name])
    c.update(overrides)
    return make_inputs(c["P"], c["H"], c["W"], c["seed"], sigma=c["sigma"], rough=c["rough"], vis_p=c["vis_p"],
                       env_count=c.get("K", 1))


# ---- mesh inputs of the visibility-gather helpers (get_nearest_mesh_points / get_uv_of_triangle) ----

def make_sphere_mesh(n_lat, n_lon, seed, jitter=0.01):
    """A closed UV sphere of radius 1 with jittered vertices: vertex_pos [3, N_vertex] float32,
    face_vertex_list [3, N_face] int32 (two poles + n_lat rings of n_lon vertices)."""
    g = torch.Generator().manual_seed(seed)
    th = (torch.arange(1, n_lat + 1, dtype=torch.float64) / (n_lat + 1)) * math.pi
    ph = torch.arange(n_lon, dtype=torch.float64) / n_lon * 2 * math.pi
    T, Ph = torch.meshgrid(th, ph, indexing="ij")
    ring = torch.stack([torch.sin(T) * torch.cos(Ph), torch.cos(T), torch.sin(T) * torch.sin(Ph)], 0).reshape(3, -1)
    pos = torch.cat([torch.tensor([[0.0], [1.0], [0.0]], dtype=torch.float64), ring,
                     torch.tensor([[0.0], [-1.0], [0.0]], dtype=torch.float64)], 1)
    pos = pos + jitter * torch.randn(pos.shape, generator=g, dtype=torch.float64)
    top, bot = 0, 1 + n_lat * n_lon
    vid = lambda i, j: 1 + i * n_lon + (j % n_lon)  # noqa: E731
    faces = []
    for j in range(n_lon):
        faces.append((top, vid(0, j + 1), vid(0, j)))
        faces.append((bot, vid(n_lat - 1, j), vid(n_lat - 1, j + 1)))
    for i in range(n_lat - 1):
        for j in range(n_lon):
            a, b, c, d = vid(i, j), vid(i, j + 1), vid(i + 1, j), vid(i + 1, j + 1)
            faces.append((a, b, c))
            faces.append((b, d, c))
    f = torch.tensor(faces, dtype=torch.int32).T.contiguous()
    return pos.float().contiguous(), f


def vertex_adjacency(face_vertex_list, N_vertex):
    """adjacency_head [2, N_vertex] int32 (faces per vertex; inclusive prefix sum of the counts) and
    adjacency_list int32 (face ids per vertex, ascending), the layout the reference's
    get_nearest_mesh_points_forward reads."""
    f = face_vertex_list.long()
    N_face = f.shape[1]
    verts = f.reshape(-1)
    fid = torch.arange(N_face).repeat(3)
    order = torch.argsort(verts * N_face + fid)
    lst = fid[order].to(torch.int32)
    count = torch.bincount(verts, minlength=N_vertex).to(torch.int32)
    head = torch.stack([count, torch.cumsum(count, 0).to(torch.int32)], 0).contiguous()
    return head, lst.contiguous()


def make_mesh_queries(vertex_pos, P, K, seed, spread=0.05, device="cpu"):
    """Query points near the mesh surface [3, P] and their K nearest vertices [P, K] int64."""
    g = torch.Generator().manual_seed(seed)
    N_vertex = vertex_pos.shape[1]
    base = torch.randint(0, N_vertex, (P,), generator=g)
    q = vertex_pos[:, base] + spread * torch.randn(3, P, generator=g)
    qd, vd = q.to(device), vertex_pos.to(device)
    idx = []
    for s in range(0, P, 4096):  # brute-force kNN in blocks
        d = torch.cdist(qd[:, s:s + 4096].T.double(), vd.T.double())
        idx.append(torch.topk(d, K, dim=1, largest=False).indices.cpu())
    return q.contiguous(), torch.cat(idx, 0).to(torch.int64).contiguous()
