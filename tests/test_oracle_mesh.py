"""CPU checks of the oracle's mesh-side and env-map helpers (oracle/mesh_oracle.cpp).

Pinned to the reference's own outputs: tests/golden/etc_*.npz were written by
tests/golden/make_golden.py --only-etc from the reference extension on a B200.  Bounds (FP64 oracle
against the reference's FP32):
  * barycentric coordinates: max |d| <= 1e-5 for get_uv_of_triangle, 5e-5 for the nearest point
    (the reference's FP32 rounding of s, t);
  * gradients of the closest-point map: max |d| <= 1e-4 * max|ref| on at least 99% of the queries
    (the map's Jacobian jumps across region boundaries, where FP32 and FP64 may classify a query
    differently);
  * nearest triangle: the same face, or an equally close one (|d^2 difference| <= 1e-6);
  * extract_bitfield: bit-exact; sample_envmap: max relative |d| <= 1e-4 (FP32 atan2f / asinf
    rounding of the lookup coordinate, amplified by the map's texel-to-texel gradient).
The adjoints are also checked against central finite differences of the FP64 forward.
"""
import numpy as np
import pytest
import torch

from conftest import GOLDEN
from oracle import oracle as orc


def _load(name):
    return np.load(f"{GOLDEN}/{name}")


def test_uv_of_triangle_matches_reference_fixture():
    d = _load("etc_uv_of_triangle.npz")
    b = orc.uv_of_triangle(d["triangles"], d["query_pos"])
    assert np.abs(b - d["ref_barycentric_coord"]).max() <= 1e-5
    g = orc.uv_of_triangle_backward(d["triangles"], d["query_pos"], d["grad_barycentric_coord"])
    r = d["ref_grad_query_pos"]
    ok = (np.abs(g - r) <= 1e-4 * np.abs(r).max()).all(1)
    assert ok.mean() >= 0.99, ok.mean()


def test_uv_of_triangle_adjoint_matches_finite_differences():
    g = np.random.default_rng(1)
    P = 400
    tri = g.normal(size=(P, 3, 3))
    q = tri.mean(1) + 0.7 * g.normal(size=(P, 3))
    gb = g.normal(size=(P, 3))
    ana = orc.uv_of_triangle_backward(tri, q, gb)
    h = 1e-7
    fd = np.zeros_like(q)
    for c in range(3):
        e = np.zeros(3)
        e[c] = h
        fd[:, c] = ((orc.uv_of_triangle(tri, q + e) - orc.uv_of_triangle(tri, q - e)) * gb).sum(1) / (2 * h)
    # away from region boundaries (where the map has kinks) the two agree to FD precision
    ok = (np.abs(ana - fd) <= 1e-5 * (1 + np.abs(fd))).all(1)
    assert ok.mean() >= 0.98, ok.mean()


def test_nearest_mesh_points_matches_reference_fixture():
    d = _load("etc_nearest_mesh_points.npz")
    tri, bary, missing = orc.nearest_mesh_points(d["adjacency_head"], d["adjacency_list"], d["face_vertex_list"],
                                                 d["vertex_pos"], d["query_pos"], d["idxs"])
    assert missing == 0
    ref_tri, ref_bary = d["ref_nearest_triangle_id"], d["ref_barycentric_coord"]
    V = d["vertex_pos"].astype(np.float64)
    F = d["face_vertex_list"]
    Q = d["query_pos"].astype(np.float64)

    def dist2(face, b):
        p = b[0] * V[:, F[0, face]] + b[1] * V[:, F[1, face]] + b[2] * V[:, F[2, face]]
        return ((p - Q) ** 2).sum(0)

    same = tri == ref_tri
    tie = np.abs(dist2(tri, bary) - dist2(ref_tri, ref_bary.astype(np.float64))) <= 1e-6
    assert (same | tie).all()
    assert np.abs(bary[:, same] - ref_bary[:, same]).max() <= 5e-5


def test_nearest_mesh_points_is_the_global_nearest_on_a_closed_sphere():
    from diff_envshade_b200 import workloads as wl
    pos, faces = wl.make_sphere_mesh(12, 24, seed=3)
    head, lst = wl.vertex_adjacency(faces, pos.shape[1])
    q, idx = wl.make_mesh_queries(pos, 300, 4, seed=4)
    tri, bary, missing = orc.nearest_mesh_points(head, lst, faces, pos, q, idx)
    assert missing == 0
    V = pos.numpy().astype(np.float64)
    F = faces.numpy()
    T = np.stack([V[:, F[0]].T, V[:, F[1]].T, V[:, F[2]].T], 1)
    for i in range(0, 300, 7):
        b = orc.uv_of_triangle(T, np.repeat(q.numpy()[:, i:i + 1].T.astype(np.float64), len(T), 0))
        cp = (b[:, :, None] * T).sum(1)
        d2 = ((cp - q.numpy()[:, i].astype(np.float64)) ** 2).sum(1)
        assert d2[tri[i]] <= d2.min() + 1e-12


def test_nearest_mesh_points_adjoint_matches_finite_differences():
    from diff_envshade_b200 import workloads as wl
    pos, faces = wl.make_sphere_mesh(10, 20, seed=5)
    head, lst = wl.vertex_adjacency(faces, pos.shape[1])
    q, idx = wl.make_mesh_queries(pos, 200, 4, seed=6)
    q = q.double().numpy()
    tri, bary, _ = orc.nearest_mesh_points(head, lst, faces, pos.double(), q, idx)
    gb = np.random.default_rng(2).normal(size=(3, 200))
    ana = orc.nearest_mesh_points_backward(faces, pos.double(), q, tri, gb)
    h = 1e-7
    fd = np.zeros_like(q)
    V = pos.double().numpy()
    F = faces.numpy()
    T = np.stack([V[:, F[0, tri]].T, V[:, F[1, tri]].T, V[:, F[2, tri]].T], 1)  # the selected faces, held fixed
    for c in range(3):
        e = np.zeros((3, 1))
        e[c] = h
        bp = orc.uv_of_triangle(T, (q + e).T)
        bm = orc.uv_of_triangle(T, (q - e).T)
        fd[c] = ((bp - bm).T * gb).sum(0) / (2 * h)
    ok = (np.abs(ana - fd) <= 1e-5 * (1 + np.abs(fd))).all(0)
    assert ok.mean() >= 0.98, ok.mean()


def test_nearest_mesh_points_without_candidates_reports_them():
    from diff_envshade_b200 import workloads as wl
    pos, faces = wl.make_sphere_mesh(4, 8, seed=1)
    head, lst = wl.vertex_adjacency(faces, pos.shape[1])
    q = torch.zeros(3, 5)
    idx = torch.full((5, 2), -1, dtype=torch.int64)
    idx[2, 1] = 0  # only query 2 has a candidate vertex
    tri, bary, missing = orc.nearest_mesh_points(head, lst, faces, pos, q, idx)
    assert missing == 4 and (tri[[0, 1, 3, 4]] == -1).all() and tri[2] >= 0
    assert (bary[:, [0, 1, 3, 4]] == 0).all()


def test_extract_bitfield_matches_reference_fixture_and_unpack():
    from diff_envshade_b200 import workloads as wl
    d = _load("etc_extract_bitfield.npz")
    nbit, i0, i1 = (int(x) for x in d["meta"])
    out = orc.extract_bitfield(d["bitfield"], nbit, i0, i1)
    assert np.array_equal(out, d["ref_out"])
    full = wl.unpack_bits(torch.from_numpy(d["bitfield"]), nbit).numpy()[i0:i1]
    assert np.array_equal(out, full.astype(np.float32))


def test_sample_envmap_matches_reference_fixture():
    d = _load("etc_envmap_sampling.npz")
    s = orc.sample_envmap(d["query_point"], d["envmap"])
    r = d["ref_sample"]
    assert (np.abs(s - r) / np.abs(r)).max() <= 1e-4


def test_sample_envmap_at_texel_centres_returns_the_texel_and_wraps_the_seam():
    H, W = 6, 10
    env = np.random.default_rng(3).random((3, H, W)) + 0.5
    rows, cols = np.meshgrid(np.arange(H), np.arange(W), indexing="ij")
    theta = (0.5 - (rows + 0.5) / H) * np.pi          # row 0 = top
    phi = (cols + 0.5) / W * 2 * np.pi
    dirs = np.stack([np.cos(theta) * np.cos(phi), np.sin(theta), np.cos(theta) * np.sin(phi)]).reshape(3, -1)
    s = orc.sample_envmap(dirs, env)
    assert np.allclose(s, env.reshape(3, -1), rtol=0, atol=1e-9)
    # on the seam (phi = 0) a lookup mixes the last and the first column half and half
    seam = np.array([[1.0], [0.0], [0.0]])
    mid = H // 2
    v = orc.sample_envmap(seam, env)[:, 0]
    expect = 0.5 * (0.5 * (env[:, mid - 1, 0] + env[:, mid - 1, W - 1]) + 0.5 * (env[:, mid, 0] + env[:, mid, W - 1]))
    assert np.allclose(v, expect, atol=1e-9)
