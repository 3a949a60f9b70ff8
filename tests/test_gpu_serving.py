"""Serving runtime (continuous batching) on the GPU.

* served results equal the plain single-request operators (and the FP64 oracle) within the suite's
  tolerances (conftest.py);
* a request's result is the same when it runs alone and when it shares ticks with 40 others of
  mixed sizes, env resolutions, visibility and forward/adjoint kinds (per-point outputs bit-exact;
  the env-map gradient, summed with FP64 atomics, within the gradient tolerance);
* admission respects a small HBM budget: everything completes and the arena never exceeds it.
"""
import numpy as np
import pytest
import torch

from conftest import assert_close_fwd, assert_close_grad

pytestmark = pytest.mark.gpu


def _mesh(seed, N_vertex=20000, N_face=40000, n_slots=64, p_on=0.7):
    g = torch.Generator().manual_seed(seed)
    from diff_envshade_b200 import workloads as wl
    faces = torch.randint(0, N_vertex, (3, N_face), generator=g).to(torch.int32)
    bits = torch.rand(N_vertex, n_slots * 32, generator=g) < p_on
    return faces.contiguous(), wl.pack_bits(bits)


def _points(P, seed, N_face):
    from diff_envshade_b200 import workloads as wl
    inp = wl.make_inputs(P, 4, 8, seed=seed)
    g = torch.Generator().manual_seed(seed + 7)
    tri = torch.randint(0, N_face, (P,), generator=g)
    e = -torch.log(torch.rand(3, P, generator=g).clamp_min(1e-12))
    bary = (e / e.sum(0, keepdim=True)).contiguous()
    return inp, tri, bary


def _plain(des, inp, tri, bary, faces, vis_bits, env, backward, use_vis):
    d = inp.to("cuda")
    envd, R = env.cuda(), torch.eye(3, device="cuda")
    base = (d.normal, d.view_dir, d.albedo, d.specular_albedo, d.roughness, envd, R)
    if use_vis:
        v = (faces.cuda(), tri.cuda(), bary.cuda(), vis_bits.cuda())
        sh, wh = des.bruteforce_specularvisibility_shader_forward2(*base, *v, True)
        g = des.bruteforce_specularvisibility_shader_backward2(d.grad_shading, d.grad_diffuse_shading, *base, *v,
                                                               True) if backward else None
    else:
        sh, wh = des.bruteforce_specular_shader_forward2(*base, True)
        g = des.bruteforce_specular_shader_backward2(d.grad_shading, d.grad_diffuse_shading, *base,
                                                     True) if backward else None
    out = {"shading": sh.cpu(), "diffuse_shading": wh.cpu()}
    if g is not None:
        for k, t in zip(("g_normal", "g_view_dir", "g_albedo", "g_specular_albedo", "g_roughness", "g_envmap"), g):
            out[k] = t.cpu()
    return out


def _submit(srv, inp, tri, bary, env_id, mesh_id, backward):
    return srv.submit(inp.normal, inp.view_dir, inp.albedo, inp.specular_albedo, inp.roughness, env_id=env_id,
                      mesh_id=mesh_id, nearest_triangle_id=tri if mesh_id >= 0 else None,
                      barycentric_coord=bary if mesh_id >= 0 else None, backward=backward,
                      grad_shading=inp.grad_shading, grad_diffuse_shading=inp.grad_diffuse_shading)


def _compare(got, want, tag, exact=False):
    for k, w in want.items():
        g = got[k].reshape(w.shape)
        if exact and not k == "g_envmap":
            assert torch.equal(g, w), f"{tag}:{k} differs"
        elif k in ("shading", "diffuse_shading"):
            assert_close_fwd(g, w, f"{tag}:{k}")
        else:
            assert_close_grad(g, w, f"{tag}:{k}")


@pytest.fixture(scope="module")
def setup():
    import diff_envshade_b200 as des
    from diff_envshade_b200.serving import Server
    g = torch.Generator().manual_seed(5)
    envs = {(16, 32): torch.exp(torch.randn(3, 16, 32, generator=g)),
            (32, 64): torch.exp(1.5 * torch.randn(3, 32, 64, generator=g))}
    faces, vis_bits = _mesh(11)
    srv = Server(device=0, hbm_budget_bytes=2 << 30, tick_us=100)
    env_ids = {k: srv.add_envmap(v) for k, v in envs.items()}
    mesh_id = srv.add_mesh(faces, vis_bits)
    yield des, srv, envs, env_ids, faces, vis_bits, mesh_id
    srv.close()


@pytest.mark.parametrize("P,res,use_vis,backward", [
    (5000, (16, 32), True, True),
    (777, (32, 64), False, True),
    (20001, (32, 64), True, False),
    (1, (16, 32), False, True),
])
def test_served_results_match_plain_operators(setup, P, res, use_vis, backward):
    des, srv, envs, env_ids, faces, vis_bits, mesh_id = setup
    inp, tri, bary = _points(P, seed=P, N_face=faces.shape[1])
    req = _submit(srv, inp, tri, bary, env_ids[res], mesh_id if use_vis else -1, backward)
    srv.drain(60)
    srv.poll()
    assert req.done is not None
    want = _plain(des, inp, tri, bary, faces, vis_bits, envs[res], backward, use_vis)
    _compare(req.outputs, want, f"P{P}")


def test_same_result_alone_and_in_the_mix(setup):
    des, srv, envs, env_ids, faces, vis_bits, mesh_id = setup
    inp, tri, bary = _points(70000, seed=70, N_face=faces.shape[1])
    alone = _submit(srv, inp, tri, bary, env_ids[(16, 32)], mesh_id, True)
    srv.drain(60)
    srv.poll()
    rng = np.random.default_rng(3)
    others = []
    for i in range(40):
        P = int(np.exp(rng.uniform(np.log(1000), np.log(120000))))
        o_inp, o_tri, o_bary = _points(P, seed=1000 + i, N_face=faces.shape[1])
        res = (16, 32) if rng.random() < 0.5 else (32, 64)
        others.append(_submit(srv, o_inp, o_tri, o_bary, env_ids[res], mesh_id if rng.random() < 0.5 else -1,
                              bool(rng.random() < 0.3)))
        if i == 20:
            mixed = _submit(srv, inp, tri, bary, env_ids[(16, 32)], mesh_id, True)
    srv.drain(120)
    done = srv.poll()
    assert mixed.done is not None and all(o.done is not None for o in others), len(done)
    assert mixed.status == 0 and all(o.status == 0 for o in others)
    _compare(mixed.outputs, alone.outputs, "mix-vs-alone", exact=True)
    assert_close_grad(mixed.outputs["g_envmap"], alone.outputs["g_envmap"], "mix-vs-alone:g_envmap")
    want = _plain(des, inp, tri, bary, faces, vis_bits, envs[(16, 32)], True, True)
    _compare(mixed.outputs, want, "mix-vs-plain")
    # the ticks really mixed requests: fewer ticks than requests, many items per tick
    st = srv.stats()
    assert st["device_error"] == 0


def test_admission_respects_hbm_budget():
    from diff_envshade_b200.serving import Server
    g = torch.Generator().manual_seed(8)
    budget = 48 << 20
    with Server(device=0, hbm_budget_bytes=budget, tick_us=100) as srv:
        env_id = srv.add_envmap(torch.exp(torch.randn(3, 16, 32, generator=g)))
        reqs = []
        for i in range(24):
            inp, tri, bary = _points(100000, seed=500 + i, N_face=10)
            reqs.append(_submit(srv, inp, tri, bary, env_id, -1, i % 3 == 0))
        srv.drain(120)
        srv.poll()
        st = srv.stats()
    assert all(r.done is not None for r in reqs)
    assert 0 < st["peak_arena_bytes"] <= budget
    # admission had to wait for memory: some request was admitted well after it was submitted
    assert max(r.done[1] - r.done[0] for r in reqs) > 0


def _outputs(P, H, W, where):
    kw = {"pinned": dict(pin_memory=True), "pageable": {}, "device": dict(device="cuda")}[where]
    o = {k: torch.empty(P, 3, **kw) for k in ("shading", "diffuse_shading", "g_normal", "g_view_dir", "g_albedo",
                                               "g_specular_albedo")}
    o["g_roughness"] = torch.empty(P, 1, **kw)
    o["g_envmap"] = torch.empty(3, H, W, **kw)
    return o


def test_outputs_in_place_and_staged_agree():
    """Outputs given as device memory or pinned host memory are stored in place by the batch
    kernel; pageable host outputs (and pinned ones of an ordered request) are staged in the arena
    and copied back.  Inputs of a request in input order are read in place (pinned host or device
    memory); an ordered request's inputs are uploaded.  Every placement, ordered or not, gives the
    same per-point results."""
    from diff_envshade_b200.serving import Server
    g = torch.Generator().manual_seed(21)
    faces, vis_bits = _mesh(12)
    env = torch.exp(torch.randn(3, 16, 32, generator=g))
    inp, tri, bary = _points(40000, seed=40, N_face=faces.shape[1])
    results = {}
    for order_min in (1 << 30, 16384):  # input order, then normal-direction order
        with Server(device=0, hbm_budget_bytes=1 << 30, tick_us=100, order_min_points=order_min) as srv:
            env_id = srv.add_envmap(env)
            mesh_id = srv.add_mesh(faces, vis_bits)
            for src, where in (("host", "pinned"), ("host", "pageable"), ("host", "device"), ("device", "pinned"),
                               ("device", "device")):
                d = inp.to("cuda") if src == "device" else inp
                t, b = (tri.cuda(), bary.cuda()) if src == "device" else (tri, bary)
                outs = _outputs(inp.P, 16, 32, where)
                req = srv.submit(d.normal, d.view_dir, d.albedo, d.specular_albedo, d.roughness,
                                 env_id=env_id, mesh_id=mesh_id, nearest_triangle_id=t, barycentric_coord=b,
                                 backward=True, grad_shading=d.grad_shading,
                                 grad_diffuse_shading=d.grad_diffuse_shading, outputs=outs)
                srv.drain(60)
                srv.poll()
                assert req.status == 0
                torch.cuda.synchronize()
                results[(order_min, src, where)] = {k: v.cpu() for k, v in outs.items()}
            assert srv.stats()["device_error"] == 0
    ref = results[(1 << 30, "host", "pageable")]
    for key, got in results.items():
        _compare(got, ref, f"{key}", exact=True)
        assert_close_grad(got["g_envmap"], ref["g_envmap"], f"{key}:g_envmap")


def test_requests_may_omit_outputs():
    """A request may leave outputs out (no diffuse shading, no view or roughness gradient): the
    outputs it names equal those of the same request naming all of them, whether they are stored
    in place (pinned host) or staged (pageable host), and nothing else is written."""
    from diff_envshade_b200.serving import Server
    g = torch.Generator().manual_seed(31)
    faces, vis_bits = _mesh(13)
    env = torch.exp(torch.randn(3, 16, 32, generator=g))
    inp, tri, bary = _points(9001, seed=90, N_face=faces.shape[1])
    keep = ("shading", "g_normal", "g_albedo", "g_specular_albedo", "g_envmap")
    with Server(device=0, hbm_budget_bytes=1 << 30, tick_us=100) as srv:
        env_id = srv.add_envmap(env)
        mesh_id = srv.add_mesh(faces, vis_bits)

        def run(outs):
            req = srv.submit(inp.normal, inp.view_dir, inp.albedo, inp.specular_albedo, inp.roughness,
                             env_id=env_id, mesh_id=mesh_id, nearest_triangle_id=tri, barycentric_coord=bary,
                             backward=True, grad_shading=inp.grad_shading,
                             grad_diffuse_shading=inp.grad_diffuse_shading, outputs=outs)
            srv.drain(60)
            srv.poll()
            assert req.status == 0
            return {k: v.clone() for k, v in outs.items()}

        full = run(_outputs(inp.P, 16, 32, "pinned"))
        for where in ("pinned", "pageable"):
            some = {k: v for k, v in _outputs(inp.P, 16, 32, where).items() if k in keep}
            got = run(some)
            assert set(got) == set(keep)
            for k in keep:
                if k == "g_envmap":
                    assert_close_grad(got[k], full[k], f"{where}:{k}")
                else:
                    assert torch.equal(got[k], full[k]), f"{where}:{k} differs"
        assert srv.stats()["device_error"] == 0



def test_malformed_and_oversized_requests():
    """Malformed requests are refused at submission -- an unknown env map or mesh, a mesh with too
    few visibility slots for the env map, no shading term -- and leave the server working; a
    request whose buffers could never fit the HBM budget finishes at once with DES_ERR_WORKSPACE
    (3) instead of waiting for memory forever."""
    import ctypes
    from diff_envshade_b200 import workloads as wl
    from diff_envshade_b200.serving import Server, _Request
    g = torch.Generator().manual_seed(41)
    faces16, vis16 = _mesh(14, n_slots=16)  # 512 visibility bits: enough for 16x32, not for 32x64
    inp, tri, bary = _points(1000, seed=41, N_face=faces16.shape[1])
    with Server(device=0, hbm_budget_bytes=8 << 20, tick_us=100) as srv:
        e16 = srv.add_envmap(torch.exp(torch.randn(3, 16, 32, generator=g)))
        e32 = srv.add_envmap(torch.exp(torch.randn(3, 32, 64, generator=g)))
        mesh = srv.add_mesh(faces16, vis16)
        for env_id, mesh_id in ((99, -1), (e16, 7), (e32, mesh)):
            with pytest.raises(RuntimeError):
                _submit(srv, inp, tri, bary, env_id, mesh_id, False)
        good = _submit(srv, inp, tri, bary, e16, mesh, False)
        # no shading term (flags 0), through the C ABI
        q = _Request()
        q.P, q.env_id, q.mesh_id, q.flags, q.backward = inp.P, e16, -1, 0, 0
        for k in ("normal", "view_dir", "albedo", "specular_albedo", "roughness"):
            setattr(q, k, good._inputs[k].data_ptr())
        q.shading = good.outputs["shading"].data_ptr()
        ticket = ctypes.c_int64()
        assert srv._L.des_server_submit(srv._h, ctypes.byref(q), ctypes.byref(ticket)) == 1
        # the outputs of 500k points alone take 12 MB of arena: more than the 8 MiB budget
        big = wl.make_inputs(500000, 4, 8, seed=42)
        huge = srv.submit(big.normal, big.view_dir, big.albedo, big.specular_albedo, big.roughness, env_id=e16)
        after = _submit(srv, inp, tri, bary, e16, mesh, True)
        srv.drain(60)
        srv.poll()
        assert good.status == 0 and after.status == 0
        assert huge.status == 3
        assert srv.stats()["device_error"] == 0


def test_scheduling_options_change_no_result():
    """Ranking by remaining work or by points x texels, and ordering large requests or not, change
    when tiles run, not what they compute: a mixed batch of requests gives bit-identical per-point
    outputs under every setting (env-map gradients within the gradient tolerance)."""
    from diff_envshade_b200.serving import Server
    g = torch.Generator().manual_seed(51)
    faces, vis_bits = _mesh(15)
    env = torch.exp(torch.randn(3, 16, 32, generator=g))
    reqs = [(_points(P, seed=500 + P, N_face=faces.shape[1]), bool(i % 2), i % 3 == 0)
            for i, P in enumerate((3000, 20000, 47000, 70001))]
    results = []
    for rank_by_size, order_min in ((False, 1 << 40), (True, 1 << 40), (False, 16384)):
        with Server(device=0, hbm_budget_bytes=1 << 30, tick_us=50, rank_by_size=rank_by_size,
                    order_min_points=order_min) as srv:
            env_id = srv.add_envmap(env)
            mesh_id = srv.add_mesh(faces, vis_bits)
            handles = [_submit(srv, inp, tri, bary, env_id, mesh_id if use_vis else -1, backward)
                       for (inp, tri, bary), use_vis, backward in reqs]
            srv.drain(60)
            srv.poll()
            assert all(h.status == 0 for h in handles)
            assert srv.stats()["device_error"] == 0
            results.append([{k: v.clone() for k, v in h.outputs.items()} for h in handles])
    for other in results[1:]:
        for i, (got, want) in enumerate(zip(other, results[0])):
            _compare(got, want, f"request {i}", exact=True)
