"""Stream ordering of the operators' kernels.

The kernels of the shading path are launched with programmatic stream serialization: each may be
scheduled while its predecessor in the stream still runs, and waits for that predecessor to
complete before it reads memory.  These tests put a foreign kernel (a PyTorch elementwise kernel)
between the operators' kernels, writing an input the next kernel reads, and check that the results
are bit-identical to the same call on inputs prepared beforehand -- i.e. that no kernel of the path
read an input before the kernel that wrote it had finished.
"""
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def des():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import diff_envshade_b200
    return diff_envshade_b200


@pytest.fixture(scope="module")
def d():
    from diff_envshade_b200 import workloads as wl
    return wl.make_inputs(40000, 16, 32, 4711, vis_p=0.7).to("cuda")


def _base(d, normal=None):
    return (d.normal if normal is None else normal, d.view_dir, d.albedo, d.specular_albedo, d.roughness, d.envmap,
            d.light2obj_rotmat)


def _vis(d):
    return (d.face_vertex_list, d.nearest_triangle_id, d.barycentric_coord, d.visibility)


def test_forward_waits_for_the_kernel_that_writes_its_normals(des, d):
    # normals rotated by 90 degrees about z: a different ordering and different shading
    rot = d.normal[:, [1, 0, 2]].clone()
    rot[:, 0] = -rot[:, 0]
    want = des.bruteforce_specularvisibility_shader_forward2(*_base(d, rot), *_vis(d), True)
    torch.cuda.synchronize()
    buf = d.normal.clone()
    torch.cuda.synchronize()
    for _ in range(3):
        # a long foreign kernel ahead of the ordering kernels: the large copy, then the rotation
        big = torch.empty(64 << 20, device="cuda")
        big.fill_(1.0)
        buf.copy_(rot)
        got = des.bruteforce_specularvisibility_shader_forward2(*_base(d, buf), *_vis(d), True)
        torch.cuda.synchronize()
        for g, w in zip(got, want):
            assert torch.equal(g, w)
        buf.copy_(d.normal)


def test_adjoint_waits_for_the_kernel_that_writes_its_incoming_gradient(des, d):
    g2 = (2.0 * d.grad_shading).contiguous()
    want = des.bruteforce_specularvisibility_shader_backward2(g2, d.grad_diffuse_shading, *_base(d), *_vis(d), True)
    torch.cuda.synchronize()
    for _ in range(3):
        gs = d.grad_shading.clone()
        des.bruteforce_specularvisibility_shader_forward2(*_base(d), *_vis(d), True)
        gs.mul_(2.0)  # between the forward's kernels and the adjoint's, in the same stream
        got = des.bruteforce_specularvisibility_shader_backward2(gs, d.grad_diffuse_shading, *_base(d), *_vis(d),
                                                                 True)
        torch.cuda.synchronize()
        # per-point gradients are deterministic by construction; the env-map gradient's FP64 partials
        # depend on which CTA shaded which tile, so it is held to a relative 1e-6 of its scale
        for g, w in zip(got[:5], want[:5]):
            assert torch.equal(g, w)
        scale = float(want[5].abs().max())
        assert float((got[5] - want[5]).abs().max()) <= 1e-6 * scale


def test_next_call_waits_for_the_adjoints_env_reduction(des, d):
    # the env-gradient of one call feeds the env map of the next (as an optimiser step would)
    for _ in range(3):
        g = des.bruteforce_specularvisibility_shader_backward2(d.grad_shading, d.grad_diffuse_shading, *_base(d),
                                                               *_vis(d), True)
        env = d.envmap - 1e-3 * g[5]
        got = des.bruteforce_specularvisibility_shader_forward2(d.normal, d.view_dir, d.albedo, d.specular_albedo,
                                                                d.roughness, env, d.light2obj_rotmat, *_vis(d), True)
        torch.cuda.synchronize()
        # the same forward on the same env map, called once everything before it has finished
        want = des.bruteforce_specularvisibility_shader_forward2(d.normal, d.view_dir, d.albedo, d.specular_albedo,
                                                                 d.roughness, env.clone(), d.light2obj_rotmat, *_vis(d),
                                                                 True)
        torch.cuda.synchronize()
        for a, b in zip(got, want):
            assert torch.equal(a, b)


def test_graph_replay_matches_eager_calls(des, d):
    # the operator pair captured in a CUDA graph (its kernels become programmatic dependencies of
    # one another) and replayed on changed inputs gives what eager calls give on the same inputs
    normal = d.normal.clone()
    gsh = d.grad_shading.clone()

    def step():
        sh, wh = des.bruteforce_specularvisibility_shader_forward2(*_base(d, normal), *_vis(d), True)
        g = des.bruteforce_specularvisibility_shader_backward2(gsh, d.grad_diffuse_shading, *_base(d, normal),
                                                               *_vis(d), True)
        return [sh, wh] + list(g)

    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        for _ in range(2):
            step()
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        outs = step()
    for k in range(3):
        normal.copy_(torch.roll(d.normal, shifts=k + 1, dims=0))
        gsh.copy_(torch.roll(d.grad_shading, shifts=2 * k + 1, dims=0))
        torch.autograd.graph.increment_version(normal)
        graph.replay()
        torch.cuda.synchronize()
        want = des.bruteforce_specularvisibility_shader_forward2(*_base(d, normal.clone()), *_vis(d), True)
        wg = des.bruteforce_specularvisibility_shader_backward2(gsh.clone(), d.grad_diffuse_shading,
                                                                *_base(d, normal.clone()), *_vis(d), True)
        torch.cuda.synchronize()
        want = list(want) + list(wg)
        for got, w in zip(outs[:7], want[:7]):
            assert torch.equal(got, w)
        scale = float(want[7].abs().max())
        assert float((outs[7] - want[7]).abs().max()) <= 1e-6 * scale
    del graph
