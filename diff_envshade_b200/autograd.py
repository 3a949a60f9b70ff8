"""``torch.autograd.Function`` wrappers over the reference-surface operators.

The reference extension ships no autograd glue (callers wrap ``_diff_envshade`` themselves);
these Functions are the wrapping a caller of the reference would write: ``forward`` calls the
``*_forward*`` operator and saves its inputs, ``backward`` calls the matching ``*_backward*``
operator with the incoming gradients (zeros for an output that received none).  Light rotation,
mesh indices, barycentrics and visibility receive no gradient, as in the reference.

The backward operators are native kernels that autograd cannot trace, so every ``backward`` is
``once_differentiable``: asking for second derivatives (``create_graph=True``) raises instead of
silently returning zeros.
"""
import torch
from torch.autograd.function import once_differentiable

from . import _C


def _grad_or_zeros(g, like):
    return torch.zeros_like(like) if g is None else g.contiguous()


class DiffuseShade(torch.autograd.Function):
    """Lambert-only shading: bruteforce_diffuse_shader_{forward,backward}."""

    @staticmethod
    def forward(ctx, normal, albedo, envmap, light2obj_rotmat):
        shading = _C.bruteforce_diffuse_shader_forward(normal, albedo, envmap, light2obj_rotmat)
        ctx.save_for_backward(normal, albedo, envmap, light2obj_rotmat)
        return shading

    @staticmethod
    @once_differentiable
    def backward(ctx, g_shading):
        normal, albedo, envmap, rot = ctx.saved_tensors
        gn, ga, ge = _C.bruteforce_diffuse_shader_backward(_grad_or_zeros(g_shading, albedo), normal, albedo,
                                                           envmap, rot)
        return gn, ga, ge, None


class _SpecularV1(torch.autograd.Function):
    _fwd = None
    _bwd = None

    @classmethod
    def _forward(cls, ctx, normal, view_dir, albedo, specular_albedo, roughness, envmap, light2obj_rotmat,
                 enable_diffuse, enable_specular):
        shading = cls._fwd(normal, view_dir, albedo, specular_albedo, roughness, envmap, light2obj_rotmat,
                           enable_diffuse, enable_specular)
        ctx.save_for_backward(normal, view_dir, albedo, specular_albedo, roughness, envmap, light2obj_rotmat)
        ctx.flags = (enable_diffuse, enable_specular)
        return shading

    @classmethod
    def _backward(cls, ctx, g_shading):
        normal, view, albedo, spec, rough, envmap, rot = ctx.saved_tensors
        gn, gv, ga, gs, gr, ge = cls._bwd(_grad_or_zeros(g_shading, albedo), normal, view, albedo, spec, rough,
                                          envmap, rot, *ctx.flags)
        return gn, gv, ga, gs, gr.view_as(rough), ge, None, None, None


class SpecularShade(_SpecularV1):
    """Diffuse + GGX, shading output only: bruteforce_specular_shader_{forward,backward}."""

    @staticmethod
    def forward(ctx, normal, view_dir, albedo, specular_albedo, roughness, envmap, light2obj_rotmat,
                enable_diffuse=True, enable_specular=True):
        return SpecularShade._forward(ctx, normal, view_dir, albedo, specular_albedo, roughness, envmap,
                                      light2obj_rotmat, enable_diffuse, enable_specular)

    @staticmethod
    @once_differentiable
    def backward(ctx, g_shading):
        return SpecularShade._backward(ctx, g_shading)


SpecularShade._fwd = staticmethod(_C.bruteforce_specular_shader_forward)
SpecularShade._bwd = staticmethod(_C.bruteforce_specular_shader_backward)


class SpecularShadeClamp(_SpecularV1):
    """As SpecularShade, with points facing away from the viewer (n.v <= 0) shaded to zero:
    bruteforce_specular_shader_clamp_{forward,backward}."""

    @staticmethod
    def forward(ctx, normal, view_dir, albedo, specular_albedo, roughness, envmap, light2obj_rotmat,
                enable_diffuse=True, enable_specular=True):
        return SpecularShadeClamp._forward(ctx, normal, view_dir, albedo, specular_albedo, roughness, envmap,
                                           light2obj_rotmat, enable_diffuse, enable_specular)

    @staticmethod
    @once_differentiable
    def backward(ctx, g_shading):
        return SpecularShadeClamp._backward(ctx, g_shading)


SpecularShadeClamp._fwd = staticmethod(_C.bruteforce_specular_shader_clamp_forward)
SpecularShadeClamp._bwd = staticmethod(_C.bruteforce_specular_shader_clamp_backward)


class SpecularShade2(torch.autograd.Function):
    """Diffuse + optional GGX with the white-diffuse second output:
    bruteforce_specular_shader_{forward2,backward2}.  Returns (shading, diffuse_shading)."""

    @staticmethod
    def forward(ctx, normal, view_dir, albedo, specular_albedo, roughness, envmap, light2obj_rotmat,
                enable_specular=True):
        shading, white = _C.bruteforce_specular_shader_forward2(normal, view_dir, albedo, specular_albedo,
                                                                roughness, envmap, light2obj_rotmat,
                                                                enable_specular)
        ctx.save_for_backward(normal, view_dir, albedo, specular_albedo, roughness, envmap, light2obj_rotmat)
        ctx.enable_specular = enable_specular
        return shading, white

    @staticmethod
    @once_differentiable
    def backward(ctx, g_shading, g_white):
        normal, view, albedo, spec, rough, envmap, rot = ctx.saved_tensors
        gn, gv, ga, gs, gr, ge = _C.bruteforce_specular_shader_backward2(
            _grad_or_zeros(g_shading, albedo), _grad_or_zeros(g_white, albedo), normal, view, albedo, spec, rough,
            envmap, rot, ctx.enable_specular)
        return gn, gv, ga, gs, gr.view_as(rough), ge, None, None


class SpecularVisibilityShade2(torch.autograd.Function):
    """SpecularShade2 with per-texel visibility interpolated over each point's nearest triangle:
    bruteforce_specularvisibility_shader_{forward2,backward2}."""

    @staticmethod
    def forward(ctx, normal, view_dir, albedo, specular_albedo, roughness, envmap, light2obj_rotmat,
                face_vertex_list, nearest_triangle_id, barycentric_coord, visibility, enable_specular=True):
        shading, white = _C.bruteforce_specularvisibility_shader_forward2(
            normal, view_dir, albedo, specular_albedo, roughness, envmap, light2obj_rotmat, face_vertex_list,
            nearest_triangle_id, barycentric_coord, visibility, enable_specular)
        ctx.save_for_backward(normal, view_dir, albedo, specular_albedo, roughness, envmap, light2obj_rotmat,
                              face_vertex_list, nearest_triangle_id, barycentric_coord, visibility)
        ctx.enable_specular = enable_specular
        return shading, white

    @staticmethod
    @once_differentiable
    def backward(ctx, g_shading, g_white):
        (normal, view, albedo, spec, rough, envmap, rot, faces, tri, bary, vis) = ctx.saved_tensors
        gn, gv, ga, gs, gr, ge = _C.bruteforce_specularvisibility_shader_backward2(
            _grad_or_zeros(g_shading, albedo), _grad_or_zeros(g_white, albedo), normal, view, albedo, spec, rough,
            envmap, rot, faces, tri, bary, vis, ctx.enable_specular)
        return gn, gv, ga, gs, gr.view_as(rough), ge, None, None, None, None, None, None


def shade(normal, view_dir, albedo, specular_albedo, roughness, envmap, light2obj_rotmat=None, visibility=None,
          enable_specular=True):
    """Differentiable shading of P points under a lat-long env map.

    ``visibility`` is ``None`` or the tuple ``(face_vertex_list, nearest_triangle_id,
    barycentric_coord, visibility_bits)`` in the reference's layouts.  Returns
    ``(shading, diffuse_shading)``, each ``P x 3``.
    """
    if light2obj_rotmat is None:
        light2obj_rotmat = torch.eye(3, device=normal.device, dtype=normal.dtype)
    if visibility is None:
        return SpecularShade2.apply(normal, view_dir, albedo, specular_albedo, roughness, envmap,
                                    light2obj_rotmat, enable_specular)
    faces, tri, bary, bits = visibility
    return SpecularVisibilityShade2.apply(normal, view_dir, albedo, specular_albedo, roughness, envmap,
                                          light2obj_rotmat, faces, tri, bary, bits, enable_specular)
