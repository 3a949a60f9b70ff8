"""diff_envshade_b200 -- a B200-native differentiable environment-map shader.

Drop-in for the shading operators of zjumsj/diff_envshade (module ``_diff_envshade``):
the ten ``bruteforce_*`` functions exported here keep the reference's names, argument
order, tensor layouts and return order (reference bindings.cpp:6-19, gsface_shader.h:1-118).
They run hand-written sm_100a CUDA kernels through the C ABI in
``include/diff_envshade_b200.h``; there is no CPU fallback.

On top of the reference surface this package adds ``torch.autograd.Function`` wrappers
(the reference ships none) and the ``shade`` convenience function.

Build the native parts with ``python diff_envshade_b200/build.py``.
"""
import os as _os

_HERE = _os.path.dirname(_os.path.abspath(__file__))

try:
    from . import _C  # noqa: F401  (torch extension; loads libdes_b200.so)
except ImportError as _e:  # fail loudly: the CUDA path is the product, there is no fallback
    raise ImportError(
        "diff_envshade_b200: native extension not built or not loadable "
        f"({_e}). Build it with `python {_os.path.join(_HERE, 'build.py')}`."
    ) from _e

from ._C import (  # noqa: E402,F401  reference operator surface
    bruteforce_diffuse_shader_forward,
    bruteforce_diffuse_shader_backward,
    bruteforce_specular_shader_forward,
    bruteforce_specular_shader_backward,
    bruteforce_specular_shader_clamp_forward,
    bruteforce_specular_shader_clamp_backward,
    bruteforce_specular_shader_forward2,
    bruteforce_specular_shader_backward2,
    bruteforce_specularvisibility_shader_forward2,
    bruteforce_specularvisibility_shader_backward2,
    get_nearest_mesh_points_forward,
    get_nearest_mesh_points_backward,
    get_uv_of_triangle_forward,
    get_uv_of_triangle_backward,
    extract_bitfield_forward,
    sample_envmap_forward,
    blur_envmap_forward,
    texel_table,
    workspace_bytes,
    set_timing_events,
    kernel_launches,
    relight_multienv,
)
from .autograd import (  # noqa: E402,F401
    DiffuseShade,
    SpecularShade,
    SpecularShadeClamp,
    SpecularShade2,
    SpecularVisibilityShade2,
    shade,
)

NATIVE_LIBRARIES = (
    _os.path.join(_HERE, "libdes_b200.so"),
    _C.__file__,
)

__all__ = [
    "bruteforce_diffuse_shader_forward",
    "bruteforce_diffuse_shader_backward",
    "bruteforce_specular_shader_forward",
    "bruteforce_specular_shader_backward",
    "bruteforce_specular_shader_clamp_forward",
    "bruteforce_specular_shader_clamp_backward",
    "bruteforce_specular_shader_forward2",
    "bruteforce_specular_shader_backward2",
    "bruteforce_specularvisibility_shader_forward2",
    "bruteforce_specularvisibility_shader_backward2",
    "texel_table",
    "workspace_bytes",
    "relight_multienv",
    "DiffuseShade",
    "SpecularShade",
    "SpecularShadeClamp",
    "SpecularShade2",
    "SpecularVisibilityShade2",
    "shade",
]
