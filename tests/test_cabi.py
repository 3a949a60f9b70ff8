"""CPU tests of the C ABI and the torch binding surface (no kernel launches)."""
import ctypes
import inspect

import pytest

import cabi


def test_library_exports_every_declared_symbol():
    L = cabi.lib()
    names = cabi.declared_functions()
    assert len(names) >= 16
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_status_strings_and_version():
    L = cabi.lib()
    assert L.des_abi_version() == 1
    for code in range(7):
        assert len(L.des_status_string(code)) > 0
    assert b"Channel number not supported" in L.des_status_string(cabi.DES_ERR_UNSUPPORTED)


def _host_args(**kw):
    a = cabi.ShadeArgs()
    a.P, a.H, a.W, a.C = 10, 16, 32, 3
    dummy = ctypes.c_void_p(0x1000)  # never dereferenced: validation fails before any launch
    for f in ("normal", "view_dir", "albedo", "specular_albedo", "roughness", "envmap", "light2obj_rotmat"):
        setattr(a, f, dummy)
    for k, v in kw.items():
        setattr(a, k, v)
    return a, dummy


@pytest.mark.parametrize("field,value,status", [
    ("C", 4, cabi.DES_ERR_UNSUPPORTED),
    ("C", 1, cabi.DES_ERR_UNSUPPORTED),
    ("P", -1, cabi.DES_ERR_INVALID_ARGUMENT),
    ("H", 0, cabi.DES_ERR_INVALID_ARGUMENT),
    ("W", -3, cabi.DES_ERR_INVALID_ARGUMENT),
    ("normal", None, cabi.DES_ERR_INVALID_ARGUMENT),
    ("envmap", None, cabi.DES_ERR_INVALID_ARGUMENT),
    ("roughness", None, cabi.DES_ERR_INVALID_ARGUMENT),
])
def test_forward_rejects_bad_arguments_before_launch(field, value, status):
    L = cabi.lib()
    a, dummy = _host_args(**{field: value})
    st = L.des_shade_forward(ctypes.byref(a), cabi.DES_DIFFUSE | cabi.DES_SPECULAR, dummy, None, dummy, 1 << 20,
                             None)
    assert st == status


def test_visibility_needs_enough_slots():
    L = cabi.lib()
    a, dummy = _host_args()
    a.visibility = dummy
    a.face_vertex_list = a.nearest_triangle_id = a.barycentric_coord = dummy
    a.N_face, a.N_vertex, a.N_slot = 4, 4, 15  # 16x32 texels need 16 slots
    st = L.des_shade_forward(ctypes.byref(a), cabi.DES_DIFFUSE, dummy, None, dummy, 1 << 20, None)
    assert st == cabi.DES_ERR_INVALID_ARGUMENT
    st = L.des_shade_backward(ctypes.byref(a), 8, dummy, None, dummy, None, None, None, None, None, dummy,
                              1 << 20, None)
    assert st == cabi.DES_ERR_INVALID_ARGUMENT  # unknown flag bit


def test_texel_table_rejects_bad_sizes():
    L = cabi.lib()
    assert L.des_texel_table(0, 32, ctypes.c_void_p(0x1000), ctypes.c_void_p(0x1000), None) == 1
    assert L.des_texel_table(16, 32, None, ctypes.c_void_p(0x1000), None) == 1


# argument counts of the reference operators (gsface_shader.h:1-118)
REFERENCE_ARITY = {
    "bruteforce_diffuse_shader_forward": 4,
    "bruteforce_diffuse_shader_backward": 5,
    "bruteforce_specular_shader_forward": 9,
    "bruteforce_specular_shader_backward": 10,
    "bruteforce_specular_shader_clamp_forward": 9,
    "bruteforce_specular_shader_clamp_backward": 10,
    "bruteforce_specular_shader_forward2": 8,
    "bruteforce_specular_shader_backward2": 10,
    "bruteforce_specularvisibility_shader_forward2": 12,
    "bruteforce_specularvisibility_shader_backward2": 14,
}


def test_torch_extension_keeps_reference_surface():
    import diff_envshade_b200 as des
    for name, n in REFERENCE_ARITY.items():
        fn = getattr(des, name)
        sig = fn.__doc__.splitlines()[0]  # pybind: "name(arg0: ..., ...) -> ..."
        args = sig[sig.index("(") + 1: sig.rindex(")")].split(" -> ")[0]
        count = args.count("arg")
        assert count == n, (name, sig)


def test_package_fails_loudly_without_native_code(tmp_path, monkeypatch):
    """The package has no CPU fallback: without its extension, import raises."""
    import shutil
    import subprocess
    import sys
    import os
    pkg = os.path.join(cabi.ROOT, "diff_envshade_b200")
    dst = tmp_path / "diff_envshade_b200"
    shutil.copytree(pkg, dst, ignore=shutil.ignore_patterns("*.so", "__pycache__"))
    r = subprocess.run([sys.executable, "-c", "import diff_envshade_b200"], cwd=tmp_path,
                       capture_output=True, text=True)
    assert r.returncode != 0 and "native extension not built" in r.stderr


def test_autograd_functions_have_reference_argument_order():
    import diff_envshade_b200 as des
    params = list(inspect.signature(des.SpecularVisibilityShade2.forward).parameters)[1:]
    assert params == ["normal", "view_dir", "albedo", "specular_albedo", "roughness", "envmap", "light2obj_rotmat",
                      "face_vertex_list", "nearest_triangle_id", "barycentric_coord", "visibility",
                      "enable_specular"]
