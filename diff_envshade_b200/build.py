"""In-tree build of the native parts of diff_envshade_b200.

Products (all next to this file, git-ignored, shipped with the source tree):
  libdes_b200.so                    CUDA kernels + C ABI (include/diff_envshade_b200.h), sm_100a
  _C<EXT_SUFFIX>                    torch extension with the reference's operator surface,
                                    linked against libdes_b200.so (rpath $ORIGIN)

Each product is rebuilt only when one of its sources is newer than it.  The compile flags
keep nvcc's defaults for floating point (-fmad=true, IEEE division, no fast-math), which the
bit-exact texel table depends on.

Usage:  python diff_envshade_b200/build.py [--force] [--verbose] [--ptxas]
"""
import argparse
import glob
import os
import subprocess
import sys
import sysconfig

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CUDA_LIB = os.path.join(PKG, "libdes_b200.so")
CUDA_SOURCES = ["des_shade.cu", "des_capi.cu"]
EXTRA_CUDA_SOURCES = ["des_noalloc.cu", "des_multienv.cu", "des_serve.cu", "des_mesh.cu", "des_envtools.cu"]  # built when present


def ext_path():
    return os.path.join(PKG, "_C" + sysconfig.get_config_var("EXT_SUFFIX"))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd, verbose):
    if verbose:
        print("+", " ".join(cmd), flush=True)
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout)
        raise RuntimeError(f"build step failed ({r.returncode}): {' '.join(cmd[:3])} ...")
    if verbose and r.stdout.strip():
        print(r.stdout)
    return r.stdout


def cuda_sources():
    srcs = [os.path.join(CSRC, s) for s in CUDA_SOURCES]
    srcs += [os.path.join(CSRC, s) for s in EXTRA_CUDA_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    return srcs


def build_cuda_lib(force=False, verbose=False, ptxas_verbose=False):
    srcs = cuda_sources()
    deps = srcs + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + [
        os.path.join(INCLUDE, "diff_envshade_b200.h")]
    if not force and not _stale(CUDA_LIB, deps):
        return CUDA_LIB
    cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           f"-I{INCLUDE}", f"-I{CSRC}", "-o", CUDA_LIB + ".tmp", *srcs]
    if ptxas_verbose:
        cmd.insert(1, "-Xptxas=-v")
    out = _run(cmd, verbose)
    os.replace(CUDA_LIB + ".tmp", CUDA_LIB)
    return out if ptxas_verbose else CUDA_LIB


def build_torch_ext(force=False, verbose=False):
    import torch
    import torch.utils.cpp_extension as ce

    target = ext_path()
    src = os.path.join(CSRC, "torch_binding.cpp")
    deps = [src, os.path.join(INCLUDE, "diff_envshade_b200.h"), CUDA_LIB]
    if not force and not _stale(target, deps):
        return target
    incs = ce.include_paths(device_type="cuda") + [sysconfig.get_paths()["include"], INCLUDE]
    libdirs = ce.library_paths()
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    cmd = ["g++", "-shared", "-fPIC", "-O2", "-std=c++17", src, "-o", target + ".tmp",
           "-DTORCH_EXTENSION_NAME=_C", "-DTORCH_API_INCLUDE_EXTENSION_H", f"-D_GLIBCXX_USE_CXX11_ABI={abi}",
           *[f"-I{p}" for p in incs], *[f"-L{p}" for p in libdirs], f"-L{CUDA_HOME}/lib64", f"-L{PKG}",
           "-ldes_b200", "-lc10", "-lc10_cuda", "-ltorch", "-ltorch_cpu", "-ltorch_cuda", "-ltorch_python",
           "-lcudart", "-Wl,-rpath,$ORIGIN", *[f"-Wl,-rpath,{p}" for p in libdirs]]
    _run(cmd, verbose)
    os.replace(target + ".tmp", target)
    return target


def build(force=False, verbose=False):
    build_cuda_lib(force=force, verbose=verbose)
    build_torch_ext(force=force, verbose=verbose)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print ptxas register/spill report")
    a = ap.parse_args()
    if a.ptxas:
        print(build_cuda_lib(force=True, verbose=a.verbose, ptxas_verbose=True))
    build(force=a.force, verbose=a.verbose)
    print("built", CUDA_LIB, ext_path())


if __name__ == "__main__":
    main()
