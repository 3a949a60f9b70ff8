"""Build the reference CUDA extension (zjumsj/diff_envshade) from its own sources.

Test infrastructure only: the resulting ``oracle/_ref/_diff_envshade*.so`` is the
reference implementation used by the GPU parity tests and by the fixture generator
under ``tests/golden/``.  It is never imported by the product package.

The recipe compiles the reference's three translation units (``etc.cu``,
``bruteforce_shader.cu``, ``bindings.cpp``) where they lie, with nvcc/g++ invoked
directly (the reference's ``setup.py`` is not run), for sm_100 -- the flags mirror
what a stock ``TORCH_CUDA_ARCH_LIST=10.0`` build of that setup.py would pass, so the
kernels are the reference's default-flag (no fast-math, ``-fmad=true``) code.

Usage:  python oracle/build_ref.py [--src /path/to/reference] [-j N]
The source directory is ``--src``, else the environment variable ``DES_REFERENCE_SRC``; with
neither, or when the directory holds no ``bruteforce_shader.cu``, nothing is built and the script
exits 0 (the GPU tests that need the reference then skip).
Outputs go only to ``oracle/_ref/`` (git-ignored; it travels with the repo snapshot).
"""
import argparse
import os
import subprocess
import sys
import sysconfig
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")


def _torch_paths():
    import torch
    import torch.utils.cpp_extension as ce
    inc = ce.include_paths(device_type="cuda")
    lib = ce.library_paths()
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    return inc, lib, abi


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--src", default=os.environ.get("DES_REFERENCE_SRC"))
    ap.add_argument("-j", type=int, default=3)
    args = ap.parse_args()
    if not args.src:
        print("no reference source directory (--src or DES_REFERENCE_SRC); nothing built")
        return 0
    src = os.path.abspath(args.src)
    if not os.path.isfile(os.path.join(src, "bruteforce_shader.cu")):
        print(f"reference sources not found under {src}; nothing built")
        return 0
    os.makedirs(OUT, exist_ok=True)
    inc, lib, abi = _torch_paths()
    py_inc = sysconfig.get_paths()["include"]
    ext = sysconfig.get_config_var("EXT_SUFFIX")
    common_defs = [
        "-DTORCH_EXTENSION_NAME=_diff_envshade",
        "-DTORCH_API_INCLUDE_EXTENSION_H",
        f"-D_GLIBCXX_USE_CXX11_ABI={abi}",
    ]
    incs = [f"-I{p}" for p in inc] + [f"-I{py_inc}", f"-I{src}"]
    nvcc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    jobs = []
    for cu in ("etc.cu", "bruteforce_shader.cu"):
        obj = os.path.join(OUT, cu.replace(".cu", ".o"))
        cmd = [nvcc, "-c", os.path.join(src, cu), "-o", obj, "-O3", "-std=c++17",
               "-gencode", "arch=compute_100,code=sm_100",
               "--expt-relaxed-constexpr", "--compiler-options", "-fPIC",
               "-D__CUDA_NO_HALF_OPERATORS__", "-D__CUDA_NO_HALF_CONVERSIONS__",
               "-D__CUDA_NO_BFLOAT16_CONVERSIONS__", "-D__CUDA_NO_HALF2_OPERATORS__",
               ] + common_defs + incs
        jobs.append((obj, cmd))
    obj = os.path.join(OUT, "bindings.o")
    jobs.append((obj, ["g++", "-c", os.path.join(src, "bindings.cpp"), "-o", obj, "-O3",
                       "-std=c++17", "-fPIC"] + common_defs + incs))

    def run(job):
        o, c = job
        print("+", " ".join(c), flush=True)
        subprocess.check_call(c)
        return o

    with ThreadPoolExecutor(args.j) as ex:
        objs = list(ex.map(run, jobs))
    so = os.path.join(OUT, "_diff_envshade" + ext)
    link = ["g++", "-shared", "-o", so] + objs + [f"-L{p}" for p in lib] + [
        "-L/usr/local/cuda/lib64", "-lc10", "-lc10_cuda", "-ltorch", "-ltorch_cpu",
        "-ltorch_cuda", "-ltorch_python", "-lcudart"] + [f"-Wl,-rpath,{p}" for p in lib]
    print("+", " ".join(link), flush=True)
    subprocess.check_call(link)
    print("built", so)
    return 0


if __name__ == "__main__":
    sys.exit(main())
