"""Build the native libraries in-tree (no JIT cache; the .so files travel with
the source tree).

  lib/libbemgpu.so       CUDA kernels + C ABI (include/bemgpu.h), sm_100a
  lib/libbem3_aw_qd2.so  C host library implementing include/bem3_aw_qd2.h,
                         calling libbemgpu.so
  lib/aw_d3qd2_bv_solver, lib/example1.out
                         the reference's own driver programs compiled
                         unchanged against libbem3_aw_qd2.so (only when the
                         reference sources are available at build time)
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib")
INCLUDE = os.path.join(ROOT, "include")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_SOURCES = ["bem_assemble.cu", "bem_solve.cu", "bem_lu.cu", "bem_capi.cu", "bem_static.cu", "bem_mixed.cu",
                "bem_server.cu", "bem_transform.cu", "bem_gmres.cu", "bem_tc.cu"]
HOST_SOURCES = ["host/aqd2_io.c", "host/aqd2_init.c", "host/aqd2_gpu.c"]
REFERENCE = os.environ.get("BEM_REFERENCE_DIR", "/root/reference")


def _run(cmd, cwd=None):
    r = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd))
    return r


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _deps(exts):
    out = []
    for base, _, files in os.walk(CSRC):
        out += [os.path.join(base, f) for f in files if f.endswith(exts)]
    out += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    return out


def build(force=False, verbose=False):
    os.makedirs(LIB, exist_ok=True)
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    gpu_so = os.path.join(LIB, "libbemgpu.so")
    if force or _stale(gpu_so, _deps((".cu", ".cuh", ".h"))):
        cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
               "-diag-suppress", "550,177", "-o", gpu_so] + [os.path.join(CSRC, s) for s in CUDA_SOURCES] + \
              []
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
    host_so = os.path.join(LIB, "libbem3_aw_qd2.so")
    if force or _stale(host_so, _deps((".c", ".h")) + [gpu_so]):
        cmd = ["gcc", "-O2", "-std=gnu11", "-fPIC", "-shared", "-Wall", "-Wno-unused-function", "-I" + INCLUDE,
               "-o", host_so] + [os.path.join(CSRC, s) for s in HOST_SOURCES] + \
              ["-L" + LIB, "-lbemgpu", "-Wl,-rpath,$ORIGIN", "-lm"]
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
    # the reference's driver programs, compiled unchanged against this library
    drivers = {"aw_d3qd2_bv_solver": os.path.join(REFERENCE, "d3qd2_src", "aw_d3qd2_bv_solver.c"),
               "example1.out": os.path.join(REFERENCE, "example1.c")}
    for name, src in drivers.items():
        exe = os.path.join(LIB, name)
        if os.path.exists(src) and (force or _stale(exe, [src, host_so])):
            # compiled from stdin so that its #include "bem3_aw_qd2.h" resolves to
            # include/ of this repository, not to the header next to the source
            with open(src) as f:
                r = subprocess.run(["gcc", "-O2", "-std=gnu11", "-w", "-I" + INCLUDE, "-x", "c", "-", "-o", exe,
                                    "-L" + LIB, "-lbem3_aw_qd2", "-Wl,-rpath,$ORIGIN", "-lm"], stdin=f,
                                   capture_output=True, text=True)
            if r.returncode != 0:
                sys.stderr.write(r.stderr)
                raise RuntimeError("failed to build " + name)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print("built into", LIB)
