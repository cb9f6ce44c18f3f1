"""Build the B200 extension in-tree: chameleon_b200/libchameleon_b200.so.

The library is plain CUDA C++ for sm_100a behind a C ABI (include/
chameleon_b200.h); it links only the CUDA runtime (statically).  Run as
``python -m chameleon_b200.build`` or through ``__graft_entry__.build()``.
"""
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libchameleon_b200.so")

SOURCES = ["control.cu", "executor.cu", "exec_f64.cu", "exec_f32.cu", "exec_f32tc.cu", "exec_tf32.cu", "tile_abi.cu", "mixed.cu", "batch.cu", "tc05.cu", "noalloc.cu", "serve.cu", "inverse.cu", "dispatch.cu", "batch_blas.cu", "gered.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path():
    p = shutil.which("nvcc")
    if p:
        return p
    cand = "/usr/local/cuda/bin/nvcc"
    if os.path.exists(cand):
        return cand
    raise RuntimeError("nvcc not found")


def build(verbose=False, extra=()):
    srcs = [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps.append(os.path.join(ROOT, "include", "chameleon_b200.h"))
    if os.path.exists(OUT) and all(os.path.getmtime(OUT) >= os.path.getmtime(d) for d in deps) and not extra:
        return OUT
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    nvcc = nvcc_path()
    common = [nvcc, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
              "-I", os.path.join(ROOT, "include"), "--expt-relaxed-constexpr", *extra]
    def compile_one(s):
        o = os.path.join(objdir, os.path.basename(s) + ".o")
        cmd = common + ["-c", s, "-o", o]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        return s, o, subprocess.run(cmd, capture_output=True, text=True)

    with ThreadPoolExecutor(max_workers=min(len(srcs), os.cpu_count() or 1)) as ex:
        results = list(ex.map(compile_one, srcs))
    for s, o, r in results:
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("nvcc failed on %s" % s)
        if verbose:
            sys.stderr.write(r.stderr)
        objs.append(o)
    cmd = [nvcc, *ARCH, "-shared", "-o", OUT + ".tmp", *objs, "-Xcompiler", "-fPIC"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
