"""Build libpdgpu.so in-tree for sm_100a (B200).

    python pd.arcus_b200/build.py [--force] [--verbose-ptxas]

Compiles every csrc/*.cu with nvcc (-gencode arch=compute_100a,code=sm_100a)
and links them into pdgpu/_lib/libpdgpu.so with the CUDA runtime linked
statically, so the library travels with the source tree.
"""
import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(ROOT, "_build", "pdgpu")
OUT = os.path.join(HERE, "pdgpu", "_lib", "libpdgpu.so")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
         "-I", os.path.join(ROOT, "include"), "-I", CSRC]
# per-file flags: the LCPO term's FP64 arithmetic follows the reference's
# rounding, so it is compiled without fused multiply-adds; the evaluation
# kernel's FP32 pair arithmetic never meets subnormal values, so it is
# compiled with them flushed (no subnormal fix-ups around the MUFU ops)
FILE_FLAGS = {"lcpo.cu": ["-fmad=false"], "evaltiles.cu": ["-ftz=true"]}


def _stale(src, obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in [src] + deps)


def build(force=False, ptxas_verbose=False, quiet=False):
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    deps = sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + [os.path.join(ROOT, "include", "pdgpu.h")]
    jobs = []
    for s in srcs:
        o = os.path.join(OBJ, os.path.basename(s)[:-3] + ".o")
        if force or _stale(s, o, deps):
            cmd = [NVCC] + ARCH + FLAGS + FILE_FLAGS.get(os.path.basename(s), []) + \
                (["-Xptxas", "-v"] if ptxas_verbose else []) + ["-c", s, "-o", o]
            jobs.append((s, cmd))

    def run(job):
        s, cmd = job
        r = subprocess.run(cmd, capture_output=True, text=True)
        return s, r

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for s, r in ex.map(run, jobs):
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise RuntimeError("nvcc failed on %s" % s)
            if ptxas_verbose:
                sys.stderr.write(r.stderr)
    objs = [os.path.join(OBJ, os.path.basename(s)[:-3] + ".o") for s in srcs]
    if force or jobs or not os.path.exists(OUT):
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-Xcompiler", "-fPIC", "-o", OUT] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
    if not quiet:
        print("built", OUT)
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args()
    build(a.force, a.verbose_ptxas)
