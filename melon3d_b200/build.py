"""Build libmelon3d_gpu.so for sm_100a from melon3d_b200/csrc.

Every translation unit is compiled by nvcc with
  -gencode arch=compute_100a,code=sm_100a   (B200 only)
  --fmad=false                               (no a*b+c contraction on the GPU)
  -Xcompiler -ffp-contract=off               (none in host code either)
so each float operation rounds exactly as the source writes it, which is what
makes the step bit-comparable with the reference built without contraction.
Division and square root stay IEEE (nvcc's defaults, no fast-math).

Usage:  python -m melon3d_b200.build [--force]
"""
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libmelon3d_gpu.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "--prec-div=true", "--prec-sqrt=true",
         "-ftz=false", "-Xcompiler", "-fPIC,-ffp-contract=off,-O2,-fvisibility=default",
         "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the GPU library cannot be built")


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def headers():
    out = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    inc = os.path.join(ROOT, "include")
    out += [os.path.join(inc, f) for f in os.listdir(inc) if f.endswith(".h")]
    return out


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, extra_flags=()):
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    cc = nvcc()
    hdrs = headers()
    jobs = []
    objs = []
    for src in sources():
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src[:-3] + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            jobs.append([cc] + ARCH + FLAGS + list(extra_flags) + ["-c", s, "-o", o])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    failed = []
    if jobs:
        with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
            for cmd, r in ex.map(run, jobs):
                if r.returncode != 0:
                    failed.append((cmd[-3], r.stdout + r.stderr))
                elif verbose and (r.stdout or r.stderr):
                    print(r.stdout + r.stderr)
    if failed:
        for src, log in failed:
            sys.stderr.write("---- %s\n%s\n" % (src, log))
        raise RuntimeError("nvcc failed for: " + ", ".join(s for s, _ in failed))
    if force or jobs or _stale(LIB, objs):
        cmd = [cc] + ARCH + ["-shared", "-cudart=static", "-o", LIB] + objs + ["-Xlinker", "-Bsymbolic"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
