"""Build libecgpu.so (the C-ABI CUDA library) in-tree for sm_100a.

    python elemco.jl_b200/build.py [-v] [--force]

Objects go to elemco.jl_b200/_build/, the shared library to
elemco.jl_b200/ecgpu/libecgpu.so.  Sources are recompiled when they, or any
header in csrc/ or include/, are newer than their object.
"""
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "ecgpu", "libecgpu.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _flags():
    return ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3",
            "-I" + CSRC, "-I" + os.path.join(ROOT, "include")] + ARCH


def _newest_header():
    hs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def build(verbose=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    hdr = _newest_header()
    cc = nvcc()
    jobs = []
    objs = []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s) + ".o")
        objs.append(o)
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr):
            cmd = [cc] + _flags() + ["-c", s, "-o", o]
            if s.endswith(".cu"):
                cmd += ["-Xptxas", "-v"] if verbose else []
            else:
                cmd += ["-x", "cu"] if False else []
            jobs.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    ok = True
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for cmd, r in ex.map(run, jobs):
            if verbose or r.returncode:
                sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
            ok &= r.returncode == 0
    if not ok:
        raise RuntimeError("libecgpu compilation failed")
    if force or jobs or not os.path.exists(OUT):
        cmd = [cc] + ARCH + ["-shared", "-cudart", "static", "-o", OUT] + objs + ["-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
            raise RuntimeError("libecgpu link failed")
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="--force" in sys.argv))
