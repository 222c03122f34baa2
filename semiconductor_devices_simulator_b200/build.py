"""Build the solver library in-tree: every CUDA / C++ source of csrc/ compiled for
sm_100a with nvcc and linked into lib/libsemisim_b200.so (static CUDA runtime, only the
api3_* ABI and the b200x_* test hooks exported).

    python -m semiconductor_devices_simulator_b200.build [--jobs N]
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib", "libsemisim_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def compile_one(src, extra):
    out = os.path.join(OBJ, src + ".o")
    path = os.path.join(CSRC, src)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))] + [path]
    if os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(d) for d in deps):
        return out, ""
    cmd = [nvcc(), "-c", path, "-o", out] + COMMON + extra
    if src.endswith(".cu"):
        cmd += ARCH + ["-Xptxas", "-v"] if os.environ.get("SEMISIM_PTXAS_V") else ARCH
    else:
        cmd += ["-x", "cu"] + ARCH
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return out, r.stderr


def build(jobs=None, verbose=False, extra=()):
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, len(srcs))) as ex:
        res = list(ex.map(lambda s: compile_one(s, list(extra)), srcs))
    if verbose:
        for _, log in res:
            if log.strip():
                print(log)
    objs = [o for o, _ in res]
    cmd = [nvcc(), "-shared", "-o", LIB] + objs + ARCH + [
        "-cudart", "static", "-Xlinker", "--version-script=" + os.path.join(CSRC, "exports.map"),
        "-Xlinker", "-Bsymbolic"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    print(build(a.jobs, a.v))
