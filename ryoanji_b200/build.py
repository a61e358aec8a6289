"""Build the ryoanji-b200 CUDA library in-tree: ryoanji_b200/libryoanji_b200.so (sm_100a).

    python -m ryoanji_b200.build            # incremental
    python -m ryoanji_b200.build --force    # rebuild everything

nvcc compiles each translation unit for sm_100a only (no PTX for other targets) and links them into one shared
library with the C ABI of include/ryoanji_b200.h; the CUDA runtime is linked statically.
"""
from __future__ import annotations

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
LIB = os.path.join(HERE, "libryoanji_b200.so")

SOURCES = ["sfc.cu", "sort.cu", "octree.cu", "upsweep.cu", "traverse.cu", "traverse64.cu", "ewald.cu", "direct.cu", "probe.cu", "batch.cu", "engine.cu", "groups.cu", "let.cu",
           "capi.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-ffp-contract=off",
                "-Xcompiler", "-fvisibility=hidden", f"-I{os.path.join(ROOT, 'include')}"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _deps() -> list[str]:
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp")) + [
        os.path.join(ROOT, "include", "ryoanji_b200.h")]


def _digest(inputs: list[str], cmd: list[str]) -> str:
    """hash of the inputs' contents and the compile command"""
    import hashlib
    h = hashlib.sha256(" ".join(cmd).encode())
    for path in sorted(inputs):
        with open(path, "rb") as f:
            h.update(path.encode() + b"\0" + f.read())
    return h.hexdigest()


def _stale(target: str, inputs: list[str], cmd: list[str]) -> bool:
    """an object is rebuilt unless it exists and was compiled from exactly these contents with this command (file
    times are not enough: a source edited while its compile runs would leave an object newer than the edit)"""
    stamp = target + ".sha256"
    if not (os.path.exists(target) and os.path.exists(stamp)):
        return True
    with open(stamp) as f:
        return f.read().strip() != _digest(inputs, cmd)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    cc = nvcc()
    deps = _deps()
    jobs = []
    objs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(obj)
        cmd = [cc, *FLAGS, "-c", path, "-o", obj]
        if force or _stale(obj, [path] + deps, cmd):
            if ptxas_info:
                cmd += ["-Xptxas", "-v"]
            # the digest is taken before compiling: an edit during the compile makes the next build redo it
            jobs.append((src, cmd, obj, _digest([path] + deps, [cc, *FLAGS, "-c", path, "-o", obj])))

    def run(job):
        src, cmd, obj, digest = job
        stamp = obj + ".sha256"
        if os.path.exists(stamp):
            os.remove(stamp)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode == 0:
            with open(stamp, "w") as f:
                f.write(digest)
        return src, r

    failed = []
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        for src, r in ex.map(run, jobs):
            if verbose or r.returncode != 0 or ptxas_info:
                sys.stderr.write(r.stdout + r.stderr)
            if r.returncode != 0:
                failed.append(src)
    if failed:
        raise RuntimeError(f"nvcc failed for {failed}")
    if force or jobs or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [cc, *ARCH, "-shared", "-o", LIB, *objs, "-Xcompiler", "-fPIC"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
