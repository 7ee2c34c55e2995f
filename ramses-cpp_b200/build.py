"""Build librgpu.so (the B200 Godunov level step) in-tree with nvcc.

    python ramses-cpp_b200/build.py [--force] [--verbose]

Every translation unit is compiled for sm_100a only, with -fmad=false: the
reference CPU code is built by g++ for baseline x86-64, which has no FMA, so
contracting a*b+c on the GPU would change the last bit of the results.
"""
import argparse
import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "librgpu.so"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC,-O2",
                "--expt-relaxed-constexpr", f"-I{ROOT / 'include'}"]
SOURCES = ["rg_api.cu", "rg_plan.cu", "rg_step.cu", "rg_face.cu", "rg_face_1d.cu", "rg_face_3d.cu",
           "rg_noalloc.cu", "rg_exact.cu", "rg_mlp.cu", "rg_host_level.cu",
           "rg_lattice.cu", "rg_output.cu", "rg_tree.cu", "rg_amr.cu", "rg_measure.cu"]


def _newer(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force=False, verbose=False, ptxas_info=False) -> Path:
    BUILD.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + [ROOT / "include" / "rgpu.h"]
    objs = []
    jobs = []
    for src in SOURCES:
        obj = BUILD / (Path(src).stem + ".o")
        objs.append(obj)
        if force or _newer(obj, [CSRC / src] + headers):
            cmd = [NVCC] + FLAGS + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", str(CSRC / src), "-o", str(obj)]
            jobs.append(cmd)
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        for cmd, res in zip(jobs, ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), jobs)):
            if verbose or res.returncode != 0 or ptxas_info:
                sys.stdout.write(" ".join(cmd) + "\n" + res.stdout + res.stderr)
            if res.returncode != 0:
                raise RuntimeError(f"nvcc failed: {cmd[-3]}")
    if force or jobs or _newer(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", str(LIB)] + [str(o) for o in objs] + ["-lcudart"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            sys.stdout.write(res.stdout + res.stderr)
            raise RuntimeError("link of librgpu.so failed")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose, a.ptxas_info))
