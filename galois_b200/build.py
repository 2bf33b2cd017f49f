"""Build libgb.so (CUDA sm_100a kernels + C ABI) in-tree.

Usage:  python galois_b200/build.py [--jobs N] [--force]   (run as a file: importing
        the package needs the built library)

Every .cu under csrc/ is compiled with
    nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo -O3
and every .cpp with g++ -O3 -fopenmp; the objects are linked into
galois_b200/libgb.so against the static CUDA runtime.  Objects live in
galois_b200/_build/ and are rebuilt when a source or header is newer.
The command-line programs in apps/ (bfs-gpu, sssp-gpu, cc-gpu, pagerank-gpu,
bc-gpu, operator-example) are then linked against libgb.so into apps/bin/.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "libgb.so"
INCLUDE = HERE.parent / "include"
APPS = HERE / "apps"
APPS_BIN = APPS / "bin"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libgb")
    return cand


def _headers() -> list[Path]:
    return sorted(list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h")))


def _stale(src: Path, obj: Path, headers: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or any(h.stat().st_mtime > t for h in headers)


def _compile(cmd: list[str]) -> tuple[list[str], int, str]:
    p = subprocess.run(cmd, capture_output=True, text=True)
    return cmd, p.returncode, p.stdout + p.stderr


def build(jobs: int | None = None, force: bool = False, verbose: bool = False) -> Path:
    nvcc = _nvcc()
    BUILD.mkdir(exist_ok=True)
    headers = _headers()
    inc = [f"-I{CSRC}", f"-I{INCLUDE}"]
    cmds = []
    objs = []
    for src in sorted(CSRC.glob("*.cu")):
        obj = BUILD / (src.stem + ".cu.o")
        objs.append(obj)
        if force or _stale(src, obj, headers):
            cmds.append([nvcc, *ARCH, "-lineinfo", "-O3", "-std=c++17", "--expt-relaxed-constexpr",
                         "-Xcompiler", "-fPIC,-O3", *inc, "-c", str(src), "-o", str(obj)])
    for src in sorted(CSRC.glob("*.cpp")):
        obj = BUILD / (src.stem + ".cpp.o")
        objs.append(obj)
        if force or _stale(src, obj, headers):
            cmds.append(["/usr/bin/g++", "-O3", "-std=c++17", "-fPIC", "-fopenmp", *inc, "-c", str(src), "-o", str(obj)])
    failed = []
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        for cmd, rc, out in ex.map(_compile, cmds):
            if verbose or rc != 0:
                sys.stderr.write(" ".join(cmd) + "\n" + out)
            if rc != 0:
                failed.append(cmd[-3])
    if failed:
        raise RuntimeError(f"compilation failed: {failed}")
    if cmds or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        link = [nvcc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-cudart", "static",
                "-Xcompiler", "-fopenmp", "-lgomp"]
        cmd, rc, out = _compile(link)
        if rc != 0:
            sys.stderr.write(" ".join(cmd) + "\n" + out)
            raise RuntimeError("link of libgb.so failed")
    build_apps(jobs, force, verbose)
    return LIB


def build_apps(jobs: int | None = None, force: bool = False, verbose: bool = False) -> list[Path]:
    """Link every apps/*.cpp (g++) and apps/*.cu (nvcc, extended lambdas) into
    apps/bin/<name with '-' for '_'> against libgb.so (rpath $ORIGIN/../..)."""
    nvcc = _nvcc()
    APPS_BIN.mkdir(exist_ok=True)
    headers = _headers() + sorted(APPS.glob("*.h")) + sorted(INCLUDE.glob("*.cuh")) + [LIB]
    link = [f"-L{HERE}", "-lgb", "-Wl,-rpath,$ORIGIN/../.."]
    cmds, outs = [], []
    for src in sorted(APPS.glob("*.cpp")) + sorted(APPS.glob("*.cu")):
        exe = APPS_BIN / src.stem.replace("_", "-")
        outs.append(exe)
        if not (force or _stale(src, exe, headers)):
            continue
        if src.suffix == ".cpp":
            cmds.append(["/usr/bin/g++", "-O2", "-std=c++17", f"-I{INCLUDE}", f"-I{APPS}", str(src),
                         "-o", str(exe), *link])
        else:
            cmds.append([nvcc, *ARCH, "-O2", "-std=c++17", "--extended-lambda", f"-I{INCLUDE}", f"-I{APPS}",
                         str(src), "-o", str(exe), "-Xlinker", f"-L{HERE},-lgb,-rpath,$ORIGIN/../.."])
    failed = []
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        for cmd, rc, out in ex.map(_compile, cmds):
            if verbose or rc != 0:
                sys.stderr.write(" ".join(cmd) + "\n" + out)
            if rc != 0:
                failed.append(cmd[-1] if cmd[0].endswith("g++") else cmd[-3])
    if failed:
        raise RuntimeError(f"app build failed: {failed}")
    return outs


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    args = ap.parse_args()
    print(build(args.jobs, args.force, args.verbose))


if __name__ == "__main__":
    main()
