"""Build libgmpm.so in-tree with nvcc for sm_100a.

    python explicit-gpumpm-ductile-fracture_b200/build.py [--force] [--verbose-ptxas]

Compiles csrc/*.cu and csrc/*.cpp in parallel into _build/ and links
libgmpm.so next to this file.  Rebuilds only when a source or header is newer
than the library.
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
ROOT = HERE.parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "libgmpm.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xcompiler", "-Wall", "-Xcompiler", "-Wno-unused-function",
              # host code: no fused multiply-add, so the host restatements of the reference's
              # samplers round as the reference does
              "-Xcompiler", "-ffp-contract=off"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def headers() -> list[Path]:
    return sorted(list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [ROOT / "include" / "gmpm.h"])


def up_to_date() -> bool:
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in sources() + headers() + [Path(__file__)])


def compile_one(src: Path, verbose_ptxas: bool) -> tuple[Path, str]:
    obj = BUILD / (src.name + ".o")
    cmd = [nvcc_path(), *ARCH, *NVCC_FLAGS, "-I", str(ROOT / "include"), "-I", str(CSRC), "-c", str(src), "-o",
           str(obj)]
    if verbose_ptxas and src.suffix == ".cu":
        cmd[1:1] = ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(force: bool = False, verbose_ptxas: bool = False) -> Path:
    if not force and not verbose_ptxas and up_to_date():
        return LIB
    BUILD.mkdir(exist_ok=True)
    srcs = sources()
    objs = []
    logs = []
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        for obj, log in ex.map(lambda s: compile_one(s, verbose_ptxas), srcs):
            objs.append(obj)
            if log.strip():
                logs.append(log)
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc_path(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart_static", "-lrt", "-ldl",
           "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    if verbose_ptxas:
        sys.stderr.write("\n".join(logs))
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose_ptxas=a.verbose_ptxas))


if __name__ == "__main__":
    main()
