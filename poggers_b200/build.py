"""Build recipe for libpoggers_b200.so (sm_100a) and its C++ test drivers.

Compiles every CUDA source under poggers_b200/csrc with nvcc for sm_100a,
in parallel, into objects under poggers_b200/_build/, and links them into
poggers_b200/libpoggers_b200.so in-tree (the shared library travels with the
source tree; nothing is installed into site-packages).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libpoggers_b200.so"
INCLUDE = ROOT / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    f"-I{INCLUDE}", f"-I{CSRC}",
]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build poggers_b200")
    return cand


def _needs(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _headers() -> list[Path]:
    return sorted(INCLUDE.rglob("*.h")) + sorted(INCLUDE.rglob("*.cuh")) + sorted(CSRC.glob("*.cuh"))


def _compile(src: Path, extra: list[str]) -> Path:
    obj = BUILD / (src.stem + ".o")
    if _needs(obj, [src] + _headers()):
        cmd = [nvcc(), *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(verbose: bool = False, extra: list[str] | None = None, lib: Path | None = None,
          build_dir: Path | None = None) -> Path:
    """Compile and link libpoggers_b200.so (or a variant at `lib` built with
    `extra` nvcc flags in `build_dir`); returns its path."""
    global BUILD
    lib = Path(lib) if lib else LIB
    if build_dir:
        BUILD = Path(build_dir)
    BUILD.mkdir(parents=True, exist_ok=True)
    extra = list(extra or [])
    srcs = sorted(CSRC.glob("*.cu"))
    with cf.ThreadPoolExecutor(max_workers=min(len(srcs), os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra), srcs))
    if _needs(lib, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "shared", "-o", str(lib), *map(str, objs)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(f"built {lib}")
    return lib


TEST_SRC = ROOT / "tests" / "cpp"
TEST_BIN = TEST_SRC / "_bin"


def build_tests(verbose: bool = False) -> list[Path]:
    """C++ drivers written against the reference-shaped template API (tests/cpp)."""
    lib = build()
    TEST_BIN.mkdir(exist_ok=True)
    out = []
    for src in sorted(TEST_SRC.glob("*.cu")):
        exe = TEST_BIN / src.stem
        if _needs(exe, [src, lib] + _headers()):
            cmd = [nvcc(), *NVCC_FLAGS, str(src), "-o", str(exe), f"-L{PKG}", "-lpoggers_b200",
                   f"-Xlinker", f"-rpath={PKG}", "-Xlinker", "-rpath=$ORIGIN/../../../poggers_b200"]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
        out.append(exe)
        if verbose:
            print(f"built {exe}")
    return out


if __name__ == "__main__":
    build(verbose=True, extra=sys.argv[1:])
