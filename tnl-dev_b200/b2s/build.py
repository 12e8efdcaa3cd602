"""Build recipe for libb2sparse.so (sm_100a) and the C++ TNL-interface tests.

Compiles every ``csrc/*.cu`` with nvcc for ``compute_100a/sm_100a`` into
``tnl-dev_b200/_build`` and links ``tnl-dev_b200/libb2sparse.so`` in-tree.
Incremental: a translation unit is rebuilt when it or any header is newer
than its object file.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent.parent          # tnl-dev_b200/
ROOT = PKG.parent                                      # repository root
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libb2sparse.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
              "--expt-relaxed-constexpr", "-I", str(ROOT / "include"), "-DB2S_BUILD"]


def _sources():
    return sorted(CSRC.glob("*.cu"))


def _headers():
    return list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h"))


def _needs(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or any(h.stat().st_mtime > t for h in _headers())


def _compile(src: Path, extra) -> Path:
    obj = BUILD / (src.stem + ".o")
    if _needs(obj, src):
        cmd = [NVCC, *ARCH, *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed for {src.name}")
    return obj


def build(verbose: bool = False, extra=()) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = _sources()
    with ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, list(extra)), srcs))
    if not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link of libb2sparse.so failed")
    build_cpp_tests()
    if verbose:
        print(f"built {LIB}")
    return LIB


CPP_TEST_SRC = ROOT / "tests" / "cpp" / "tnl_api_test.cpp"
CPP_TEST_BIN = BUILD / "tnl_api_test"


def build_cpp_tests() -> Path:
    """Host C++ program written against the TNL-shaped headers, linked to libb2sparse.so."""
    deps = [CPP_TEST_SRC, PKG / "include" / "TNL" / "b2s_tnl.h", ROOT / "include" / "b2s.h", LIB]
    if CPP_TEST_BIN.exists() and all(d.stat().st_mtime <= CPP_TEST_BIN.stat().st_mtime for d in deps):
        return CPP_TEST_BIN
    cuda = Path(NVCC).resolve().parent.parent
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-I", str(ROOT / "include"), "-I", str(PKG / "include"),
           "-I", str(cuda / "include"), str(CPP_TEST_SRC), "-o", str(CPP_TEST_BIN),
           "-L", str(PKG), "-lb2sparse", f"-Wl,-rpath,{PKG}", "-Wl,-rpath,$ORIGIN/..",
           "-L", str(cuda / "lib64"), "-lcudart", f"-Wl,-rpath,{cuda / 'lib64'}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build of tests/cpp/tnl_api_test.cpp failed")
    return CPP_TEST_BIN


if __name__ == "__main__":
    build(verbose=True)
