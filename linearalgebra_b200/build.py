"""Build the B200 kernel library in-tree.

    python -m linearalgebra_b200.build        # -> linearalgebra_b200/libb200la.so

Compiles every csrc/*.cu for sm_100a only (nvcc cross-compiles; no GPU is
needed to build) and links them into one shared library exporting the C ABI
declared in include/b200la.h.  Object files go to linearalgebra_b200/_build/.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libb200la.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
def cutlass_include() -> str:
    """CuTe/CUTLASS header tree (used for the tcgen05 descriptor layouts)."""
    cands = []
    try:
        import flashinfer  # noqa: F401
        cands.append(os.path.join(os.path.dirname(flashinfer.__file__), "data", "cutlass", "include"))
    except Exception:
        pass
    cands.append(os.path.join(sys.prefix, "lib", f"python{sys.version_info.major}.{sys.version_info.minor}",
                              "site-packages", "flashinfer", "data", "cutlass", "include"))
    for c in cands:
        if os.path.exists(os.path.join(c, "cute", "arch", "mma_sm100_desc.hpp")):
            return c
    raise RuntimeError("CuTe headers (cute/arch/mma_sm100_desc.hpp) not found")


NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "-I", os.path.join(ROOT, "include"),
]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, os.path.splitext(os.path.basename(src))[0] + ".o")
    deps = (glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(ROOT, "include", "**", "*.h"), recursive=True)
            + [src])
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(d) for d in deps):
        return obj
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-I", cutlass_include(), "-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{res.stdout}\n{res.stderr}")
    if verbose:
        sys.stderr.write(res.stderr)
    return obj


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    with ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    return LIB


CPP_TEST_SRC = os.path.join(ROOT, "tests", "cpp", "test_backend_b200.cpp")
CPP_TEST_BIN = os.path.join(ROOT, "tests", "cpp", "test_backend_b200")


def build_cpp_test() -> str:
    """Compile the C++ operator-API test program against libb200la.so."""
    build()
    if os.path.exists(CPP_TEST_BIN) and os.path.getmtime(CPP_TEST_BIN) >= max(
            os.path.getmtime(CPP_TEST_SRC), os.path.getmtime(LIB)):
        return CPP_TEST_BIN
    cmd = [nvcc(), "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), CPP_TEST_SRC,
           "-o", CPP_TEST_BIN, "-L", HERE, "-lb200la", "-Xlinker", f"-rpath={HERE}", "-lcudart"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"C++ test build failed:\n{res.stdout}\n{res.stderr}")
    return CPP_TEST_BIN


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
