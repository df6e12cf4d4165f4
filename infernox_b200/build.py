"""In-tree build of libcmscan_gpu.so for sm_100a (nvcc, no JIT cache)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libcmscan_gpu.so")

SOURCES = ["qdb_scan.cu", "sweep_scan.cu", "capi.cpp", "cm_prep.cpp", "qdb_plan.cpp", "noalloc.cu", "p7_vit.cu", "p7_msv.cu", "hb_scan.cu", "trq_scan.cu", "calibrate.cpp", "p7_fwd.cu"]
HEADERS = ["devbuf.h", "trunc_report.h", "cm_internal.h", "qdb_plan.h", "qdb_kernel.h", "model_internal.h",
           "semiring.cuh", "sweep_plan.h", "sweep_kernel.h"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-fmad=false",                      # no contraction in device float math
    "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math",
]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "cmscan_gpu.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles every source to an object file (in parallel), then links the
    shared library; the objects live in a temporary folder."""
    if not force and not _stale():
        return LIB
    import tempfile
    from concurrent.futures import ThreadPoolExecutor

    os.makedirs(LIBDIR, exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    with tempfile.TemporaryDirectory(prefix="cmscan_obj_") as tmp:
        def compile_one(src: str) -> str:
            obj = os.path.join(tmp, os.path.splitext(src)[0] + ".o")
            cmd = [nvcc] + NVCC_FLAGS + ["-c", "-o", obj, os.path.join(CSRC, src)]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            subprocess.run(cmd, check=True)
            return obj

        with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 1)) as ex:
            objs = list(ex.map(compile_one, SOURCES))
        cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "--shared", "-o", LIB + ".tmp"] + objs
        subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
