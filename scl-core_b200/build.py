"""Build the B200 diffusion libraries in-tree.

    python scl-core_b200/build.py            # incremental
    python scl-core_b200/build.py --clean    # from scratch

Compiles the CUDA engine (csrc/*.cu) once for sm_100a and the C-ABI layer
(csrc/c_api_*.cpp) once per scl-core library variant, then links
scl/libs/libscl_<f32|f64>_<i32|i64>.so — the names scl-core's Python loader
searches for (codegen/cli.py:441-460). CUDA runtime is linked statically and
only SCL_EXPORT symbols are visible.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent
CSRC = ROOT / "csrc"
INCLUDE = ROOT.parent / "include"
BUILD = ROOT / "_build"
LIBS = ROOT / "scl" / "libs"

CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
CXX = shutil.which("g++", path="/usr/bin") or "g++"

VARIANTS = {
    "f32_i32": ["-DSCL_USE_FLOAT32", "-DSCL_USE_INT32"],
    "f32_i64": ["-DSCL_USE_FLOAT32", "-DSCL_USE_INT64"],
    "f64_i32": ["-DSCL_USE_FLOAT64", "-DSCL_USE_INT32"],
    "f64_i64": ["-DSCL_USE_FLOAT64", "-DSCL_USE_INT64"],
}

NVCC_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
    "-diag-suppress", "177",
    f"-I{INCLUDE}", f"-I{CSRC}",
]
CXX_FLAGS = ["-std=c++17", "-O2", "-fPIC", "-fvisibility=hidden", "-Wall", "-Wno-unused-parameter",
             f"-I{INCLUDE}", f"-I{CSRC}", f"-I{CUDA_HOME / 'include'}"]


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed ({r.returncode}): {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def build(clean: bool = False, verbose: bool = False, jobs: int | None = None) -> list[Path]:
    if clean and BUILD.exists():
        shutil.rmtree(BUILD)
    BUILD.mkdir(parents=True, exist_ok=True)
    LIBS.mkdir(parents=True, exist_ok=True)
    headers = sorted(CSRC.glob("*.hpp")) + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))
    cu_srcs = sorted(CSRC.glob("*.cu"))
    cpp_srcs = sorted(CSRC.glob("c_api_*.cpp"))

    jobs_list = []  # (out, cmd, deps)
    cu_objs = []
    for src in cu_srcs:
        out = BUILD / (src.stem + ".cu.o")
        cu_objs.append(out)
        jobs_list.append((out, [NVCC, *NVCC_FLAGS, "-c", str(src), "-o", str(out)], [src, *headers]))
    var_objs: dict[str, list[Path]] = {}
    for var, defs in VARIANTS.items():
        var_objs[var] = []
        for src in cpp_srcs:
            out = BUILD / f"{src.stem}.{var}.o"
            var_objs[var].append(out)
            jobs_list.append((out, [CXX, *CXX_FLAGS, *defs, "-c", str(src), "-o", str(out)], [src, *headers]))

    todo = [(o, c) for (o, c, d) in jobs_list if _stale(o, d)]
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        futs = {ex.submit(_run, c): o for (o, c) in todo}
        for f in cf.as_completed(futs):
            f.result()
            if verbose:
                print("built", futs[f].name)

    libs = []
    for var, objs in var_objs.items():
        lib = LIBS / f"libscl_{var}.so"
        libs.append(lib)
        deps = objs + cu_objs
        if _stale(lib, deps):
            cmd = [CXX, "-shared", "-o", str(lib), *map(str, objs), *map(str, cu_objs),
                   f"-L{CUDA_HOME / 'lib64'}", "-lcudart_static", "-lrt", "-lpthread", "-ldl",
                   "-Wl,--exclude-libs,ALL", "-Wl,-z,defs", "-Wl,-soname," + lib.name]
            _run(cmd)
            if verbose:
                print("linked", lib.name)
    return libs


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    for p in build(clean=a.clean, verbose=a.verbose):
        print(p)
    sys.exit(0)
