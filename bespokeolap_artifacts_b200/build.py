"""Builds the native parts in-tree.

* ``libbespoke_gpu.so``: the CUDA kernels and the C ABI (``include/bespoke_gpu.h``),
  compiled by nvcc for sm_100a only, linked against the static CUDA runtime.
* ``oracle/liboracle.so`` and ``oracle/_ref/*``: the CPU checker (built by
  ``oracle/build_oracle.py``; test infrastructure, never loaded by the product).

Run ``python -m bespokeolap_artifacts_b200.build`` or call :func:`build_all`.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
LIB_PATH = PKG / "libbespoke_gpu.so"

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-lineinfo",
    "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC",
]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libbespoke_gpu.so")
    return cand


def _sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build_gpu_lib(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> Path:
    """Compiles every ``csrc/*.cu`` into one shared library (parallel objects)."""
    nvcc = _nvcc()
    obj_dir = PKG / "_build"
    obj_dir.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    srcs = _sources()
    procs = []
    objs = []
    for src in srcs:
        obj = obj_dir / (src.stem + ".o")
        objs.append(obj)
        if not force and not _stale(obj, [src] + headers):
            continue
        cmd = [nvcc, *ARCH_FLAGS, *NVCC_FLAGS, f"-I{INCLUDE}", f"-I{CSRC}", "-c", str(src), "-o", str(obj)]
        if ptxas_info:
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append((src, out))
        elif out and (verbose or ptxas_info):
            print(out)
    if failed:
        msg = "\n".join(f"--- {s.name}\n{o}" for s, o in failed)
        raise RuntimeError(f"nvcc failed:\n{msg}")
    if force or procs or _stale(LIB_PATH, objs):
        cmd = [nvcc, *ARCH_FLAGS, "-shared", "-o", str(LIB_PATH), *map(str, objs)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB_PATH


HOST = PKG / "host"
HOST_LIB = HOST / "libbespoke_tpch_gpu.so"
HOST_DRIVER = HOST / "bespoke_tpch_gpu"


def build_host(force: bool = False) -> Path | None:
    """The drop-in C++ host (load / build / query over the C ABI) and a stand-in
    driver executable, against the Arrow / Parquet C++ libraries that come
    with pyarrow.  Skipped (None) when pyarrow is not importable."""
    try:
        import pyarrow as pa
    except ImportError:
        return None
    inc, libdir = pa.get_include(), pa.get_library_dirs()[0]
    srcs = [HOST / "tpch_gpu.cpp"]
    deps = srcs + [HOST / "tpch_gpu.hpp", INCLUDE / "bespoke_gpu.h", CSRC / "host_threads.cuh", LIB_PATH]
    arrow = [f"-L{libdir}", "-l:libarrow.so.2400", "-l:libparquet.so.2400", f"-Wl,-rpath,{libdir}"]
    if force or _stale(HOST_LIB, deps):
        subprocess.run(["g++", "-std=c++20", "-O2", "-pthread", "-fPIC", "-shared", f"-I{INCLUDE}", f"-I{CSRC}", f"-I{inc}",
                        *map(str, srcs),
                        f"-L{PKG}", "-lbespoke_gpu", f"-Wl,-rpath,{PKG}", *arrow, "-o", str(HOST_LIB)], check=True)
    main = HOST / "driver_main.cpp"
    if force or _stale(HOST_DRIVER, [main, HOST_LIB, HOST / "tpch_gpu.hpp"]):
        subprocess.run(["g++", "-std=c++20", "-O2", f"-I{INCLUDE}", f"-I{inc}", str(main), f"-L{HOST}",
                        "-lbespoke_tpch_gpu", f"-Wl,-rpath,{HOST}", f"-L{PKG}", "-lbespoke_gpu", f"-Wl,-rpath,{PKG}",
                        *arrow, "-o", str(HOST_DRIVER)], check=True)
    return HOST_LIB


def build_oracle(force: bool = False) -> None:
    """Builds the CPU checker under ``oracle/`` (C restatement and, when the
    reference sources are present on this machine, the compiled reference)."""
    script = ROOT / "oracle" / "build_oracle.py"
    if script.exists():
        subprocess.run([sys.executable, str(script)] + (["--force"] if force else []), check=True)


def build_all(force: bool = False) -> None:
    build_gpu_lib(force=force)
    build_host(force=force)
    build_oracle(force=force)


if __name__ == "__main__":
    force = "--force" in sys.argv
    info = "--ptxas" in sys.argv
    build_gpu_lib(force=force or info, verbose="-v" in sys.argv, ptxas_info=info)
    if "--gpu-only" not in sys.argv:
        build_host(force=force)
        build_oracle(force=force)
    print(f"built {LIB_PATH}")
