"""Build recipe for the CPU checker (test infrastructure, not the product).

* ``oracle/liboracle.so``: the plain-C restatement (``bo_oracle.c``).
* ``oracle/_ref/libref_tpch.so`` and ``libref_tpch_trace.so`` (``-DTRACE``): the
  reference's own TPC-H pipelines compiled unchanged from the reference tree
  (``query_impl.cpp`` via ``ref_harness.cpp``, plus ``builder_impl.cpp`` and
  ``loader_impl.cpp``) against the Arrow/Parquet C++ libraries bundled with
  pyarrow.  Built only where the reference sources are present (the development
  container); the outputs are plain files that travel with the repository
  snapshot, so machines without the sources use the prebuilt copies.
* ``oracle/_ref/ref_tpch_driver`` and ``ref_ceb_driver``: the reference's own
  load / build / query of its TPC-H and CEB engines behind a stand-in driver
  main (``ref_driver_main.cpp``).

Usage: ``python oracle/build_oracle.py [--force]``.  The reference tree is
read from ``$BO_REFERENCE_DIR`` (default ``/root/reference``).
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF_DIR = Path(os.environ.get("BO_REFERENCE_DIR", "/root/reference"))
OUT_REF = HERE / "_ref"


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build_c_oracle(force: bool = False) -> Path:
    out = HERE / "liboracle.so"
    src = HERE / "bo_oracle.c"
    if force or _stale(out, [src]):
        subprocess.run(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", str(src), "-o", str(out)], check=True)
    return out


def build_reference(force: bool = False) -> list[Path]:
    tpch = REF_DIR / "bespoke_tpch"
    if not (tpch / "query_impl.cpp").exists():
        print(f"reference sources not found under {REF_DIR}; keeping prebuilt oracle/_ref", file=sys.stderr)
        return []
    import pyarrow as pa

    inc = pa.get_include()
    libdir = pa.get_library_dirs()[0]
    OUT_REF.mkdir(exist_ok=True)
    srcs = [HERE / "ref_harness.cpp", tpch / "builder_impl.cpp", tpch / "loader_impl.cpp"]
    deps = srcs + list(tpch.glob("*.hpp")) + list(tpch.glob("query_q*.cpp")) + [tpch / "query_impl.cpp"]
    deps += list((HERE / "ref_stubs").glob("*.hpp"))
    outs = []
    jobs = []
    for name, extra in (("libref_tpch.so", []), ("libref_tpch_trace.so", ["-DTRACE"])):
        out = OUT_REF / name
        outs.append(out)
        if not force and not _stale(out, deps):
            continue
        cmd = [
            "g++", "-std=c++20", "-O3", "-fPIC", "-shared", *extra,
            f"-I{tpch}", f"-I{HERE / 'ref_stubs'}", f"-I{inc}",
            *map(str, srcs),
            f"-L{libdir}", "-l:libarrow.so.2400", "-l:libparquet.so.2400",
            f"-Wl,-rpath,{libdir}", "-lpthread", "-o", str(out),
        ]
        jobs.append(subprocess.Popen(cmd))
    # The reference's own load / build / query behind a stand-in driver main.
    drv = OUT_REF / "ref_tpch_driver"
    outs.append(drv)
    dsrcs = [HERE / "ref_driver_main.cpp", tpch / "query_impl.cpp", tpch / "builder_impl.cpp", tpch / "loader_impl.cpp"]
    if force or _stale(drv, dsrcs + deps):
        jobs.append(subprocess.Popen([
            "g++", "-std=c++20", "-O2", f"-I{tpch}", f"-I{HERE / 'ref_stubs'}", f"-I{inc}", *map(str, dsrcs),
            f"-L{libdir}", "-l:libarrow.so.2400", "-l:libparquet.so.2400", f"-Wl,-rpath,{libdir}", "-lpthread",
            "-o", str(drv)]))
    # The reference's CEB engine (its generic column builder and the IMDB
    # queries) behind the same stand-in driver main.
    ceb = REF_DIR / "bespoke_ceb"
    if (ceb / "query_impl.cpp").exists():
        cdrv = OUT_REF / "ref_ceb_driver"
        outs.append(cdrv)
        csrcs = [HERE / "ref_driver_main.cpp", ceb / "query_impl.cpp", ceb / "builder_impl.cpp", ceb / "loader_impl.cpp"]
        cdeps = csrcs + list(ceb.glob("*.hpp")) + list(ceb.glob("query_q*.cpp")) + list((HERE / "ref_stubs").glob("*.hpp"))
        if force or _stale(cdrv, cdeps):
            jobs.append(subprocess.Popen([
                "g++", "-std=c++20", "-O2", f"-I{ceb}", f"-I{HERE / 'ref_stubs'}", f"-I{inc}", *map(str, csrcs),
                f"-L{libdir}", "-l:libarrow.so.2400", "-l:libparquet.so.2400", f"-Wl,-rpath,{libdir}", "-lpthread",
                "-o", str(cdrv)]))
    for j in jobs:
        if j.wait() != 0:
            raise RuntimeError("building the reference harness failed")
    return outs


if __name__ == "__main__":
    force = "--force" in sys.argv
    print(build_c_oracle(force))
    for p in build_reference(force):
        print(p)
