"""Build the in-tree CUDA library gradscf_b200/_lib/libb200jk.so for sm_100a.

Every translation unit under csrc/ is compiled by nvcc in parallel
(jk_inst.cu once per class pair, -DBRA_CLASS=x -DKET_CLASS=y, y <= x), then linked into one
shared library exporting the C ABI of include/b200jk.h.  Object files are
cached under gradscf_b200/_build/ and rebuilt when a source or header is
newer.  Usage: python -m gradscf_b200.build [-j JOBS] [--force]
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "_lib" / "libb200jk.so"
INCLUDE = PKG.parent / "include"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC",
         "-Xptxas", "-warn-spills"] + ARCH


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def units():
    out = []
    for src in sorted(CSRC.glob("*.cu")):
        if src.name == "jk_inst.cu":
            for x in range(9, -1, -1):
                for y in range(x, -1, -1):
                    out.append((src, BUILD / f"jk_inst_{x}_{y}.o", [f"-DBRA_CLASS={x}", f"-DKET_CLASS={y}"]))
        else:
            out.append((src, BUILD / (src.stem + ".o"), []))
    return out


def _stale(obj, src):
    if not obj.exists():
        return True
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    newest = max([src.stat().st_mtime] + [h.stat().st_mtime for h in headers])
    return obj.stat().st_mtime < newest


def build(jobs=None, force=False, verbose=False):
    BUILD.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    todo = [(s, o, d) for s, o, d in units() if force or _stale(o, s)]

    def compile_one(item):
        src, obj, defs = item
        cmd = [nvcc()] + FLAGS + defs + ["-I", str(CSRC), "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src.name} {defs}:\n{r.stderr[-6000:]}")
        return r.stderr

    with ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        for log in ex.map(compile_one, todo):
            if verbose and log.strip():
                print(log)
    objs = [str(o) for _, o, _ in units()]
    if todo or not LIB.exists():
        cmd = [nvcc()] + ARCH + ["-shared", "-o", str(LIB)] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr[-4000:]}")
    return LIB


FFI_SRC = PKG / "ffi" / "b200jk_xla_ffi.cc"
FFI_LIB = PKG / "_lib" / "libgradscf_b200_ffi.so"


def build_ffi():
    """The XLA FFI handler (ffi/b200jk_xla_ffi.cc), built only where JAX's FFI
    headers exist (jax.ffi.include_dir()); returns the library path or None."""
    try:
        import jax  # noqa: F401
        inc = jax.ffi.include_dir()
    except Exception as e:  # JAX absent: the handler cannot be compiled
        print(f"XLA FFI handler not built: {e}")
        return None
    lib = build()
    cmd = [nvcc(), "-std=c++17", "-O2", "-Xcompiler", "-fPIC", "-shared", "-I", inc, "-I", str(INCLUDE),
           str(FFI_SRC), "-o", str(FFI_LIB), "-L", str(lib.parent), "-lb200jk", "-Xlinker", "-rpath=$ORIGIN",
           "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"FFI handler build failed:\n{r.stderr[-4000:]}")
    return FFI_LIB


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("-j", "--jobs", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ffi", action="store_true", help="also build the XLA FFI handler (needs JAX)")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(a.jobs, a.force, a.verbose))
    if a.ffi:
        print(build_ffi())


if __name__ == "__main__":
    main(sys.argv[1:])
