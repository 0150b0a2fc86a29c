"""Build libquax_b200.so for sm_100a (in-tree, no JIT cache).

Each CUDA translation unit is compiled by nvcc in parallel into
quax_b200/_build/*.o; an object is rebuilt when its source or a local header it
includes (recursively) is newer.  The objects are linked into
quax_b200/libquax_b200.so with the CUDA runtime linked statically, so the
library does not depend on which libcudart the host process loaded first.
"""
from __future__ import annotations

import glob
import os
import re
import shutil
import subprocess
import sys
import time
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libquax_b200.so")
PEAKS_LIB = os.path.join(PKG, "libqx_peaks.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-lineinfo",
    "-O3",
    "-std=c++17",
    "-Xcompiler",
    "-fPIC",
    "-I" + os.path.join(ROOT, "include"),
    "-I" + CSRC,
]


def nvcc() -> str:
    for cand in (os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc"), shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "gen", "*.cu")))


_INC = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.M)


def _deps_mtime(src: str, seen=None) -> float:
    """Newest mtime of src and of every local header it includes, recursively
    (quoted includes resolved against the including file's folder, csrc/ and
    include/), so a header change rebuilds only the translation units that use it."""
    seen = set() if seen is None else seen
    if src in seen or not os.path.exists(src):
        return 0.0
    seen.add(src)
    t = os.path.getmtime(src)
    with open(src, errors="replace") as f:
        text = f.read()
    for name in _INC.findall(text):
        for base in (os.path.dirname(src), CSRC, os.path.join(ROOT, "include")):
            cand = os.path.normpath(os.path.join(base, name))
            if os.path.exists(cand):
                t = max(t, _deps_mtime(cand, seen))
                break
    return t


def _obj(src: str) -> str:
    rel = os.path.relpath(src, CSRC).replace(os.sep, "_")
    return os.path.join(BUILD, rel[:-3] + ".o")


def _compile(src: str, verbose: bool):
    obj = _obj(src)
    if os.path.exists(obj) and os.path.getmtime(obj) >= _deps_mtime(src):
        return obj, False
    flags = NVCC_FLAGS
    if os.path.basename(src).startswith("k_rys_"):
        # the 55 Rys-engine units carry ~7 kernels each; their line tables would
        # more than double the library, so they are built without -lineinfo
        flags = [f for f in NVCC_FLAGS if f != "-lineinfo"]
    cmd = [nvcc()] + flags + ["-c", src, "-o", obj]
    t0 = time.time()
    r = subprocess.run(cmd, capture_output=True, text=True)
    if verbose:
        print(f"{time.time() - t0:7.1f}s  {os.path.basename(src)}", flush=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    return obj, True


def build(verbose: bool = False, jobs: int | None = None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    # the generator rewrites only files whose content changed; a stamp records the run
    stamp = os.path.join(CSRC, "gen", ".stamp")
    if not os.path.exists(stamp) or os.path.getmtime(stamp) < os.path.getmtime(os.path.join(CSRC, "gen_eri.py")):
        subprocess.run([sys.executable, os.path.join(CSRC, "gen_eri.py")], check=True)
        with open(stamp, "w") as f:
            f.write("generated\n")
    srcs = sources()
    with ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose), srcs))
    objs = [o for o, _ in results]
    _link(LIB, objs, any(b for _, b in results))
    # FMA throughput probe used by the benchmark's roofline (separate library)
    psrc = os.path.join(CSRC, "peaks", "qx_peaks.cu")
    pobj, pb = _compile(psrc, verbose)
    _link(PEAKS_LIB, [pobj], pb)
    return LIB


def _link(lib: str, objs, rebuilt: bool):
    if rebuilt or not os.path.exists(lib) or os.path.getmtime(lib) < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", lib] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")


if __name__ == "__main__":
    t = time.time()
    print(build(verbose="-v" in sys.argv), f"{time.time() - t:.1f}s")
