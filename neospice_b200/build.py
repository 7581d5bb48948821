"""Build libnsgpu.so in-tree with nvcc for sm_100a.

Host C++ and CUDA sources under csrc/ are compiled to objects in _build/ and
linked into neospice_b200/libnsgpu.so.  nvcc cross-compiles without a GPU.
Run directly (``python -m neospice_b200.build``) or through
``__graft_entry__.build()``.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import pathlib
import shutil
import subprocess

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libnsgpu.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3",
          f"-I{ROOT / 'include'}", f"-I{CSRC}"]
# No FMA contraction: every multiply and add is rounded separately, as on the
# reference's x86-64 build, so factor and solve values are bit-identical.
DEVICE = ["-fmad=false", "--expt-relaxed-constexpr"]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libnsgpu")
    return cand


def sources() -> list[pathlib.Path]:
    return sorted(list(CSRC.rglob("*.cu")) + list(CSRC.rglob("*.cpp")))


def _obj(src: pathlib.Path) -> pathlib.Path:
    rel = src.relative_to(CSRC).with_suffix(src.suffix + ".o")
    return BUILD / rel


def _headers_mtime() -> float:
    hs = list(CSRC.rglob("*.hpp")) + list(CSRC.rglob("*.cuh")) + list((ROOT / "include").glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def _compile(src: pathlib.Path, verbose: bool) -> pathlib.Path:
    obj = _obj(src)
    obj.parent.mkdir(parents=True, exist_ok=True)
    cmd = [nvcc(), *ARCH, *COMMON, *DEVICE, "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cu":
        cmd += ["-Xptxas", "-v"] if verbose else []
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{res.stdout}\n{res.stderr}")
    if verbose and res.stderr:
        print(res.stderr)
    return obj


def build(force: bool = False, verbose: bool = False) -> pathlib.Path:
    srcs = sources()
    hdr = _headers_mtime()
    todo = [s for s in srcs if force or not _obj(s).exists()
            or _obj(s).stat().st_mtime < max(s.stat().st_mtime, hdr)]
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        list(ex.map(lambda s: _compile(s, verbose), todo))
    objs = [_obj(s) for s in srcs]
    if force or todo or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    return LIB


if __name__ == "__main__":
    import sys
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
