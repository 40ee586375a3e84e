"""Build recipe for the native library libcup3d_b200.so (sm_100a) and the oracle.

`python -m cup3d_b200.build` compiles every CUDA/C++ source of cup3d_b200/csrc
with nvcc for sm_100a into cup3d_b200/libcup3d_b200.so (in-tree, so the built
library travels with the repository snapshot), and the CPU oracle used by the
tests into oracle/liboracle.so.
"""
from __future__ import annotations

import concurrent.futures as cf
import hashlib
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = ROOT / "_build"
LIB = PKG / "libcup3d_b200.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--extended-lambda", "-Xcompiler", "-fPIC",
    "-Xcompiler", "-Wall", "-I", str(ROOT / "include"),
]
HOSTCXX = "g++"
# Per-file flags: device obstacle creation repeats the host code's arithmetic
# bit for bit, so it is compiled without fused multiply-adds.
FILE_FLAGS = {"obstacles_dev.cu": ["--fmad=false"]}


def _sources():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _headers_digest() -> str:
    h = hashlib.sha1()
    for p in sorted(list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h"))):
        h.update(p.read_bytes())
    return h.hexdigest()[:12]


def _compile(src: Path, digest: str, verbose: bool) -> Path:
    obj = BUILD / f"{src.stem}.{src.suffix[1:]}.{digest}.o"
    if obj.exists() and obj.stat().st_mtime >= src.stat().st_mtime:
        return obj
    cmd = [NVCC, "-ccbin", HOSTCXX] + NVFLAGS + FILE_FLAGS.get(src.name, []) + ["-c", str(src), "-o", str(obj)]
    if src.suffix == ".cpp":
        cmd = [NVCC, "-ccbin", HOSTCXX, "-x", "cu"] + NVFLAGS + ["-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr.strip():
        print(r.stderr, file=sys.stderr)
    return obj


def build_native(verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    digest = _headers_digest()
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, digest, verbose), srcs))
    newest = max(o.stat().st_mtime for o in objs)
    if not LIB.exists() or LIB.stat().st_mtime < newest:
        cmd = [NVCC, "-ccbin", HOSTCXX] + ARCH + ["-shared", "-cudart", "static", "-o", str(LIB)] + [
            str(o) for o in objs]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


def build_oracle(verbose: bool = False) -> Path:
    r = subprocess.run(["make", "-C", str(ROOT / "oracle")], capture_output=True, text=True)
    if verbose:
        print(r.stdout, r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    return ROOT / "oracle" / "liboracle.so"


def main() -> None:
    verbose = "-v" in sys.argv
    print(build_native(verbose))
    print(build_oracle(verbose))


if __name__ == "__main__":
    main()
