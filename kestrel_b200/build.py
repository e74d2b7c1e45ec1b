"""Build recipes for the native libraries, in-tree.

* ``kestrel_b200/libkestrel_cuda.so``: the CUDA backend (sm_100a only), the
  product. Built with nvcc for ``arch=compute_100a,code=sm_100a``.
* ``kestrel_b200/libkestrel_host.so``: the host-side driver that produces the
  backend's per-block inputs (bank, MIDI timeline, gate/channel tables,
  admission), C++17.
* ``kestrel_b200/libkestrel_serve.so``: the render server (continuous
  batching over kc_batch_render, or the plain path one job at a time), C++17,
  linked against the two libraries above.
* ``oracle/liboracle.so``: the CPU restatement of the reference backend, the
  checker used only by the tests and the CPU-baseline legs of the benchmark.

Each target is rebuilt only when one of its sources is newer than the output.
Run ``python -m kestrel_b200.build`` (or ``__graft_entry__.build()``).
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "kestrel_b200"
CSRC = PKG / "csrc"
ORACLE = ROOT / "oracle"
INCLUDE = ROOT / "include"

CUDA_LIB = PKG / "libkestrel_cuda.so"
HOST_LIB = PKG / "libkestrel_host.so"
ORACLE_LIB = ORACLE / "liboracle.so"
SERVE_LIB = PKG / "libkestrel_serve.so"

NVCC_ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.exists(cand) or cand == "nvcc"):
            return cand
    return "nvcc"


def _stale(out: Path, srcs: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(s.stat().st_mtime > t for s in srcs)


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)


def build_cuda(force: bool = False, extra: list[str] | None = None) -> Path:
    srcs = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + [INCLUDE / "kestrel_cuda.h"]
    if force or _stale(CUDA_LIB, srcs):
        tmp = CUDA_LIB.with_suffix(".so.tmp")
        _run([_nvcc(), *NVCC_ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
              "-Xptxas", "-warn-spills", *(extra or []),
              *[str(p) for p in sorted(CSRC.glob("*.cu"))], "-o", str(tmp)])
        os.replace(tmp, CUDA_LIB)
    return CUDA_LIB


def build_host(force: bool = False) -> Path:
    hdir = CSRC / "host"
    srcs = sorted(hdir.glob("*.cpp")) + sorted(hdir.glob("*.h")) + [INCLUDE / "kestrel_host.h",
                                                                    INCLUDE / "kestrel_cuda.h"]
    if not (INCLUDE / "kestrel_host.h").exists():
        return HOST_LIB
    if force or _stale(HOST_LIB, srcs):
        tmp = HOST_LIB.with_suffix(".so.tmp")
        _run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-pthread",
              *[str(p) for p in sorted(hdir.glob("*.cpp"))], "-o", str(tmp)])
        os.replace(tmp, HOST_LIB)
    return HOST_LIB


def build_serve(force: bool = False) -> Path:
    """The render server: links the CUDA backend and the host library."""
    sdir = CSRC / "serve"
    srcs = sorted(sdir.glob("*.cpp")) + [INCLUDE / "kestrel_serve.h", INCLUDE / "kestrel_cuda.h",
                                         INCLUDE / "kestrel_host.h", CUDA_LIB, HOST_LIB]
    if force or _stale(SERVE_LIB, srcs):
        tmp = SERVE_LIB.with_suffix(".so.tmp")
        _run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-pthread",
              *[str(p) for p in sorted(sdir.glob("*.cpp"))], f"-L{PKG}", "-lkestrel_cuda", "-lkestrel_host",
              "-Wl,-rpath,$ORIGIN", "-o", str(tmp)])
        os.replace(tmp, SERVE_LIB)
    return SERVE_LIB


def build_oracle(force: bool = False) -> Path:
    srcs = sorted(ORACLE.glob("*.cpp")) + sorted(ORACLE.glob("*.h")) + [INCLUDE / "kestrel_cuda.h"]
    if force or _stale(ORACLE_LIB, srcs):
        tmp = ORACLE_LIB.with_suffix(".so.tmp")
        _run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-pthread",
              *[str(p) for p in sorted(ORACLE.glob("*.cpp"))], "-o", str(tmp)])
        os.replace(tmp, ORACLE_LIB)
    return ORACLE_LIB


def build_all(force: bool = False) -> None:
    build_host(force)
    build_oracle(force)
    build_cuda(force)
    build_serve(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
