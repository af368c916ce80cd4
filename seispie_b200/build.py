"""Build libseispie_b200.so (the C-ABI CUDA library) in-tree for sm_100a.

    python -m seispie_b200.build [--verbose]

The library is written to seispie_b200/_build/libseispie_b200.so, next to the
package, so that it is found without installation.  The CUDA runtime is
linked statically; the library shares the process's primary CUDA context with
PyTorch, so device pointers and streams from torch can be passed to it.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OUT_DIR = os.path.join(PKG, "_build")
LIB = os.path.join(OUT_DIR, "libseispie_b200.so")
INFO = os.path.join(OUT_DIR, "build_info.json")
SOURCES = ("capi.cu", "step.cu", "march.cu", "aux.cu", "linalg.cu", "noalloc.cu", "unet.cu")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    raise RuntimeError("nvcc not found")


def flags(verbose: bool = False):
    f = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include"),
                "--expt-relaxed-constexpr"]
    if verbose:
        f += ["-Xptxas", "-v"]
    return f


def build(verbose: bool = False, force: bool = False) -> str:
    """Compile every .cu source and link the shared library; returns its path.
    Skips the work when the library is newer than every source."""
    os.makedirs(OUT_DIR, exist_ok=True)
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, h) for h in ("common.cuh", "stencil.cuh")] + [os.path.join(ROOT, "include", "seispie_b200.h")]
    if not force and os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(d) for d in deps):
        return LIB
    objs, cmds = [], []
    for s in srcs:
        o = os.path.join(OUT_DIR, os.path.basename(s) + ".o")
        cmd = [nvcc(), "-c", s, "-o", o] + flags(verbose)
        cmds.append(cmd)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or r.returncode:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode:
            raise RuntimeError("nvcc failed on %s" % s)
        objs.append(o)
    tmp = LIB + ".tmp"
    cmd = [nvcc(), "-shared", "-o", tmp] + objs + ARCH + ["-Xcompiler", "-fPIC", "-cudart", "static"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    os.replace(tmp, LIB)
    # the exact commands, for checks of the target architecture without inspecting the binary
    with open(INFO, "w") as f:
        json.dump({"compile": [" ".join(c) for c in cmds], "link": " ".join(cmd), "arch": " ".join(ARCH)}, f,
                  indent=1)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(verbose=a.verbose, force=a.force))
