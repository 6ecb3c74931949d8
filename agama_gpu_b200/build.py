"""Build the in-tree CUDA library agama_gpu_b200/libagb.so for sm_100a.

    python agama_gpu_b200/build.py            # compile if sources changed
    python agama_gpu_b200/build.py --force    # always recompile

(Run it as a script: importing the package needs the library it builds.)

nvcc cross-compiles without a GPU; the .so stays in the source tree so it is
the one Python loads (no JIT cache).
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libagb.so"
STAMP = PKG / ".libagb.stamp"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-shared",
              "--expt-relaxed-constexpr", "-Xptxas", "-v"]
SOURCES = ["eval.cu", "peak.cu"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _digest() -> str:
    h = hashlib.sha256()
    files = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.py"))
    files.append(ROOT / "include" / "agb.h")
    for f in files:
        h.update(f.name.encode())
        h.update(f.read_bytes())
    h.update(" ".join(ARCH + NVCC_FLAGS).encode())
    return h.hexdigest()


def build(force: bool = False, verbose: bool = False) -> Path:
    subprocess.run([sys.executable, str(CSRC / "gen_tables.py")], check=True)
    dig = _digest()
    if not force and LIB.exists() and STAMP.exists() and STAMP.read_text() == dig:
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [_nvcc(), *ARCH, *NVCC_FLAGS, "-I", str(ROOT / "include"),
           *[str(CSRC / s) for s in SOURCES], "-o", str(tmp)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    log = res.stdout + res.stderr
    (PKG / "build.log").write_text(" ".join(cmd) + "\n" + log)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed:\n{log[-4000:]}")
    if verbose:
        print(log)
    tmp.replace(LIB)
    STAMP.write_text(dig)
    return LIB


if __name__ == "__main__":
    p = build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(p)
