"""Build libfk.so in-tree for sm_100a (B200) with nvcc.

    python first-knowns_b200/build.py [--force]

The library lands beside this file (first-knowns_b200/libfk.so), where
fk_abi.py loads it.  No other architecture is compiled.
"""

import os
import pathlib
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIB = HERE / "libfk.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
    "-Xptxas", "-v",
]


def sources():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) +
                  list(CSRC.glob("*.h")) +
                  [HERE.parent / "include" / "fk.h"])


def needs_build():
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources())


def build(force=False, verbose=False):
    """Compile libfk.so if any source is newer than it (or force)."""
    if not force and not needs_build():
        return LIB
    cmd = [NVCC] + FLAGS + ["-o", str(LIB) + ".tmp",
                            str(CSRC / "fk_engine.cu"),
                            str(CSRC / "fk_noalloc.cu")]
    res = subprocess.run(cmd, capture_output=True, text=True)
    log = res.stdout + res.stderr
    (HERE / "build.log").write_text(log)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + log[-6000:])
    os.replace(str(LIB) + ".tmp", LIB)
    if verbose:
        print(log)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
