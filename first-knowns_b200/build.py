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
    "-Xcompiler", "-fPIC",
    "-Xptxas", "-v",
]
OBJ = HERE / "_obj"


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
    """Compile libfk.so if any source is newer than it (or force): every
    translation unit in csrc/ to an object, in parallel (the kernel
    variants sit in units of their own), then one shared-library link."""
    if not force and not needs_build():
        return LIB
    OBJ.mkdir(exist_ok=True)
    units = sorted(CSRC.glob("*.cu"))
    jobs = []
    for cu in units:
        obj = OBJ / (cu.stem + ".o")
        cmd = [NVCC] + FLAGS + ["-c", "-o", str(obj), str(cu)]
        jobs.append((cu, obj, subprocess.Popen(
            cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
            text=True)))
    log, failed = [], []
    for cu, obj, proc in jobs:
        out = proc.communicate()[0]
        log.append(f"== {cu.name}\n{out}")
        if proc.returncode != 0:
            failed.append(cu.name)
    if not failed:
        cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a",
               "-shared", "-o", str(LIB) + ".tmp"] + \
              [str(o) for _, o, _ in jobs]
        res = subprocess.run(cmd, capture_output=True, text=True)
        log.append("== link\n" + res.stdout + res.stderr)
        if res.returncode != 0:
            failed.append("link")
    text = "".join(log)
    (HERE / "build.log").write_text(text)
    if failed:
        raise RuntimeError("nvcc failed (" + ", ".join(failed) + "):\n" +
                           text[-6000:])
    os.replace(str(LIB) + ".tmp", LIB)
    if verbose:
        print(text)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
