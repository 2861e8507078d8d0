"""Builds libinfraga_gpu.so (and the drop-in CLI binaries) in-tree with nvcc
for sm_100a.  Run as ``python -m infraga_b200.build`` or via
``__graft_entry__.build()``.  Rebuilds only when a source is newer than the
library."""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libinfraga_gpu.so")
BIN_DIR = os.path.join(ROOT, "bin")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-O2",
              "-Xptxas", "-warn-spills"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libinfraga_gpu.so")


def _host_cxx() -> list[str]:
    # The system g++ links libstdc++ dynamically, so the library shares the
    # C++ runtime already loaded by Python/numpy/torch processes.
    return ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_lib(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(LIB_DIR, exist_ok=True)
    srcs = sources()
    deps = srcs + glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        [os.path.join(ROOT, "include", "infraga_gpu.h")]
    if not force and not _stale(LIB, deps):
        return LIB
    cmd = [_nvcc(), *_host_cxx(), *ARCH, *NVCC_FLAGS, "-shared", "-o", LIB + ".tmp", *srcs,
           "-Xlinker", "--exclude-libs,ALL"]
    if verbose:
        cmd += ["-Xptxas", "-v"]
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building libinfraga_gpu.so")
    if verbose:
        sys.stderr.write(r.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


def build_cli(verbose: bool = False, force: bool = False) -> list[str]:
    """Drop-in command-line binaries (bin/infraga-3d ...) linked against the library."""
    cli_dir = os.path.join(CSRC, "cli")
    mains = sorted(glob.glob(os.path.join(cli_dir, "main_*.cpp")))
    if not mains:
        return []
    os.makedirs(BIN_DIR, exist_ok=True)
    out = []
    common = sorted(glob.glob(os.path.join(cli_dir, "cli_*.cpp")))
    deps_common = common + glob.glob(os.path.join(cli_dir, "*.h")) + [LIB]
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    for m in mains:
        name = os.path.basename(m)[len("main_"):-len(".cpp")].replace("_", "-")
        target = os.path.join(BIN_DIR, name)
        if not force and not _stale(target, [m] + deps_common):
            out.append(target)
            continue
        cmd = [cxx, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), m, *common,
               "-L", LIB_DIR, "-linfraga_gpu", "-Wl,-rpath," + LIB_DIR, "-o", target]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"building {name} failed")
        out.append(target)
    return out


def build(verbose: bool = False, force: bool = False) -> None:
    build_lib(verbose=verbose, force=force)
    build_cli(verbose=verbose, force=force)


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
