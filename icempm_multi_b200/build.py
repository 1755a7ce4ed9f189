"""Build recipe for the in-tree native libraries.

``build()`` compiles, into this package directory (so they travel with the
source tree):
  * ``libicempm_b200.so`` -- CUDA kernels for sm_100a + the C-ABI of
    ``include/icempm.h`` + the host-side C++ of ``csrc/`` (nvcc);
  * ``libicempm_host.so`` -- the C++ host layer of ``host/`` (icy::Model,
    GPU_Implementation5, HostSideSOA, SnapshotManager, the HDF5 point-cloud
    reader; C entry points in ``include/icempm_host.h``), linked to the former;
  * ``icy_cli`` -- the headless driver (``host/icy_cli.cpp``).
Run ``python -m icempm_multi_b200.build``.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libicempm_b200.so")
HOST = os.path.join(HERE, "host")
HOST_LIB = os.path.join(HERE, "libicempm_host.so")
CLI = os.path.join(HERE, "icy_cli")
HOST_SOURCES = ["h5lite.cpp", "icy_host.cpp", "capi_host.cpp"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_SOURCES = ["capi.cu", "instance.cu", "noalloc.cu", "batch.cu", "batch_cargs.cu", "batch_uargs.cu", "partition.cu"]
CXX_SOURCES = ["params.cpp", "scene.cpp"]


def _sources():
    return [os.path.join(CSRC, s) for s in CUDA_SOURCES + CXX_SOURCES]


def _deps(dirs=None):
    out = []
    for d in dirs or (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if f.endswith((".cu", ".cuh", ".cpp", ".h", ".hpp")):
                out.append(os.path.join(d, f))
    return out


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in _deps())


def _host_needs_build():
    if not (os.path.exists(HOST_LIB) and os.path.exists(CLI)):
        return True
    t = min(os.path.getmtime(HOST_LIB), os.path.getmtime(CLI))
    return any(os.path.getmtime(f) > t for f in _deps((HOST, os.path.join(ROOT, "include")))) or \
        os.path.getmtime(LIB) > t


def _run(cmd, what, verbose):
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or r.returncode != 0:
        sys.stdout.write(r.stdout)
        sys.stderr.write(r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"building {what} failed")


def build_host(verbose=False, force=False):
    """libicempm_host.so and icy_cli (g++, C++17), linked to libicempm_b200.so."""
    if not force and not _host_needs_build():
        return HOST_LIB
    cxx = os.environ.get("CXX", "g++")
    inc = ["-I", os.path.join(ROOT, "include")]
    common = ["-O2", "-std=c++17", "-Wall", "-Wno-unused-result", *inc]
    rpath = "-Wl,-rpath,$ORIGIN"
    _run([cxx, *common, "-shared", "-fPIC", "-o", HOST_LIB + ".tmp",
          *[os.path.join(HOST, s) for s in HOST_SOURCES], "-L", HERE, "-licempm_b200", "-lz", rpath],
         "libicempm_host.so", verbose)
    os.replace(HOST_LIB + ".tmp", HOST_LIB)
    _run([cxx, *common, "-o", CLI + ".tmp", os.path.join(HOST, "icy_cli.cpp"), "-L", HERE,
          "-licempm_host", "-licempm_b200", "-lpthread", rpath], "icy_cli", verbose)
    os.replace(CLI + ".tmp", CLI)
    return HOST_LIB


def build(verbose=False, force=False):
    if not force and not needs_build():
        build_host(verbose=verbose, force=force)
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
           "-Xptxas", "-v" if verbose else "-O3",
           "-I", os.path.join(ROOT, "include"), "-o", LIB + ".tmp", *_sources(), "-lcudart"]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or r.returncode != 0:
        sys.stdout.write(r.stdout)
        sys.stderr.write(r.stderr)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed building libicempm_b200.so")
    os.replace(LIB + ".tmp", LIB)
    build_host(verbose=verbose, force=True)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force=True)
    print(LIB)
