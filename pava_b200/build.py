"""Builds the engine's shared libraries in-tree for sm_100a.

    python -m pava_b200.build

* ``pava_b200/lib/libpava_gpu.so``  -- the CUDA engine and its C ABI (include/pava_gpu.h)
* ``pava_b200/lib/libpava_host.so`` -- host-side C++: seeded matrix generators, the Matrix
  Market reader/writer and the COO->CSR conversion (include/pava_host.h)
* ``pava_b200/lib/pava_bench``      -- main.cpp's CVR / CSR5 benchmark loop over the C ABI
* ``pava_b200/lib/libpava_probe.so`` -- floor kernels for measurements (include/pava_probe.h)
* ``pava_b200/lib/libpava_gpu_bounds.so`` -- the engine built with PAVA_BOUNDS_CHECK: every
  data-derived index tested, failures counted instead of faulting (load it with PAVA_GPU_LIB)

nvcc cross-compiles for sm_100a without a GPU, so this runs on any machine with the CUDA
toolkit.  CUDA runtime is linked statically, so the library does not depend on the
toolkit's shared runtime at load time.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
GPU_SOURCES = ["api.cu", "k_support.cu", "k_cvr.cu", "k_csr5.cu", "k_group.cu", "noalloc.cu",
               "batch.cu", "k_gen.cu", "k_features.cu", "k_mlp.cu", "select.cu", "k_coo.cu",
               "k_sell.cu", "k_sell_spmm.cu"]
HOST_SOURCES = ["host/gen.cpp", "host/mtx.cpp"]


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build_gpu(force: bool = False, verbose_ptxas: bool = False, out: str | None = None,
              extra: tuple = ()) -> str:
    """libpava_gpu.so; `out` and `extra` (nvcc flags such as -D macros) build a variant of it
    elsewhere, e.g. with other launch bounds for a tuning sweep (loaded through PAVA_GPU_LIB)."""
    os.makedirs(LIBDIR, exist_ok=True)
    out = out or os.path.join(LIBDIR, "libpava_gpu.so")
    srcs = [os.path.join(CSRC, s) for s in GPU_SOURCES]
    deps = srcs + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".h", ".cuh"))]
    deps.append(os.path.join(ROOT, "include", "pava_gpu.h"))
    if not force and not _stale(out, deps):
        return out
    objdir = os.path.join(os.path.dirname(out), "obj" if not extra else
                          "obj_" + os.path.splitext(os.path.basename(out))[0])
    os.makedirs(objdir, exist_ok=True)
    objs, cmds = [], []
    for s in srcs:
        o = os.path.join(objdir, os.path.basename(s) + ".o")
        cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
               "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include"), *extra,
               "-c", s, "-o", o]
        if verbose_ptxas:
            cmd.insert(1, "-Xptxas=-v")
        cmds.append(cmd)
        objs.append(o)
    # the translation units compile independently: one nvcc per core
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        list(ex.map(_run, cmds))
    _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", out, *objs])
    return out


def build_host(force: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    out = os.path.join(LIBDIR, "libpava_host.so")
    srcs = [os.path.join(CSRC, s) for s in HOST_SOURCES]
    deps = srcs + [os.path.join(ROOT, "include", "pava_host.h")]
    if not force and not _stale(out, deps):
        return out
    _run(["g++", "-O2", "-fPIC", "-fopenmp", "-std=c++17", "-shared", "-I",
          os.path.join(ROOT, "include"), "-o", out, *srcs])
    return out


def build_driver(force: bool = False) -> str:
    """pava_bench: main.cpp's CVR / CSR5 benchmark loop over the C ABI (csrc/host/pava_bench.cpp)."""
    out = os.path.join(LIBDIR, "pava_bench")
    src = os.path.join(CSRC, "host", "pava_bench.cpp")
    deps = [src, os.path.join(LIBDIR, "libpava_gpu.so"), os.path.join(LIBDIR, "libpava_host.so"),
            os.path.join(ROOT, "include", "pava_gpu.h"), os.path.join(ROOT, "include", "pava_host.h")]
    if not force and not _stale(out, deps):
        return out
    _run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), src, "-o", out,
          "-L", LIBDIR, "-lpava_gpu", "-lpava_host", "-Wl,-rpath,$ORIGIN"])
    return out


def build_probe(force: bool = False) -> str:
    """libpava_probe.so: the floor kernels of include/pava_probe.h (measurement aids)."""
    os.makedirs(LIBDIR, exist_ok=True)
    out = os.path.join(LIBDIR, "libpava_probe.so")
    src = os.path.join(CSRC, "k_probe.cu")
    deps = [src, os.path.join(CSRC, "pava_common.cuh"), os.path.join(CSRC, "k_bulk.cuh"),
            os.path.join(ROOT, "include", "pava_probe.h")]
    if not force and not _stale(out, deps):
        return out
    _run([NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
          "-cudart", "static", "-o", out, src])
    return out


def build_bounds(force: bool = False) -> str:
    """libpava_gpu_bounds.so: the engine with PAVA_BOUNDS_CHECK, whose SpMV kernels test every
    data-derived index and count failures instead of faulting (pava_bounds_report).  Load it
    through PAVA_GPU_LIB, e.g. to run the GPU test suite under the checks."""
    return build_gpu(force=force, out=os.path.join(LIBDIR, "libpava_gpu_bounds.so"),
                     extra=("-DPAVA_BOUNDS_CHECK",))


def build(force: bool = False) -> None:
    with ThreadPoolExecutor(max_workers=2) as ex:
        fp = ex.submit(build_probe, force)
        build_host(force)
        build_gpu(force)
        build_bounds(force)
        fp.result()
    build_driver(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
