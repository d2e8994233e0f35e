"""Build the sm_100a shared library ``freelb_b200/libflb_b200.so`` in place.

    python -m freelb_b200.build          (or: python freelb_b200/build.py)

nvcc cross-compiles for sm_100a without a GPU.  The library has a plain C ABI
(include/flb.h), links the CUDA runtime statically and has no torch
dependency, so ctypes, the C++17 host classes and any FFI can load it.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libflb_b200.so")
SOURCES = ["flb_api.cu", "flb_noalloc.cu", "flb_boundary.cu"]
DEPS = ["flb_api.cu", "flb_noalloc.cu", "flb_kernels.cuh", "flb_lattice.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise FileNotFoundError("nvcc not found")
    return cand


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    deps = [os.path.join(CSRC, d) for d in DEPS] + [os.path.join(ROOT, "include", "flb.h"),
                                                    os.path.abspath(__file__)]
    deps += [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh"))]
    if not force and not _stale(LIB, deps):
        return LIB
    cmd = [nvcc(), "-std=c++17", *ARCH, "-O3", "-lineinfo", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-fvisibility=hidden", "-shared", "-o", LIB + ".tmp"]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    cmd += [os.path.join(CSRC, s) for s in SOURCES]
    env = dict(os.environ)
    # the image exports CC/CXX pointing at a compiler without OpenMP specs;
    # nvcc only needs a host C++ compiler on PATH
    env.pop("CC", None)
    env.pop("CXX", None)
    res = subprocess.run(cmd, capture_output=True, text=True, env=env)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
    if verbose:
        print(res.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


EXAMPLES = ("cavity3d_b200", "cavity3d_vtk", "periodic3d_b200")
EXAMPLE_SRC = os.path.join(HERE, "cpp", "examples", "cavity3d_b200.cpp")
EXAMPLE_BIN = os.path.join(HERE, "cpp", "_build", "cavity3d_b200")


def build_example(name: str, force: bool = False) -> str:
    """Compile one C++17 host-class example against libflb_b200.so (g++)."""
    src = os.path.join(HERE, "cpp", "examples", name + ".cpp")
    out = os.path.join(HERE, "cpp", "_build", name)
    deps = [src, os.path.join(HERE, "cpp", "freelb.h"), LIB]
    if not force and not _stale(out, deps):
        return out
    os.makedirs(os.path.dirname(out), exist_ok=True)
    cmd = ["g++", "-std=c++17", "-O2", "-o", out, src, "-L" + HERE, "-lflb_b200",
           "-Wl,-rpath,$ORIGIN/../.."]
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    res = subprocess.run(cmd, capture_output=True, text=True, env=env)
    if res.returncode != 0:
        raise RuntimeError("g++ failed:\n" + res.stdout + res.stderr)
    return out


def build_examples(force: bool = False) -> str:
    """Compile every example; returns the cavity example's path."""
    for name in EXAMPLES:
        build_example(name, force)
    return EXAMPLE_BIN


# The reference's own programs, their sources untouched, built against the
# host classes (only the include path differs): kind -> (source under the
# reference root, output name, compiler, extra flags).  The cavity3d example is
# built for both of its FLOAT_TYPE settings (its Makefile uses double).
REF_PROGRAMS = {
    "cpu": ("benchmarks/cavity3d/cavity3d.cpp", "ref_cavity3d", "g++", []),
    "cu": ("benchmarks/cavity3d_cu/cavity3d.cu", "ref_cavity3d_cu", "nvcc", []),
    "example": ("examples/cavity3d/cavity3d.cpp", "ref_example_cavity3d", "g++",
                ["-DFLOAT_TYPE=double"]),
    "example_f32": ("examples/cavity3d/cavity3d.cpp", "ref_example_cavity3d_f32", "g++",
                    ["-DFLOAT_TYPE=float"]),
}


def ref_program_path(kind: str) -> str:
    return os.path.join(HERE, "cpp", "_build", REF_PROGRAMS[kind][1])


def build_reference_program(kind: str, ref_root: str, force: bool = False) -> str:
    """Compile one of the reference's programs (read in place under ref_root)
    against the host classes and libflb_b200.so; returns the executable."""
    rel, _, cc, extra = REF_PROGRAMS[kind]
    src = os.path.join(ref_root, rel)
    out = ref_program_path(kind)
    deps = [src, os.path.join(HERE, "cpp", "freelb.h"), LIB]
    if not force and not _stale(out, deps):
        return out
    os.makedirs(os.path.dirname(out), exist_ok=True)
    inc = os.path.join(HERE, "cpp")
    if cc == "nvcc":
        cmd = [nvcc(), "-std=c++17", *ARCH, "-I" + inc, *extra, src, "-L" + HERE, "-lflb_b200",
               "-Xlinker", "-rpath,$ORIGIN/../..", "-o", out]
    else:
        cmd = ["g++", "-std=c++17", "-O1", "-I" + inc, *extra, src, "-L" + HERE, "-lflb_b200",
               "-Wl,-rpath,$ORIGIN/../..", "-o", out]
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    res = subprocess.run(cmd, capture_output=True, text=True, env=env)
    if res.returncode != 0:
        raise RuntimeError(f"{cc} failed on {rel}:\n" + res.stdout + res.stderr[-4000:])
    return out


def build_reference_programs(ref_root: str, force: bool = False) -> dict:
    """All of REF_PROGRAMS whose source exists under ref_root."""
    return {k: build_reference_program(k, ref_root, force) for k, v in REF_PROGRAMS.items()
            if os.path.exists(os.path.join(ref_root, v[0]))}


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
    print(build_examples(force="--force" in sys.argv))
