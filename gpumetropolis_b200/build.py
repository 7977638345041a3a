"""Build the B200 backend's shared library in-tree with nvcc (sm_100a).

``python -m gpumetropolis_b200.build`` writes ``gpumetropolis_b200/libgpum_b200.so``.
The library is the C ABI declared in ``include/gpum_b200.h``; Python loads it
with ctypes (``gpumetropolis_b200._native``).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgpum_b200.so")
SOURCES = ["capi.cu", "program.cpp", "codegen.cpp", "jit.cpp", "noalloc.cu", "mlp.cu"]
HEADERS = ["device.cuh", "interp.cuh", "kernels.cuh", "common.cuh", "compiled.cuh",
           "program.hpp", "codegen.hpp", "jit.hpp", "tc_gemm.cuh"]
# Headers the compiled engine hands to NVRTC at run time, embedded as strings.
EMBED = [("kEmbeddedDevice", "device.cuh"), ("kEmbeddedCommon", "common.cuh"),
         ("kEmbeddedCompiled", "compiled.cuh")]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def host_compiler() -> list:
    # nvcc picks `gcc` from PATH; pin the system one when present.
    return ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "gpum_b200.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def write_embedded() -> str:
    """Write csrc/_embedded.inc: the NVRTC headers as raw string literals."""
    out = os.path.join(CSRC, "_embedded.inc")
    parts = ["// generated by build.py from the kernel headers; do not edit\n"]
    for name, fn in EMBED:
        src = open(os.path.join(CSRC, fn)).read()
        assert ")GPUMSRC\"" not in src
        parts.append(f'static const char* {name} = R"GPUMSRC({src})GPUMSRC";\n')
    text = "".join(parts)
    if not os.path.exists(out) or open(out).read() != text:
        with open(out, "w") as f:
            f.write(text)
    return out


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every source to an object in parallel, then link the library."""
    if not force and not _stale():
        return LIB
    write_embedded()
    from concurrent.futures import ThreadPoolExecutor
    import tempfile
    common = [nvcc(), *host_compiler(), *ARCH, "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "-I", os.path.join(ROOT, "include")]
    if verbose:
        common.insert(1, "-Xptxas=-v")
    with tempfile.TemporaryDirectory(prefix="gpum_build_") as tmpdir:
        def compile_one(f):
            obj = os.path.join(tmpdir, f + ".o")
            cmd = common + ["-c", os.path.join(CSRC, f), "-o", obj]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            subprocess.run(cmd, check=True)
            return obj
        with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
            objs = list(ex.map(compile_one, SOURCES))
        tmp = LIB + f".{os.getpid()}.tmp"
        subprocess.run([nvcc(), *host_compiler(), *ARCH, "--shared", "-o", tmp, *objs,
                        "-lcudart", "-ldl"], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
