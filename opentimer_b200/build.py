"""Build libotg.so in-tree with nvcc for sm_100a (B200).

    python -m opentimer_b200.build        # or opentimer_b200.build.build()

Objects go to opentimer_b200/_build/, the shared library to
opentimer_b200/libotg.so (git-ignored; it travels with the source tree).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libotg.so")
SOURCES = ["otg_rc.cu", "otg_levelize.cu", "otg_synth.cu", "otg_host.cu", "otg_noalloc.cu",
           "otg_serve.cu", "otg_spef.cpp", "otg_prop.cu", "otg_move.cu", "otg_sizing.cu", "otg_spef_write.cpp",
           "otg_csr.cu", "otg_paths.cpp"]
CXX = os.environ.get("CXX", "g++")
CXXFLAGS = ["-O3", "-std=c++17", "-fPIC", "-pthread", "-Wall"]

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "--expt-relaxed-constexpr"] + ARCH


def _newer(src_list, target):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in src_list)


def build(verbose=False, extra_flags=()):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers += [os.path.join(HERE, "..", "include", f)
                for f in os.listdir(os.path.join(HERE, "..", "include"))]
    objs = []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, os.path.splitext(s)[0] + ".o")
        objs.append(obj)
        if _newer([src] + headers, obj):
            if s.endswith(".cpp"):  # host-only C++
                cmd = [CXX] + CXXFLAGS + ["-c", src, "-o", obj]
            else:
                cmd = [NVCC] + FLAGS + list(extra_flags) + ["-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if _newer(objs, LIB):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-Xcompiler", "-pthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, extra_flags=sys.argv[1:])
