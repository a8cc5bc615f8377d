"""In-tree build of the native parts of nise_2017_b200.

Products (all written next to this file, so they travel with the source tree):
  libnise_b200.so   the engine: CUDA kernels for sm_100a + the C ABI (include/nise_b200.h)
  libnise_synth.so  the seeded synthetic GROBIN trajectory generator
  nise              the NISE-compatible C driver (keyword file in, output files out)
  nise2dfft         the 2DFFT-compatible driver
  nise_translate    the translate-compatible trajectory format converter

Usage: python -m nise_2017_b200.build  (or build_all() from Python).
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = [
    "absorption.cu",
    "fft.cu",
    "twodir.cu",
    "eigen.cu",
    "util.cu",
    "noalloc.cu",
    "fft2d.cu",
    "diag.cu",
    "adjoint.cu",
    "onfly.cu",
    "linear.cu",
    "taylor_rv.cu",
    "eigen_large.cu",
    "dia_tc.cu",
]
CPP_SOURCES = [
    "api.cpp",
    "absrun.cpp",
    "input.cpp",
    "singles.cpp",
    "translate.cpp",
]


def _run(cmd, cwd=None):
    r = subprocess.run(cmd, cwd=cwd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout)
        raise RuntimeError("build step failed: %s" % cmd[0])
    return r.stdout


def _newer(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _deps(pattern_dirs, exts):
    out = []
    for d in pattern_dirs:
        for f in os.listdir(d):
            if f.endswith(exts):
                out.append(os.path.join(d, f))
    return out


def build_synth(force=False):
    out = os.path.join(HERE, "libnise_synth.so")
    srcs = [os.path.join(CSRC, "synth.c"), os.path.join(CSRC, "nise_synth.h")]
    if force or _newer(out, srcs):
        _run(["gcc", "-std=gnu99", "-O2", "-fPIC", "-shared", "-o", out, srcs[0], "-lm"])
    return out


def build_engine(force=False, verbose_ptxas=False):
    out = os.path.join(HERE, "libnise_b200.so")
    deps = _deps([CSRC, INCLUDE], (".cu", ".cuh", ".cpp", ".h", ".hpp"))
    if not (force or _newer(out, deps)):
        return out
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    common = ["-O3", "-std=c++17", "-I" + INCLUDE, "-I" + CSRC, "-Xcompiler", "-fPIC"]
    for s in CU_SOURCES:
        o = os.path.join(objdir, s + ".o")
        cmd = [NVCC] + ARCH + common + ["-lineinfo", "-c", os.path.join(CSRC, s), "-o", o]
        if verbose_ptxas:
            cmd.insert(1, "-Xptxas=-v")
        _run(cmd)
        objs.append(o)
    for s in CPP_SOURCES:
        o = os.path.join(objdir, s + ".o")
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-I" + INCLUDE, "-I" + CSRC,
              "-I" + os.path.join(CUDA_HOME, "include"), "-c", os.path.join(CSRC, s), "-o", o])
        objs.append(o)
    _run([NVCC] + ARCH + ["-shared", "-o", out] + objs +
         ["-lcudart_static", "-ldl", "-lrt", "-lpthread", "-Xlinker", "--no-undefined"])
    return out


def build_driver(force=False):
    """The drop-in executables: nise (NISE's propagation path), nise2dfft (2DFFT)
    and nise_translate (translate)."""
    for exe, c in (("nise", "nise_main.c"), ("nise2dfft", "nise2dfft_main.c"),
                   ("nise_translate", "nise_translate_main.c")):
        out = os.path.join(HERE, exe)
        src = os.path.join(CSRC, c)
        if force or _newer(out, [src, os.path.join(INCLUDE, "nise_b200.h")]):
            _run(["gcc", "-std=gnu99", "-O2", "-I" + INCLUDE, "-o", out, src,
                  "-L" + HERE, "-lnise_b200", "-Wl,-rpath,$ORIGIN", "-lm"])
    return os.path.join(HERE, "nise")


def build_all(force=False):
    build_synth(force)
    build_engine(force)
    build_driver(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print("built:", ", ".join(f for f in os.listdir(HERE) if f.endswith(".so") or f in ("nise", "nise2dfft", "nise_translate")))
