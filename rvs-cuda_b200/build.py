"""Builds the native library librvsb.so (and the rvsb CLI) in-tree.

CUDA sources are compiled for sm_100a only; host C++ with -ffp-contract=off so
the float camera math keeps the reference's rounding.  Output goes to
rvs-cuda_b200/lib/.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib")
INCLUDE = os.path.join(ROOT, "include")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

CU_SOURCES = ["launch.cu", "decode.cu", "warp.cu", "bin.cu", "tile.cu", "inpaint.cu", "noalloc.cu", "aux.cu", "ms.cu",
              "resize.cu",
              "raster_v0.cu", "raster_v1.cu", "raster_v2.cu", "raster_v3.cu", "raster_v4.cu", "raster_v5.cu",
              "raster_v6.cu", "raster_v7.cu"]
CPP_SOURCES = ["api.cpp", "engine.cpp", "server.cpp", "frontend.cpp", "camera.cpp"]
CLI_SOURCES = ["rvsb_cli.cpp"]
SCENEGEN_SOURCES = ["scenegen.cpp"]

GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = GENCODE + ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC",
                        "-Xptxas", "-v", "--expt-relaxed-constexpr"]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall", "-Wextra",
             "-Wno-unused-parameter"]

LIB_PATH = os.path.join(LIB, "librvsb.so")
SCENEGEN_PATH = os.path.join(LIB, "libscenegen.so")
CLI_PATH = os.path.join(LIB, "rvsb")


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh", ".h"))]
    hs.append(os.path.join(INCLUDE, "rvsb.h"))
    return hs


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, log=None):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if log is not None:
        with open(log, "w") as f:
            f.write(" ".join(cmd) + "\n" + r.stdout)
    if r.returncode != 0:
        sys.stderr.write(r.stdout)
        raise RuntimeError("build step failed: " + " ".join(cmd))
    return r.stdout


def build(force=False, verbose=False):
    """Compiles stale objects and links librvsb.so and the CLI.  Returns the
    library path."""
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIB, exist_ok=True)
    headers = _headers()
    jobs = []
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            jobs.append(([NVCC] + NVCC_FLAGS + ["-I", INCLUDE, "-I", CSRC, "-c", s, "-o", o],
                         os.path.join(OBJ, src + ".log")))
    for src in CPP_SOURCES + CLI_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        if src in CPP_SOURCES:
            objs.append(o)
        if force or _stale(o, [s] + headers):
            jobs.append((["g++"] + CXX_FLAGS + ["-I", INCLUDE, "-I", CSRC, "-I",
                                                os.path.join(CUDA_HOME, "include"), "-c", s, "-o", o],
                         os.path.join(OBJ, src + ".log")))
    with ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as ex:
        outs = list(ex.map(lambda j: _run(*j), jobs))
    if verbose:
        for o in outs:
            print(o)
    if force or _stale(LIB_PATH, objs):
        _run([NVCC] + GENCODE + ["-shared", "-o", LIB_PATH] + objs +
             ["-Xlinker", "-soname=librvsb.so", "-lcudart_static", "-ldl", "-lrt", "-lpthread"])
    cli_obj = os.path.join(OBJ, CLI_SOURCES[0] + ".o")
    if force or _stale(CLI_PATH, [cli_obj, LIB_PATH]):
        _run(["g++", "-o", CLI_PATH, cli_obj, "-L", LIB, "-lrvsb", "-Wl,-rpath,$ORIGIN",
              "-L", os.path.join(CUDA_HOME, "lib64"), "-lcudart"])
    sg = os.path.join(CSRC, SCENEGEN_SOURCES[0])
    if force or _stale(SCENEGEN_PATH, [sg]):
        _run(["g++", "-O3", "-std=c++17", "-fPIC", "-fopenmp", "-shared", "-o", SCENEGEN_PATH, sg])
    return LIB_PATH


def ptxas_report():
    """The -Xptxas -v output of the CUDA objects (registers, spills, smem)."""
    out = []
    for src in CU_SOURCES:
        log = os.path.join(OBJ, src + ".log")
        if os.path.exists(log):
            out.append(open(log).read())
    return "\n".join(out)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB_PATH)
