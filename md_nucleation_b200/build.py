"""Builds in-tree: md_nucleation_b200/lib/libmdn.so (the engine),
lib/libmdn_host.so and bin/mdn_run (the C++ host).

nvcc compiles the CUDA sources for sm_100a only.  --fmad=false keeps FP64
expressions rounding like the reference's x86 build; the FP32 pair kernels
request fused multiply-adds explicitly with fmaf().
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libmdn.so")
SOURCES = ["advance.cu", "advance_fp64.cu", "advance_gg.cu", "advance_gg_fp64.cu", "snapshot.cu", "snapshot_noalloc.cu", "adjoint.cu", "place.cu", "engine.cu"]
HOST = os.path.join(HERE, "host")
HOST_SOURCES = ["mdn_host.cpp"]
HOST_LIB = os.path.join(LIB_DIR, "libmdn_host.so")
BIN_DIR = os.path.join(HERE, "bin")
HOST_BIN = os.path.join(BIN_DIR, "mdn_run")
HEADERS = ["mdn_types.h", "device_util.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "--fmad=false", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "mdn.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


OBJ_DIR = os.path.join(HERE, "_build")


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles every CUDA source to an object concurrently (the step kernel
    is compiled four times: FP32 / FP64 pair terms, with and without the
    gas-gas term), then links lib/libmdn.so."""
    if force or _stale():
        os.makedirs(LIB_DIR, exist_ok=True)
        os.makedirs(OBJ_DIR, exist_ok=True)
        inc = ["-I", os.path.join(ROOT, "include"), "-I", CSRC]
        procs, objs = [], []
        for src in SOURCES:
            obj = os.path.join(OBJ_DIR, os.path.splitext(src)[0] + ".o")
            cmd = [nvcc()] + NVCC_FLAGS + inc + ["-c", os.path.join(CSRC, src), "-o", obj]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            procs.append((cmd, subprocess.Popen(cmd)))
            objs.append(obj)
        for cmd, p in procs:
            if p.wait() != 0:
                raise subprocess.CalledProcessError(p.returncode, cmd)
        cmd = [nvcc()] + NVCC_FLAGS + ["-shared"] + objs + ["-o", LIB + ".tmp"]
        subprocess.run(cmd, check=True)
        os.replace(LIB + ".tmp", LIB)
    build_host(force=force, verbose=verbose)
    return LIB


def cxx():
    for c in ("/usr/bin/g++", os.environ.get("CXX"), shutil.which("g++")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("g++ not found")


def _host_stale():
    outs = [HOST_LIB, HOST_BIN]
    if not all(os.path.exists(o) for o in outs):
        return True
    t = min(os.path.getmtime(o) for o in outs)
    deps = [os.path.join(HOST, f) for f in HOST_SOURCES + ["mdn_host.h", "mdn_run.cpp"]]
    deps += [LIB, os.path.join(ROOT, "include", "mdn.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build_host(force: bool = False, verbose: bool = False):
    """The C++ host: lib/libmdn_host.so (condition files, placement, run
    cadence, output files) and bin/mdn_run (the command line), both linked
    against lib/libmdn.so."""
    if not force and not _host_stale():
        return
    os.makedirs(BIN_DIR, exist_ok=True)
    inc = ["-I", os.path.join(ROOT, "include"), "-I", HOST]
    lib = ["-L", LIB_DIR, "-lmdn", "-Wl,-rpath,$ORIGIN", "-Wl,-rpath,$ORIGIN/../lib"]
    cmd = [cxx(), "-O2", "-std=c++17", "-fPIC", "-shared", "-Wall"] + inc
    cmd += [os.path.join(HOST, f) for f in HOST_SOURCES] + ["-o", HOST_LIB + ".tmp"] + lib
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(HOST_LIB + ".tmp", HOST_LIB)
    cmd = [cxx(), "-O2", "-std=c++17", "-Wall"] + inc + [os.path.join(HOST, "mdn_run.cpp"), "-o", HOST_BIN + ".tmp",
                                                         "-L", LIB_DIR, "-lmdn_host"] + lib
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(HOST_BIN + ".tmp", HOST_BIN)


def ptxas_report() -> str:
    """Registers / spills / shared memory of the kernels (-Xptxas -v)."""
    cmd = [nvcc()] + NVCC_FLAGS + ["-Xptxas", "-v", "-c", "-I", os.path.join(ROOT, "include"), "-I", CSRC,
                                   os.path.join(CSRC, "advance.cu"), "-o", os.devnull]
    r = subprocess.run(cmd, capture_output=True, text=True)
    return r.stderr


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
