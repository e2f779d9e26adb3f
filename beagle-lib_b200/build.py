"""Build recipe of libbeagle_b200.so: nvcc for the sm_100a kernels (k_*.cu),
g++ for the host instance and the C ABI, linked in-tree into ``lib/``.

    python beagle-lib_b200/build.py            # incremental
    python beagle-lib_b200/build.py --clean

Object files go to ``_build/`` at the repository root (git-ignored).

When the BEAGLE sources are at hand (their folder in ``BEAGLE_REF``; no
default), it also builds ``lib/libhmsbeagle-cuda.so.40.0.0``: the plugin that
lets the stock libhmsbeagle.so dispatcher run on this library
(``plugin/b200_plugin.cpp``, compiled against the dispatcher's public headers
BeagleImpl.h / Plugin.h / beagle.h).  Without them the plugin is not rebuilt.
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
OBJ = os.path.join(ROOT, "_build", "beagle_b200")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
LIBNAME = "libbeagle_b200.so"
PLUGIN = "libhmsbeagle-cuda.so.40.0.0"     # name the dispatcher dlopens (PLUGIN_VERSION 40)
PLUGIN_SRC = os.path.join(HERE, "plugin", "b200_plugin.cpp")
BEAGLE_REF = os.environ.get("BEAGLE_REF", "")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
INC = ["-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"] + INC
CXX_FLAGS = ["-O2", "-fPIC", "-std=c++17", "-Wall", "-Wno-unused-function",
             "-I" + os.path.join(CUDA, "include")] + INC


def _sources():
    cu = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    cpp = sorted(f for f in os.listdir(CSRC) if f.endswith(".cpp"))
    return cu, cpp


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(ROOT, "include", "beagle_b200.h"))
    return hs


def _stale(src, obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return os.path.getmtime(src) > t or any(os.path.getmtime(d) > t for d in deps)


def _compile(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    return cmd, r.returncode, r.stdout + r.stderr


def build(verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    cu, cpp = _sources()
    deps = _headers()
    jobs, objs = [], []
    for f in cu:
        src, obj = os.path.join(CSRC, f), os.path.join(OBJ, f + ".o")
        objs.append(obj)
        if _stale(src, obj, deps):
            jobs.append([NVCC] + NVCC_FLAGS + ["-c", src, "-o", obj])
    for f in cpp:
        src, obj = os.path.join(CSRC, f), os.path.join(OBJ, f + ".o")
        objs.append(obj)
        if _stale(src, obj, deps):
            jobs.append(["g++"] + CXX_FLAGS + ["-c", src, "-o", obj])
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        for cmd, rc, out in ex.map(_compile, jobs):
            if verbose or rc:
                print(" ".join(cmd))
                print(out)
            if rc:
                raise RuntimeError(f"compile failed: {cmd[-3]}")
    lib = os.path.join(LIBDIR, LIBNAME)
    if jobs or not os.path.exists(lib):
        cmd = [NVCC] + ARCH + ["-shared", "-o", lib] + objs + ["-lcudart_static", "-lrt", "-ldl",
                                                                 "-lpthread", "-Xlinker",
                                                                 "-soname=" + LIBNAME]
        cmd, rc, out = _compile(cmd)
        if rc:
            print(" ".join(cmd))
            print(out)
            raise RuntimeError("link failed")
    build_plugin(lib, verbose)
    return lib


def build_plugin(lib, verbose=False):
    """libhmsbeagle-cuda.so.40.0.0 beside libbeagle_b200.so (run path
    $ORIGIN).  Returns its path, or None when the BEAGLE headers are absent."""
    ref = os.environ.get("BEAGLE_REF", BEAGLE_REF)
    hdr = os.path.join(ref, "libhmsbeagle", "BeagleImpl.h")
    out = os.path.join(LIBDIR, PLUGIN)
    if not ref or not os.path.exists(hdr):
        return out if os.path.exists(out) else None
    deps = [PLUGIN_SRC, lib, os.path.join(ROOT, "include", "beagle_b200.h")]
    if os.path.exists(out) and all(os.path.getmtime(d) <= os.path.getmtime(out) for d in deps):
        return out
    cmd = ["g++", "-std=c++11", "-O2", "-fPIC", "-shared", "-Wall", "-Wno-unused-function",
           "-Wno-delete-non-virtual-dtor", "-I" + ref, "-I" + os.path.join(ROOT, "include"), PLUGIN_SRC, "-o", out,
           "-L" + LIBDIR, "-l:" + LIBNAME, "-Wl,-soname," + PLUGIN, "-Wl,-rpath,$ORIGIN"]
    cmd, rc, outp = _compile(cmd)
    if verbose or rc:
        print(" ".join(cmd))
        print(outp)
    if rc:
        raise RuntimeError("plugin build failed")
    return out


if __name__ == "__main__":
    if "--clean" in sys.argv:
        shutil.rmtree(OBJ, ignore_errors=True)
    print(build(verbose="-v" in sys.argv))
