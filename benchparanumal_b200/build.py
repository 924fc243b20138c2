"""Build the sm_100a library libbp_b200.so and the BK/BP executables in-tree.

    python -m benchparanumal_b200.build        (or: python benchparanumal_b200/build.py)

nvcc cross-compiles for sm_100a without a GPU.  Objects go to
benchparanumal_b200/_build/, the library to benchparanumal_b200/libbp_b200.so,
the executables to apps/bin/.
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libbp_b200.so")
APPS = ["BP%d" % k for k in range(1, 7)] + ["BK%d" % k for k in range(1, 7)]

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
HOSTCXX = "/usr/bin/g++"   # the system g++ carries libgomp
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-ccbin", HOSTCXX, "-Xcompiler", "-fPIC,-fopenmp,-O3",
                  "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]
CXXFLAGS = ["-O3", "-std=c++17", "-fPIC", "-fopenmp", "-march=x86-64-v3", "-Wall", "-Wno-unknown-pragmas",
            "-I/usr/local/cuda/include"]
HEADERS = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh"))) + [
    os.path.join(ROOT, "include", "bp_b200.h")]


def _newer(src, dst, extra=()):
    if not os.path.exists(dst):
        return True
    t = os.path.getmtime(dst)
    return any(os.path.getmtime(p) > t for p in (src, *extra))


def _compile(src):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if not _newer(src, obj, HEADERS):
        return obj, None
    if src.endswith(".cu"):
        cmd = [NVCC] + CUFLAGS + ["-c", src, "-o", obj]
    else:
        cmd = [HOSTCXX] + CXXFLAGS + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compile failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
    return obj, (r.stdout + r.stderr).strip()


def build(verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        results = list(ex.map(_compile, srcs))
    for _, log in results:
        if log and verbose:
            print(log)
    objs = [o for o, _ in results]
    if any(_newer(o, LIB) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-ccbin", HOSTCXX, "-o", LIB] + objs + ["-Xcompiler", "-fopenmp", "-lgomp"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed: %s\n%s" % (" ".join(cmd), r.stderr))
    bindir = os.path.join(ROOT, "apps", "bin")
    os.makedirs(bindir, exist_ok=True)
    app_src = os.path.join(ROOT, "apps", "bp_app.cpp")
    for name in APPS:
        exe = os.path.join(bindir, name)
        if _newer(app_src, exe, (LIB,)):
            cmd = [HOSTCXX, "-O2", "-std=c++17", '-DBP_APP_NAME="%s"' % name, app_src, "-o", exe,
                   "-L" + PKG, "-lbp_b200", "-Wl,-rpath,$ORIGIN/../../benchparanumal_b200"]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError("app link failed: %s\n%s" % (" ".join(cmd), r.stderr))
    return LIB


def clean():
    shutil.rmtree(BUILD, ignore_errors=True)
    if os.path.exists(LIB):
        os.remove(LIB)


if __name__ == "__main__":
    if "--clean" in sys.argv:
        clean()
    print(build(verbose="-v" in sys.argv))
