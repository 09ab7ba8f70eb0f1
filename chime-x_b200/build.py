"""Build libchimex.so (sm_100a) and the C host program in-tree.

    python chime-x_b200/build.py            # incremental
    python chime-x_b200/build.py --clean    # rebuild everything

Every .cu file under csrc/ is compiled by nvcc for sm_100a only
(-gencode arch=compute_100a,code=sm_100a) and linked into
chime-x_b200/libchimex.so.  host/correlator_test.c is compiled by gcc against
that library into chime-x_b200/correlator_test.
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libchimex.so")
HOST_BIN = os.path.join(HERE, "correlator_test")
NVCC = os.environ.get("NVCC", "nvcc")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC,-O3,-Wall",
    "--expt-relaxed-constexpr",
    "-I", os.path.join(ROOT, "include"),
]


def _newer(src_list, dst):
    if not os.path.exists(dst):
        return True
    t = os.path.getmtime(dst)
    return any(os.path.getmtime(s) > t for s in src_list)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise SystemExit("build failed: %s" % os.path.basename(cmd[-1]))
    return r.stdout + r.stderr


def build(clean=False, verbose=False):
    if clean and os.path.isdir(OBJ):
        shutil.rmtree(OBJ)
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "chimex.h"))
    sources = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))
    jobs = []
    objs = []
    for s in sources:
        o = os.path.join(OBJ, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if _newer([s] + headers, o):
            jobs.append([NVCC] + NVCC_FLAGS + ["-c", "-o", o, s])
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for out in ex.map(_run, jobs):
            if verbose and out.strip():
                print(out)
    if _newer(objs, LIB):
        _run([NVCC, "-shared", "-o", LIB] + objs + ["-lcudart"])
    host_src = os.path.join(HERE, "host", "correlator_test.c")
    if os.path.exists(host_src) and _newer([host_src, LIB, os.path.join(ROOT, "include", "chimex.h")], HOST_BIN):
        cuda_home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
        _run(["gcc", "-O2", "-std=gnu99", "-Wall", "-fopenmp", "-I", os.path.join(ROOT, "include"),
              "-I", os.path.join(cuda_home, "include"), "-o", HOST_BIN, host_src,
              "-L", HERE, "-lchimex", "-L", os.path.join(cuda_home, "lib64"), "-lcudart",
              "-Wl,-rpath,$ORIGIN", "-lm"])
    return LIB


if __name__ == "__main__":
    build(clean="--clean" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
