"""Builds the CUDA library gstar4d_b200/libgstar4d.so for sm_100a with nvcc,
and the native command line gstar4d_b200/gstar4d over its C ABI.

Both are built in-tree so that they travel with the repository to the GPU
host; nothing is installed into site-packages.
"""
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgstar4d.so")
EXE = os.path.join(HERE, "gstar4d")  # native command line
OBJ = os.path.join(HERE, "_build")

SOURCES = ["g4d_order.cu", "g4d_pba.cu", "g4d_star.cu", "g4d_api.cu", "g4d_noalloc.cu", "g4d_mlp.cu", "g4d_proposal.cu", "g4d_block.cu", "g4d_check.cu", "g4d_points.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "-I", os.path.join(REPO, "include"), "-I", CSRC, "--expt-relaxed-constexpr"]


def _cxx():
    for cand in (os.environ.get("CXX"), "/usr/bin/g++", shutil.which("g++")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("g++ not found")


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale():
    if not os.path.exists(LIB) or not os.path.exists(EXE):
        return True
    t = min(os.path.getmtime(LIB), os.path.getmtime(EXE))
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(REPO, "include", "gstar4d.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    if not force and not _stale():
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    nvcc = _nvcc()
    # the SoS table header is generated from its derivation script
    with open(os.path.join(CSRC, "sos_table.inc"), "w") as f:
        subprocess.check_call([sys.executable, os.path.join(CSRC, "gen_sos_table.py")], stdout=f)

    def compile_one(src):
        obj = os.path.join(OBJ, os.path.splitext(src)[0] + ".o")
        cmd = [nvcc] + ARCH + FLAGS + ["-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s" % (src, r.stderr))
        return obj, r.stderr

    with ThreadPoolExecutor(max_workers=4) as ex:
        results = list(ex.map(compile_one, SOURCES))
    if verbose:
        for _, err in results:
            sys.stderr.write(err)
    objs = [o for o, _ in results]
    tmp = LIB + ".tmp"
    subprocess.check_call([nvcc] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart"])
    os.replace(tmp, LIB)
    # the native command line over the C ABI, next to the library it loads
    tmp = EXE + ".tmp"
    subprocess.check_call([_cxx(), "-O2", "-std=c++17", "-I", os.path.join(REPO, "include"),
                           os.path.join(CSRC, "gstar4d_cli.cpp"), "-o", tmp, "-L", HERE, "-lgstar4d",
                           "-Wl,-rpath,$ORIGIN"])
    os.replace(tmp, EXE)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
