"""Build of libct_gravity.so (the C ABI of include/ct_gravity.h) for sm_100a.

nvcc compiles each translation unit for -gencode arch=compute_100a,code=sm_100a and links a
shared library in-tree (cosmictiger_b200/libct_gravity.so).  The tree build is compiled with
-fmad=false: its float/double geometry must not be contracted into FMAs so that node
centres, radii and boxes come out bit-identical to the reference's C++ arithmetic.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libct_gravity.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "-I" + CSRC, "-I" + os.path.join(ROOT, "include")]
UNITS = {
    "ct_tree.cu": ["-fmad=false"],
    "ct_kick.cu": ["-fmad=false"],
    "ct_api.cu": [],
    "ct_noalloc.cu": [],
    "ct_driver.cu": [],
    "ct_lightcone.cu": [],
    "ct_fourier.cu": [],
}


def _deps():
    out = []
    for f in os.listdir(CSRC):
        if f.endswith((".cu", ".cuh", ".h")):
            out.append(os.path.join(CSRC, f))
    out.append(os.path.join(ROOT, "include", "ct_gravity.h"))
    return out


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def generate():
    subprocess.check_call([sys.executable, os.path.join(CSRC, "gen_fmm.py"), "7", "5"])


def build(verbose=False, force=False, jobs=None):
    gen = os.path.join(CSRC, "gen_fmm.py")
    if force or any(_stale(os.path.join(CSRC, "fmm_p%d.h" % p), [gen]) for p in (7, 5)):
        generate()
    os.makedirs(BUILD, exist_ok=True)
    deps = _deps()
    objs = []
    procs = []
    for unit, extra in UNITS.items():
        obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, deps):
            cmd = [NVCC] + ARCH + COMMON + extra + ["-c", os.path.join(CSRC, unit), "-o", obj]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
                print(" ".join(cmd), flush=True)
            procs.append((unit, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = []
    for unit, p in procs:
        out, _ = p.communicate()
        if verbose or p.returncode:
            sys.stdout.write(out.decode(errors="replace"))
        if p.returncode:
            failed.append(unit)
    if failed:
        raise RuntimeError("nvcc failed for " + ", ".join(failed))
    if force or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-lcufft"]
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
