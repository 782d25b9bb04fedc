"""Build libyeti_b200.so in-tree with nvcc for sm_100a.

    python -m yeti_b200.build          # or yeti_b200.build.build()

The library is a plain C-ABI shared object (include/yeti_b200.h); the Python
package loads it with ctypes.  Object files go to yeti_b200/_build/.
"""
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libyeti_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
              "-Xcompiler", "-fPIC,-fvisibility=hidden,-O3",
              "-Xptxas", "-O3", "-DNDEBUG"]


# Per-file extra flags.  The Gauss-quadrature assembly and shape gradient
# mirror the reference's operation order exactly, which requires no FMA
# contraction.
EXTRA_FLAGS = {"assemble_u1.cu": ["-fmad=false"], "grad_u1.cu": ["-fmad=false"],
               "volume_u1.cu": ["-fmad=false"]}


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc",
                 shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _host_compiler():
    # the system g++ (an inherited $CXX may point at a toolchain nvcc does
    # not support)
    for cand in ("/usr/bin/g++", shutil.which("g++")):
        if cand and os.path.exists(cand):
            return cand
    return None


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) +
                  glob.glob(os.path.join(CSRC, "*.cpp")))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, jobs=None):
    os.makedirs(BUILD, exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(
        os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(ROOT, "include", "*.h"))
    cc = nvcc()
    hc = _host_compiler()
    base = [cc] + ARCH + NVCC_FLAGS + ["-I", os.path.join(ROOT, "include")]
    if hc:
        base += ["-ccbin", hc]
    objs, procs = [], []
    for src in sources():
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if _stale(obj, [src] + headers):
            cmd = base + EXTRA_FLAGS.get(os.path.basename(src), []) + [
                "-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                                stderr=subprocess.STDOUT)))
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append((src, out.decode(errors="replace")))
        elif verbose and out:
            print(out.decode(errors="replace"))
    if failed:
        msg = "\n".join(f"--- {s}\n{o}" for s, o in failed)
        raise RuntimeError(f"nvcc failed:\n{msg}")
    if _stale(LIB, objs):
        cmd = [cc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static"]
        if hc:
            cmd += ["-ccbin", hc]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)
