"""Build the CUDA library ``ducc_b200/_lib/libducc_b200.so`` in-tree.

Every source under ``csrc/`` is compiled by nvcc for sm_100a
(``-gencode arch=compute_100a,code=sm_100a``) into an object file, in parallel,
and linked into one shared library exposing the C-ABI of
``include/ducc_b200.h``.  Objects are rebuilt only when a source or header is
newer than them.

Usage:  python -m ducc_b200.build [-j N] [--force]
"""
import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
OBJDIR = os.path.join(LIBDIR, "obj")
LIB = os.path.join(LIBDIR, "libducc_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "--expt-relaxed-constexpr", "-I" + CSRC, "-I" + os.path.join(HERE, "..", "include")]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def headers():
    return (glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
            + glob.glob(os.path.join(CSRC, "*.inc"))
            + glob.glob(os.path.join(HERE, "..", "include", "*.h")))


def _obj(src):
    return os.path.join(OBJDIR, os.path.basename(src) + ".o")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, extra):
    cmd = [NVCC] + ARCH + FLAGS + extra + ["-c", src, "-o", _obj(src)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd), r.stderr))
    return src, r.stderr


def build(jobs=None, force=False, verbose=False, extra=()):
    os.makedirs(OBJDIR, exist_ok=True)
    hdrs = headers()
    todo = [s for s in sources() if force or _stale(_obj(s), [s] + hdrs)]
    jobs = jobs or min(len(todo) or 1, os.cpu_count() or 4)
    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
            for src, err in ex.map(lambda s: _compile(s, list(extra)), todo):
                if verbose:
                    print("compiled", os.path.basename(src), file=sys.stderr)
                if verbose and err.strip():
                    print(err, file=sys.stderr)
    objs = [_obj(s) for s in sources()]
    if force or todo or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true", help="print register / smem usage")
    a = ap.parse_args()
    extra = ["-Xptxas", "-v"] if a.ptxas_v else []
    print(build(a.j, a.force, a.v or a.ptxas_v, extra))


if __name__ == "__main__":
    main()
