"""In-tree build of libxkb200.so (sm_100a) with nvcc.

Every .cu/.cc under xkaapi_b200/csrc is compiled to an object in xkaapi_b200/_build and
linked into xkaapi_b200/libxkb200.so. Objects are rebuilt when their source, any header of
csrc/ or include/, or the flags change. nvcc cross-compiles: no GPU is needed to build.
"""
import concurrent.futures as cf
import hashlib
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libxkb200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "-Xptxas", "-warn-spills", "--expt-relaxed-constexpr", "-I" + os.path.join(REPO, "include")]
# XKB_NVCC_DEFINES: extra compile-time settings for tuning sweeps, e.g. "-DXKB_TILE_PF=3"
NVCC_FLAGS += os.environ.get("XKB_NVCC_DEFINES", "").split()
LINK_FLAGS = ["-shared", "-lcudart", "-lpthread"]


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers_digest():
    h = hashlib.sha256()
    for d in (CSRC, os.path.join(REPO, "include")):
        for root, _, files in os.walk(d):
            for f in sorted(files):
                if f.endswith((".h", ".cuh", ".hpp")):
                    with open(os.path.join(root, f), "rb") as fh:
                        h.update(f.encode()); h.update(fh.read())
    return h.hexdigest()


def _compile(src, extra, verbose):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    stamp = obj + ".stamp"
    with open(src, "rb") as fh:
        key = hashlib.sha256(fh.read() + extra.encode()).hexdigest()
    if os.path.exists(obj) and os.path.exists(stamp) and open(stamp).read() == key:
        return obj
    cmd = [nvcc()] + ARCH + NVCC_FLAGS + ["-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr.strip():
        print(r.stderr, file=sys.stderr)
    with open(stamp, "w") as fh:
        fh.write(key)
    return obj


def build(verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cc")))
    extra = _headers_digest() + " ".join(ARCH + NVCC_FLAGS)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra, verbose), srcs))
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [nvcc()] + ARCH + ["-o", LIB] + objs + LINK_FLAGS
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    build_examples(verbose)
    return LIB


EXAMPLES = os.path.join(PKG, "examples")


def build_examples(verbose=False):
    """C programs under examples/ (the reference's examples written against include/xkrt_capi.h),
    linked to libxkb200.so with an $ORIGIN-relative rpath so the tree can move."""
    out = []
    for f in sorted(os.listdir(EXAMPLES)):
        if not f.endswith(".c"):
            continue
        src, exe = os.path.join(EXAMPLES, f), os.path.join(EXAMPLES, f[:-2])
        if os.path.exists(exe) and os.path.getmtime(exe) >= max(os.path.getmtime(src), os.path.getmtime(LIB)):
            out.append(exe)
            continue
        cmd = ["gcc", "-std=c11", "-O2", "-Wall", "-Werror", "-D_POSIX_C_SOURCE=200809L", "-I" + os.path.join(REPO, "include"),
               src, "-o", exe, "-L" + PKG, "-lxkb200", "-lm", "-Wl,-rpath,$ORIGIN/.."]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"gcc failed on {src}:\n{r.stdout}\n{r.stderr}")
        out.append(exe)
    # C++ programs (the reference's C++ source API, include/xkrt/) with their own CUDA kernels in
    # <name>_kernel.cu
    for f in sorted(os.listdir(EXAMPLES)):
        if not f.endswith(".cc"):
            continue
        src, exe = os.path.join(EXAMPLES, f), os.path.join(EXAMPLES, f[:-3])
        kern = os.path.join(EXAMPLES, f[:-3] + "_kernel.cu")
        deps = [src, LIB] + ([kern] if os.path.exists(kern) else []) + \
            [os.path.join(r, h) for r, _, hs in os.walk(os.path.join(REPO, "include", "xkrt")) for h in hs]
        if os.path.exists(exe) and os.path.getmtime(exe) >= max(os.path.getmtime(d) for d in deps):
            out.append(exe)
            continue
        objs = []
        if os.path.exists(kern):
            kobj = os.path.join(BUILD, f[:-3] + "_kernel.o")
            cmd = [nvcc()] + ARCH + ["-O3", "-Xcompiler", "-fPIC", "-c", kern, "-o", kobj]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed on {kern}:\n{r.stdout}\n{r.stderr}")
            objs.append(kobj)
        cuda = os.path.dirname(os.path.dirname(nvcc()))
        cmd = ["g++", "-std=c++20", "-O2", "-Wall", "-Werror", "-I" + os.path.join(REPO, "include"), "-I" + os.path.join(cuda, "include"),
               src] + objs + ["-o", exe, "-L" + PKG, "-lxkb200", "-L" + os.path.join(cuda, "lib64"), "-lcudart", "-lpthread",
                              "-Wl,-rpath,$ORIGIN/.."]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"g++ failed on {src}:\n{r.stdout}\n{r.stderr}")
        out.append(exe)
    return out


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
