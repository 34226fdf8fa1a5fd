"""Builds libdiagham_b200.so in place with nvcc for sm_100a.

The library is the whole product: CUDA kernels, host set-up code and the C ABI declared in
include/diagham_b200.h.  It is built into the package directory so it travels with the source
tree; nothing is installed into site-packages.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libdiagham_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources():
    out = []
    for name in sorted(os.listdir(CSRC)):
        if name.endswith((".cu", ".cc")):
            out.append(os.path.join(CSRC, name))
    return out


def _deps():
    deps = sources() + [os.path.join(CSRC, n) for n in os.listdir(CSRC) if n.endswith(".h")]
    deps.append(os.path.join(ROOT, "include", "diagham_b200.h"))
    return deps


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in _deps())


def build(force=False, verbose=False):
    """Compile every source into objects under _build/ (parallel), then link the shared library."""
    if not force and up_to_date():
        return LIB
    objdir = os.path.join(ROOT, "_build", "diagham_b200")
    os.makedirs(objdir, exist_ok=True)
    common = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "-I", os.path.join(ROOT, "include"),
                     "-I", CSRC]
    if verbose:
        common += ["-Xptxas", "-v"]
    procs = []
    objs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        objs.append(obj)
        cmd = [NVCC] + common + ["-x", "cu" if src.endswith(".cu") else "c++", "-c", src, "-o", obj]
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = []
    for src, p in procs:
        out = p.communicate()[0].decode(errors="replace")
        if p.returncode != 0 or (verbose and out.strip()):
            sys.stderr.write(out)
        if p.returncode != 0:
            failed.append(src)
    if failed:
        raise RuntimeError("nvcc failed on: " + ", ".join(os.path.basename(f) for f in failed))
    tmp = LIB + ".tmp"
    link = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", tmp] + objs
    subprocess.run(link, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
