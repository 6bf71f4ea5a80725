"""Build of libcdgpu.so (in-tree, sm_100a).

Compiles ``parmoon_cmg_b200/csrc/*.cu`` and ``*.cpp`` with nvcc for
``-gencode arch=compute_100a,code=sm_100a`` and links them into
``parmoon_cmg_b200/libcdgpu.so`` next to this file.  Objects go to
``parmoon_cmg_b200/_build/`` (git-ignored).  Rebuilds only what changed.
"""
import os
import subprocess
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcdgpu.so")
ROOT = os.path.dirname(HERE)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "--expt-relaxed-constexpr", f"-I{os.path.join(ROOT, 'include')}"]


def _nvcc():
    for c in ("/usr/local/cuda/bin/nvcc", "nvcc"):
        if os.path.sep not in c or os.path.exists(c):
            return c
    return "nvcc"


def _sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _headers_mtime():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(ROOT, "include", "cdgpu.h"))
    return max(os.path.getmtime(h) for h in hs if os.path.exists(h))


def _compile(src, force, extra):
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    newest = max(os.path.getmtime(src), _headers_mtime())
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= newest:
        return obj, None
    cmd = [_nvcc()] + ARCH + FLAGS + extra + ["-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [_nvcc(), "-x", "c++"] + FLAGS + extra + ["-c", src, "-o", obj]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        return obj, p.stderr
    return obj, None


def build(force=False, verbose=False, extra=()):
    """Compile and link libcdgpu.so; returns its path."""
    os.makedirs(OBJ, exist_ok=True)
    srcs = _sources()
    with ThreadPoolExecutor(min(8, len(srcs))) as ex:
        res = list(ex.map(lambda s: _compile(s, force, list(extra)), srcs))
    errs = [e for _, e in res if e]
    if errs:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errs))
    objs = [o for o, _ in res]
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [_nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError("link failed:\n" + p.stderr)
    if verbose:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    build(verbose=True)
