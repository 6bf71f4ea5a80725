#!/usr/bin/env python3
"""Build recipe for the compiled reference (test infrastructure only).

This script compiles ParMooN's own C++ sources, where they lie in the read-only
reference tree, into static archives under ``oracle/_ref/`` and links the
project-written dump drivers in ``oracle/ref_driver/`` against them.  Nothing
from the reference tree is copied into this repository; the outputs under
``oracle/_ref/`` are git-ignored build products.

The source lists follow the reference's own CMake files
(``src/*/CMakeLists.txt``): ``list(APPEND ..._SOURCES ...)`` entries inside the
``AParMooN_GEO`` branches, plus the ``GLOB_RECURSE`` directories (General,
QuadFormulas, Refinement, AMG).  Flags follow ``UserConfig.cmake:126-171`` for
``AParMooN_PARALLEL_TYPE=SEQUENTIAL`` (``-D_SEQ -D__PRIVATE__ -DTRILIBRARY
-DTETLIBRARY``), with ``-O3`` instead of the reference's unoptimised RELEASE
flags so the CPU baseline is not handicapped.  Sources that do not compile with
g++ 13 (off the convection-diffusion path: direct solvers that need PARDISO /
cblas headers, ALE, TNSE) are skipped and listed in ``oracle/_ref/<geo>/skipped.txt``;
the few external symbols they would have provided are abort-stubs in
``oracle/ref_driver/stubs.C``.

Usage:  python oracle/build_ref.py [--ref <reference tree>] [--jobs 8] [--geo 2D 3D]
        (default tree: $CDGPU_REFERENCE, else /root/reference)
"""
import argparse
import os
import re
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")

INCLUDE_DIRS = ["General", "FE", "Geometry", "QuadFormulas", "FE1D", "FE2D", "FE3D",
                "AMG", "PBE", "Refinement", "System", "Parallel", "Solvers"]


def cmake_sources(path, geo):
    """Return the list(APPEND X_SOURCES ...) files active for AParMooN_GEO == geo
    and PARALLEL_TYPE == SEQUENTIAL in one reference CMakeLists.txt."""
    active = [True]
    out = []
    with open(path) as f:
        for raw in f:
            line = raw.strip()
            if line.startswith("#"):
                continue
            m = re.match(r'(if|elseif)\("\$\{AParMooN_(\w+)\}"\s+STREQUAL\s+"(\w+)"', line)
            if m:
                kind, var, val = m.groups()
                cond = (val == geo) if var == "GEO" else (val == "SEQUENTIAL")
                if kind == "if":
                    active.append(cond)
                else:
                    active[-1] = cond
                continue
            if line.startswith("else("):
                active[-1] = not active[-1]
                continue
            if line.startswith("endif"):
                active.pop()
                continue
            m = re.match(r'list\(APPEND\s+\w+\s+"\$\{PROJECT_SOURCE_DIR\}/([^"]+)"\s*\)', line)
            if m and all(active):
                out.append(m.group(1))
    return out


def source_list(ref, geo):
    srcs = []
    for d in ["General", "QuadFormulas", "Refinement"]:
        for fn in sorted(os.listdir(os.path.join(ref, "src", d))):
            if fn.endswith(".C"):
                srcs.append(f"src/{d}/{fn}")
    for d in ["Geometry", "FE", "System", "Solvers"]:
        srcs += cmake_sources(os.path.join(ref, "src", d, "CMakeLists.txt"), geo)
    for fn in sorted(os.listdir(os.path.join(ref, "src", "AMG"))):
        if fn.endswith(".c"):
            srcs.append(f"src/AMG/{fn}")
    return [s for s in srcs if s.endswith((".C", ".c"))]


def defines(geo):
    return [f"-D__{geo}__", "-D__LINUX64__", "-DTRILIBRARY", "-DTETLIBRARY",
            "-D_SEQ", "-D__PRIVATE__", "-DREDUCED", "-DNO_TIMER"]


def includes(ref):
    # EXT_LIB/tetgen holds only the tetgen *header* that include/Geometry/TetGenMeshLoader.h
    # pulls into Domain.C; no EXT_LIB binary is linked (tetgen calls resolve to abort-stubs).
    # EXT_LIB/tecplot/include likewise only provides TECIO.h to Output2D.C / Output3D.C; the
    # tecplot writer functions resolve to abort-stubs too
    return [f"-I{ref}/include/{d}" for d in INCLUDE_DIRS] + [f"-I{ref}/Examples",
                                                            f"-I{ref}/EXT_LIB/tetgen",
                                                            f"-I{ref}/EXT_LIB/tecplot/include"]


def compile_one(ref, geo, src, objdir):
    obj = os.path.join(objdir, src.replace("/", "__") + ".o")
    full = os.path.join(ref, src)
    if os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(full):
        return src, True, ""
    if src.endswith(".c"):
        cmd = ["gcc", "-O3", "-w", "-fPIC"] + defines(geo) + includes(ref) + ["-c", full, "-o", obj]
    else:
        cmd = ["g++", "-O3", "-std=c++11", "-fpermissive", "-w", "-fPIC"] + defines(geo) + \
              includes(ref) + ["-c", full, "-o", obj]
    p = subprocess.run(cmd, capture_output=True, text=True)
    return src, p.returncode == 0, p.stderr[-2000:]


def build_geo(ref, geo, jobs):
    objdir = os.path.join(OUT, geo.lower(), "obj")
    os.makedirs(objdir, exist_ok=True)
    srcs = source_list(ref, geo)
    ok, bad = [], []
    with ThreadPoolExecutor(jobs) as ex:
        for src, good, err in ex.map(lambda s: compile_one(ref, geo, s, objdir), srcs):
            (ok if good else bad).append((src, err))
    with open(os.path.join(OUT, geo.lower(), "skipped.txt"), "w") as f:
        for src, err in bad:
            f.write(f"{src}\n")
    lib = os.path.join(OUT, geo.lower(), f"libparmoon{geo.lower()}.a")
    if os.path.exists(lib):
        os.remove(lib)
    objs = [os.path.join(objdir, s.replace("/", "__") + ".o") for s, _ in ok]
    subprocess.run(["ar", "rcs", lib] + objs, check=True)
    print(f"[{geo}] compiled {len(ok)} / {len(srcs)} sources; skipped: {[s for s, _ in bad]}")
    return lib


def link_driver(ref, geo, lib, name, main_src):
    drv = os.path.join(HERE, "ref_driver")
    exe = os.path.join(OUT, name)
    cmd = ["g++", "-O3", "-std=c++11", "-fpermissive", "-w"] + defines(geo) + includes(ref) + \
          [f"-I{drv}", os.path.join(drv, main_src), os.path.join(drv, "stubs.C"),
           "-Wl,--start-group", lib, "-Wl,--end-group", "-lm", "-o", exe]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        sys.stderr.write(p.stderr[-6000:])
        raise SystemExit(f"link of {name} failed")
    print(f"linked {exe}")


def link_main(ref, geo, lib, name, main_src, gpu, shim="SystemCD3D_cdgpu.C", extra=()):
    """Link the reference's own, unchanged main program (e.g. 3DPrograms/CD3D_ParMooN.C) against
    the compiled reference; with gpu, the TSystemCD3D of parmoon_cmg_b200/shim (the
    reference-side binding of libcdgpu) comes first on the link line, so the archive's
    SystemCD3D object is not used and the program runs its assembly and solve on the GPU."""
    drv = os.path.join(HERE, "ref_driver")
    root = os.path.dirname(HERE)
    exe = os.path.join(OUT, name)
    srcs = [os.path.join(ref, main_src)]
    libs = []
    if gpu:
        srcs.append(os.path.join(root, "parmoon_cmg_b200", "shim", shim))
        libs = [f"-L{os.path.join(root, 'parmoon_cmg_b200')}", "-lcdgpu",
                "-Wl,-rpath,$ORIGIN/../../parmoon_cmg_b200"]
    cmd = ["g++", "-O2", "-std=c++11", "-fpermissive", "-w"] + defines(geo) + list(extra) + includes(ref) + \
          [f"-I{os.path.join(root, 'include')}"] + srcs + [os.path.join(drv, "stubs.C"),
                                                        "-Wl,--start-group", lib, "-Wl,--end-group"] + \
          libs + ["-lm", "-o", exe]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        sys.stderr.write(p.stderr[-6000:])
        raise SystemExit(f"link of {name} failed")
    print(f"linked {exe}")


def default_tree():
    """The reference tree this recipe compiles: $CDGPU_REFERENCE, else the container's copy."""
    return os.environ.get("CDGPU_REFERENCE", "/root/reference")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=default_tree())
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 4)
    ap.add_argument("--geo", nargs="*", default=["2D", "3D"])
    ap.add_argument("--link-only", action="store_true")
    a = ap.parse_args()
    if not os.path.isdir(a.ref):
        raise SystemExit(f"reference tree {a.ref} not present; oracle/_ref cannot be built here")
    os.makedirs(OUT, exist_ok=True)
    for geo in a.geo:
        lib = os.path.join(OUT, geo.lower(), f"libparmoon{geo.lower()}.a")
        if not a.link_only or not os.path.exists(lib):
            lib = build_geo(a.ref, geo, a.jobs)
        link_driver(a.ref, geo, lib, f"cd{geo.lower()}_dump", f"cd{geo.lower()}_dump.C")
        have_gpu_lib = os.path.exists(os.path.join(os.path.dirname(HERE), "parmoon_cmg_b200", "libcdgpu.so"))
        if geo == "3D":
            # the reference's CD3D main unchanged: on its own TSystemCD3D (CPU) and on libcdgpu
            link_main(a.ref, geo, lib, "cd3d_main", "3DPrograms/CD3D_ParMooN.C", gpu=False)
            # the reference's TCD3D main unchanged (its example amc.h), for the time-dependent
            # known answer (tests/golden/make_golden.py)
            link_main(a.ref, geo, lib, "tcd3d_main", "3DPrograms/TCD3D_ParMooN.C", gpu=False)
            if have_gpu_lib:
                link_main(a.ref, geo, lib, "cd3d_main_gpu", "3DPrograms/CD3D_ParMooN.C", gpu=True)
        elif have_gpu_lib:
            # the reference's CD2D main unchanged, built with its own test switch (_TEST: the
            # SineLaplace example, CD2D_ParMooN.C:21-26), on the TSystemCD2D of libcdgpu (the
            # reference's own TSystemCD2D solves with UMFPACK, which is not available here)
            link_main(a.ref, geo, lib, "cd2d_main_gpu", "2DPrograms/CD2D_ParMooN.C", gpu=True,
                      shim="SystemCD2D_cdgpu.C", extra=["-D_TEST"])


if __name__ == "__main__":
    main()
