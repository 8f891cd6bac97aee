"""Build libcgb.so (sm_100a) in-tree: npb-gpu_b200/lib/libcgb.so.

    python npb-gpu_b200/build.py [--verbose] [--ptxas-info] [--checked]

nvcc cross-compiles for sm_100a without a GPU.  The host generator
(makea.cpp) is compiled by the host compiler with -ffp-contract=off so its
floating-point arithmetic rounds exactly like the reference's.
"""
import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
BUILD = os.path.join(HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["session.cu", "noalloc.cu", "gnn.cu", "batch.cu", "makea_gpu.cu", "part.cu", "mg.cu",
              "ep.cu", "is.cu", "ft.cu"]
# per-source flags: MG's operators and EP's deviates keep the reference's
# separate roundings
EXTRA_FLAGS = {"mg.cu": ["-fmad=false"], "ep.cu": ["-fmad=false"]}
CPP_SOURCES = ["makea.cpp"]
LIB = os.path.join(LIBDIR, "libcgb.so")
# the checked build: the single-system solver with every SpMV index tested
CHECKED_SOURCES = ["session.cu", "noalloc.cu"]
LIB_CHECKED = os.path.join(LIBDIR, "libcgb_checked.so")
BINDIR = os.path.join(HERE, "bin")
DRIVER = os.path.join(BINDIR, "cg")
MG_DRIVER = os.path.join(BINDIR, "mg")
EP_DRIVER = os.path.join(BINDIR, "ep")
IS_DRIVER = os.path.join(BINDIR, "is")
FT_DRIVER = os.path.join(BINDIR, "ft")


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found")
    return exe


def run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    if verbose and (res.stdout or res.stderr):
        sys.stdout.write(res.stdout + res.stderr)
    return res


def sources_newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, ptxas_info=False, force=False):
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(os.path.dirname(HERE), "include", "cgb.h"))
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or sources_newer(o, [s] + headers):
            cmd = [nvcc(), "-c", s, "-o", o, *ARCH, "-O3", "-lineinfo", "-std=c++17",
                   "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
                   "--expt-relaxed-constexpr", *EXTRA_FLAGS.get(src, [])]
            if ptxas_info:
                cmd += ["-Xptxas", "-v"]
            r = run(cmd, verbose)
            if ptxas_info:
                sys.stdout.write(r.stderr)
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or sources_newer(o, [s] + headers):
            run([nvcc(), "-c", s, "-o", o, "-O2", "-std=c++17", "-Xcompiler", "-fPIC",
                 "-Xcompiler", "-ffp-contract=off", "-Xcompiler", "-pthread"], verbose)
    if force or sources_newer(LIB, objs):
        run([nvcc(), "-shared", "-o", LIB, *objs, *ARCH, "-cudart", "static",
             "-Xcompiler", "-pthread", "-lpthread"], verbose)
    # the NPB-style command-line drivers, linked against libcgb.so
    os.makedirs(BINDIR, exist_ok=True)
    main_src = os.path.join(CSRC, "cg_main.cpp")
    if force or sources_newer(DRIVER, [main_src, LIB] + headers):
        run([nvcc(), "-O2", "-std=c++17", "-o", DRIVER, main_src, "-L" + LIBDIR, "-lcgb",
             "-Xlinker", "-rpath=$ORIGIN/../lib"], verbose)
    for name, target in (("mg_main.cpp", MG_DRIVER), ("ep_main.cpp", EP_DRIVER), ("is_main.cpp", IS_DRIVER),
                         ("ft_main.cpp", FT_DRIVER)):
        src = os.path.join(CSRC, name)
        if force or sources_newer(target, [src, LIB] + headers):
            run([nvcc(), "-O2", "-std=c++17", "-o", target, src, "-L" + LIBDIR, "-lcgb",
                 "-Xlinker", "-rpath=$ORIGIN/../lib"], verbose)
    return LIB


def build_checked(verbose=False, force=False):
    """lib/libcgb_checked.so: the library with the solver's translation units
    compiled with -DCGB_CHECKED (bounds-tested SpMV indices, cgb_check_status);
    the other objects are the normal build's."""
    build(verbose, False, force)
    cdir = os.path.join(BUILD, "checked")
    os.makedirs(cdir, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(os.path.dirname(HERE), "include", "cgb.h"))
    objs = []
    for src in CU_SOURCES + CPP_SOURCES:
        if src in CHECKED_SOURCES:
            s = os.path.join(CSRC, src)
            o = os.path.join(cdir, src + ".o")
            if force or sources_newer(o, [s] + headers):
                run([nvcc(), "-c", s, "-o", o, *ARCH, "-O3", "-lineinfo", "-std=c++17",
                     "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
                     "--expt-relaxed-constexpr", "-DCGB_CHECKED"], verbose)
        else:
            o = os.path.join(BUILD, src + ".o")
        objs.append(o)
    if force or sources_newer(LIB_CHECKED, objs):
        run([nvcc(), "-shared", "-o", LIB_CHECKED, *objs, *ARCH, "-cudart", "static",
             "-Xcompiler", "-pthread", "-lpthread"], verbose)
    return LIB_CHECKED


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--checked", action="store_true", help="also build lib/libcgb_checked.so")
    a = ap.parse_args()
    print(build(a.verbose, a.ptxas_info, a.force))
    if a.checked:
        print(build_checked(a.verbose, a.force))
