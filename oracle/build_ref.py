"""Builds oracle/_ref/libref_bssn_gpu.so from the reference's own sources.

TEST INFRASTRUCTURE ONLY.  The reference's Fortran cannot be compiled in this
image (no Fortran compiler), but its 2015 CUDA port of compute_rhs_bssn
(AMSS_NCKU_source/bssn_gpu.cu, gpu_rhs at :1985) can, once its build-time
header macrodef.fh exists.  This recipe:

1. writes macrodef.fh into oracle/_ref/src with the reference's own generator
   (amss-ncku-python/generate_macrodef.py, generate_macrodef_fh) fed the
   reference's shipped AMSS_NCKU_Input.py settings -- Patch grid (no
   WithShell, no CPBC), Cell centring, 4th order (ghost_width 3), GAUGE 0,
   ABV 0 -- with only the output directory redirected;
2. links the sources bssn_gpu.cu, bssn_gpu.h, gpu_mem.h and bssn_macro.h into
   oracle/_ref/src where they lie (symbolic links, so that their
   #include "macrodef.fh" finds the generated header rather than the shipped
   one, which is configured for GAUGE 2 with shells);
3. compiles them with oracle/ref_gpu_shim.cu for sm_100a into
   oracle/_ref/libref_bssn_gpu.so.

Outputs go to oracle/_ref only (git-ignored); the .so travels with the tree to
a GPU host, where tests/test_gpu_reference_port.py compares the oracle with it.
Run: python oracle/build_ref.py   (a no-op when the reference is not mounted).
"""
import importlib.util
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF = "/root/reference/amss-ncku-python"
SRC = os.path.join(REF, "AMSS_NCKU_source")
OUT = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT, "libref_bssn_gpu.so")
FILES = ("bssn_gpu.cu", "bssn_gpu.h", "gpu_mem.h", "bssn_macro.h")


def _load(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def generate_macrodef(dst):
    """macrodef.fh for the evolution path, by the reference's generator."""
    inp = _load("AMSS_NCKU_Input", os.path.join(REF, "AMSS_NCKU_Input.py"))
    assert (inp.basic_grid_set, inp.grid_center_set, inp.Finite_Diffenence_Method, inp.gauge_choice) == \
        ("Patch", "Cell", "4th-order", 0), "the reference's shipped inputs changed"
    inp.File_directory = dst
    gen = _load("generate_macrodef", os.path.join(REF, "generate_macrodef.py"))
    gen.generate_macrodef_fh()
    text = open(os.path.join(dst, "macrodef.fh")).read()
    for want in ("#define GAUGE 0", "#define Cell", "#define ghost_width 3", "#define ABV 0"):
        assert want in text, want
    assert "#define WithShell" not in text and "#define CPBC\n" not in text


def build(force=False):
    if not os.path.isdir(SRC):
        return None
    src = os.path.join(OUT, "src")
    os.makedirs(src, exist_ok=True)
    shim = os.path.join(HERE, "ref_gpu_shim.cu")
    deps = [os.path.join(SRC, f) for f in FILES] + [shim, os.path.abspath(__file__)]
    if not force and os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(d) for d in deps):
        return LIB
    generate_macrodef(src)
    for f in FILES:
        link = os.path.join(src, f)
        if os.path.lexists(link):
            os.remove(link)
        os.symlink(os.path.join(SRC, f), link)
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17", "-shared",
           "-Xcompiler", "-fPIC", "-w", "-Dfortran3", "-I", src, "-o", LIB,
           os.path.join(src, "bssn_gpu.cu"), shim]
    subprocess.run(cmd, check=True)
    for f in FILES:   # the links point into the reference tree, which other hosts do not have
        os.remove(os.path.join(src, f))
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv) or "reference not mounted: nothing built")
