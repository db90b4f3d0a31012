"""Recipe: compile the HARM-COOL reference's own C sources into CPU checker
libraries under oracle/_ref/<config>/ (TEST INFRASTRUCTURE ONLY).

The reference fixes its grid size and physics switches at compile time in
decs.h (decs.h:59-61, 110, 114, 117) and its torus parameters as literals in
init.c (init.c:104-110).  For each configuration this recipe writes patched
copies of those two files into oracle/_ref/<config>/gen/ and compiles every
other source file where it lies in the reference tree.  The `-I-` option
makes `#include "decs.h"` resolve to the patched copy instead of the file
next to the including source.

Switches: COOL_EOS 0 except in the COOL_EOS configurations, which compile the
reference's run-time EOS (cooleos.c, cache4d.c, akima.c) with oracle/eos_standin.c
in place of the Fortran table generator (gfortran is absent here), the table fill
in this process and the cache files turned off; TRACERSDUMP 0 except in the
tracer configurations; HDFDUMP 0 (no HDF5).  MPI_USED is on and the
single-rank stand-in in oracle/fakempi provides MPI: with one rank the phi
periodicity and opposite-phi polar ghosts are MPI self-exchanges
(step_ch.c:189-198, bounds.c:161-275).  Floating point: SSE2, -O2 (the
reference Makefile's level, Makefile:19), -ffp-contract=off; the Makefile's
-mfpmath=387 (x87, Makefile:29) is dropped so results are reproducible.

The patch also sizes the four opposite-phi slice tables N3+2 instead of N3:
the reference indexes them with h in [1, N3] (mpi.c:337-422, bounds.c:194-230),
one past their end, which overwrites neighbouring globals.

Outputs per config: libharmref.so (reference objects + oracle/refdrv.cpp)
and refbench (CPU timing binary).  Nothing is written outside oracle/_ref/.
"""
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
# the reference tree's src/ directory; HARM_REFERENCE_SRC names another copy
REF_SRC = os.environ.get("HARM_REFERENCE_SRC", "/root/reference/src")
OUT = os.path.join(HERE, "_ref")

# name -> (N1, N2, N3, spin a, torus rin, torus rmax, beta)
CONFIGS = {
    # config 1 of the benchmark: 2D 128x128 Fishbone-Moncrief torus
    "c1": (128, 128, 1, 0.9375, 6.0, 12.0, 100.0),
    # small grids for fixtures and fast checks
    "t2d": (32, 32, 1, 0.9375, 6.0, 12.0, 100.0),
    "t3d": (16, 16, 4, 0.9375, 6.0, 12.0, 100.0),
    "m3d": (32, 32, 8, 0.9375, 6.0, 12.0, 100.0),
    # bounded CPU sample of the 288x256x256 workload: same r-theta grid, 4 phi planes
    "c2s": (288, 256, 4, 0.9375, 6.0, 12.0, 100.0),
    # with the reference's tracer particles (TRACERSDUMP on, tracers.c)
    "r2d": (32, 32, 1, 0.9375, 6.0, 12.0, 100.0),
    "r3d": (16, 16, 4, 0.9375, 6.0, 12.0, 100.0),
}
TRACER_CONFIGS = ("r2d", "r3d")
# COOL_EOS on (the reference's own torus literals, whose spin matches cooleos.c's
# bhs = 0.6, cooleos.c:103), with oracle/eos_standin.c in place of the Fortran
# table generator
CONFIGS["ce2d"] = (32, 32, 1, 0.6, 4.0, 11.8, 50.0)
CONFIGS["ce3d"] = (16, 16, 4, 0.6, 4.0, 11.8, 50.0)
# the 256x256 COOL_EOS torus, for the CPU timing beside the device step
CONFIGS["ce256"] = (256, 256, 1, 0.6, 4.0, 11.8, 50.0)
COOL_CONFIGS = ("ce2d", "ce3d", "ce256")
# the drop-in: the reference's host code with harm_cool_b200/shim/harm_gpu.cpp in
# place of step_ch.c, bounds.c, fixup.c and utoprim_2d.c, linked to libharm_b200
CONFIGS["g2d"] = CONFIGS["t2d"]
CONFIGS["g3d"] = CONFIGS["t3d"]
SHIM_CONFIGS = ("g2d", "g3d")
SHIM_REPLACES = ("step_ch", "bounds", "fixup", "utoprim_2d")

SOURCES = ["bounds", "coord", "diag", "dump", "fixup", "image", "interp", "main",
           "metric", "lu", "phys", "ranc", "restart", "step_ch", "u2p_util",
           "utoprim_1dfix1", "utoprim_1dvsq2fix1", "utoprim_2d", "random",
           "utoprim_5d", "mpi"]


def _sub1(pattern, repl, text, what):
    new, n = re.subn(pattern, repl, text, count=1, flags=re.M)
    if n != 1:
        raise RuntimeError("patch failed: " + what)
    return new


def patch_decs(text, n1, n2, n3, tracers=False, cool=False):
    text = _sub1(r"^#define N1\s+\(\d+\)", "#define N1       (%d)" % n1, text, "N1")
    text = _sub1(r"^#define N2\s+\(\d+\)", "#define N2       (%d)" % n2, text, "N2")
    text = _sub1(r"^#define N3\s+\(\d+\)", "#define N3       (%d)" % n3, text, "N3")
    if not cool:
        text = _sub1(r"^#define COOL_EOS\s+\(1\)", "#define COOL_EOS  (0)", text, "COOL_EOS")
    if not tracers:
        text = _sub1(r"^#define TRACERSDUMP \(1\)", "#define TRACERSDUMP (0)", text, "TRACERSDUMP")
    text = _sub1(r"^#define HDFDUMP \(1\)", "#define HDFDUMP (0)", text, "HDFDUMP")
    # the opposite-phi slice tables are indexed by h in [1, N3] (mpi.c:337-422)
    # but declared with N3 entries: size them N3+2 so no neighbour is clobbered
    text, n = re.subn(r"(slice_hopNPR2_m2|slice_hopNPR2_n1|slice_h_rankop|slice_h_hop)\[N3\]",
                      r"\g<1>[N3+2]", text)
    if n != 4:
        raise RuntimeError("patch failed: slice tables")
    return text


def patch_defs(text):
    text, n = re.subn(r"(slice_hopNPR2_m2|slice_hopNPR2_n1|slice_h_rankop|slice_h_hop)\[N3\]",
                      r"\g<1>[N3+2]", text)
    if n != 4:
        raise RuntimeError("patch failed: defs.h slice tables")
    return text


def patch_init(text, a, rin, rmax, beta):
    text = _sub1(r"^(\s*)a = 0\.6;", r"\g<1>a = %r;" % a, text, "a")
    text = _sub1(r"^(\s*)rin = 4\.0;", r"\g<1>rin = %r;" % rin, text, "rin")
    text = _sub1(r"^(\s*)rmax = 11\.8;", r"\g<1>rmax = %r;" % rmax, text, "rmax")
    text = _sub1(r"^(\s*)beta = 50\.0 ;", r"\g<1>beta = %r ;" % beta, text, "beta")
    return text


def run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("compile failed")


def build_config(name, force=False):
    n1, n2, n3, a, rin, rmax, beta = CONFIGS[name]
    cdir = os.path.join(OUT, name)
    gen = os.path.join(cdir, "gen")
    obj = os.path.join(cdir, "obj")
    lib = os.path.join(cdir, "libharmref.so")
    exe = os.path.join(cdir, "refbench")
    if not force and os.path.exists(lib) and os.path.exists(exe) and not (name in SHIM_CONFIGS and shim_stale(name)):
        return lib
    os.makedirs(gen, exist_ok=True)
    os.makedirs(obj, exist_ok=True)
    tracers = name in TRACER_CONFIGS
    cool = name in COOL_CONFIGS
    with open(os.path.join(REF_SRC, "decs.h")) as f:
        decs = patch_decs(f.read(), n1, n2, n3, tracers, cool)
    with open(os.path.join(gen, "decs.h"), "w") as f:
        f.write(decs)
    with open(os.path.join(REF_SRC, "defs.h")) as f:
        defs = patch_defs(f.read())
    with open(os.path.join(gen, "defs.h"), "w") as f:
        f.write(defs)
    if cool:
        init = open(os.path.join(REF_SRC, "init.c")).read()   # its own literals
    else:
        with open(os.path.join(REF_SRC, "init.c")) as f:
            init = patch_init(f.read(), a, rin, rmax, beta)
    with open(os.path.join(gen, "init.c"), "w") as f:
        f.write(init)
    if cool:
        # cooleos.c with the table fill in this process (no forked workers,
        # cooleos.c:47-51), cache files that can never be found or written (a stale
        # file from another generator would otherwise be loaded, cache4d.c:45-120),
        # and the checker hooks appended to the same translation unit
        src = open(os.path.join(REF_SRC, "cooleos.c")).read()
        src = _sub1(r"^#define CACHETHREADS 4", "#define CACHETHREADS 0", src, "CACHETHREADS mpi")
        src = _sub1(r"^#define CACHETHREADS 6", "#define CACHETHREADS 0", src, "CACHETHREADS")
        src = _sub1(r'sprintf \(fname, "cache/cache_blh_', 'sprintf (fname, "/dev/null/cache_blh_',
                    src, "cache file")
        src += '\n#include "%s"\n' % os.path.join(HERE, "cool_hooks.inc")
        with open(os.path.join(gen, "cooleos.c"), "w") as f:
            f.write(src)
    flags = ["g++", "-O2", "-ffp-contract=off", "-fPIC", "-w", "-DMPI_USED",
             "-Dmain=harm_reference_main", "-I" + gen, "-I-",
             "-I" + os.path.join(HERE, "fakempi"), "-I" + REF_SRC]
    shim = name in SHIM_CONFIGS
    objs = []
    sources = [s for s in SOURCES if not (shim and s in SHIM_REPLACES)]
    for s in sources + (["tracers"] if tracers else []) + (["cache4d", "akima"] if cool else []):
        o = os.path.join(obj, s + ".o")
        run(flags + ["-x", "c++", "-c", os.path.join(REF_SRC, s + ".c"), "-o", o])
        objs.append(o)
    o = os.path.join(obj, "init.o")
    run(flags + ["-x", "c++", "-c", os.path.join(gen, "init.c"), "-o", o])
    objs.append(o)
    if cool:
        o = os.path.join(obj, "cooleos.o")
        run(flags + ["-x", "c++", "-c", os.path.join(gen, "cooleos.c"), "-o", o])
        objs.append(o)
        o = os.path.join(obj, "eos_standin.o")
        run(["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-c", os.path.join(HERE, "eos_standin.c"), "-o", o])
        objs.append(o)
    o = os.path.join(obj, "refdrv.o")
    run(flags + (["-DHARM_SHIM_BUILD"] if shim else []) + ["-c", os.path.join(HERE, "refdrv.cpp"), "-o", o])
    objs.append(o)
    libs = []
    if shim:
        pkg = os.path.join(ROOT, "harm_cool_b200")
        o = os.path.join(obj, "harm_gpu.o")
        run(flags + ["-I" + os.path.join(ROOT, "include"), "-c", os.path.join(pkg, "shim", "harm_gpu.cpp"),
                     "-o", o])
        objs.append(o)
        libs = ["-L" + pkg, "-lharm_b200", "-Wl,-rpath,$ORIGIN/../../../harm_cool_b200"]
    if tracers:
        # tracers.c scales its dump files by RHO_UNIT and T_UNIT, defined in cooleos.c,
        # which needs the Fortran EOS; the checker reads no dump file
        o = os.path.join(obj, "tracer_units.o")
        run(flags + ["-c", os.path.join(HERE, "tracer_units.cpp"), "-o", o])
        objs.append(o)
    o = os.path.join(obj, "fakempi.o")
    run(["gcc", "-O2", "-fPIC", "-c", os.path.join(HERE, "fakempi", "fakempi.c"), "-o", o])
    objs.append(o)
    run(["g++", "-shared", "-o", lib] + objs + libs + ["-lm"])
    run(["g++", "-O2", "-o", exe, os.path.join(HERE, "refbench.cpp"), lib,
         "-Wl,-rpath,$ORIGIN", "-lm"])
    return lib


# Timing builds: the reference's own objects at -O3, the fastest of the flag
# sets tried for the CPU baseline on this path's 288x256x4 step (Xeon with
# AVX-512, g++ 13): -O3 3.2e5 zone-cycles/s per core, -O3 -march=x86-64-v3
# (AVX2) 3.0e5, -O2 2.8e5, -O3 -march=x86-64-v4 (AVX-512, what -march=native
# selects there) 2.5e5.  Not a parity build: the parity builds above keep -O2
# -ffp-contract=off.
TIMING_CONFIGS = ("c2s",)
TIMING_FLAGS = ["-O3"]


def build_timing(name, force=False):
    """oracle/_ref/<name>/refbench_o3 (with libharmref_o3.so)."""
    cdir = os.path.join(OUT, name)
    gen = os.path.join(cdir, "gen")
    obj = os.path.join(cdir, "obj_o3")
    lib = os.path.join(cdir, "libharmref_o3.so")
    exe = os.path.join(cdir, "refbench_o3")
    if not force and os.path.exists(lib) and os.path.exists(exe):
        return exe
    build_config(name)   # the patched headers in gen/
    os.makedirs(obj, exist_ok=True)
    flags = ["g++"] + TIMING_FLAGS + ["-fPIC", "-w", "-DMPI_USED", "-Dmain=harm_reference_main", "-I" + gen, "-I-",
                                      "-I" + os.path.join(HERE, "fakempi"), "-I" + REF_SRC]
    objs = []
    for s in SOURCES:
        o = os.path.join(obj, s + ".o")
        run(flags + ["-x", "c++", "-c", os.path.join(REF_SRC, s + ".c"), "-o", o])
        objs.append(o)
    for src, o in ((os.path.join(gen, "init.c"), "init.o"), (os.path.join(HERE, "refdrv.cpp"), "refdrv.o")):
        o = os.path.join(obj, o)
        run(flags + (["-x", "c++"] if src.endswith(".c") else []) + ["-c", src, "-o", o])
        objs.append(o)
    o = os.path.join(obj, "fakempi.o")
    run(["gcc"] + TIMING_FLAGS + ["-fPIC", "-c", os.path.join(HERE, "fakempi", "fakempi.c"), "-o", o])
    objs.append(o)
    run(["g++", "-shared", "-o", lib] + objs + ["-lm"])
    run(["g++", "-O2", "-o", exe, os.path.join(HERE, "refbench.cpp"), lib, "-Wl,-rpath,$ORIGIN", "-lm"])
    return exe


def build_all(force=False):
    if not os.path.isdir(REF_SRC):
        return []
    return [build_config(n, force) for n in CONFIGS] + [build_timing(n, force) for n in TIMING_CONFIGS]


def shim_stale(name):
    """The drop-in build is older than the shim or the library it links."""
    lib = os.path.join(OUT, name, "libharmref.so")
    deps = [os.path.join(ROOT, "harm_cool_b200", "shim", "harm_gpu.cpp"),
            os.path.join(ROOT, "harm_cool_b200", "libharm_b200.so"), os.path.join(ROOT, "include", "harm_b200.h")]
    return not os.path.exists(lib) or os.path.getmtime(lib) < max(os.path.getmtime(d) for d in deps if os.path.exists(d))


if __name__ == "__main__":
    names = sys.argv[1:] or list(CONFIGS)
    for n in names:
        print(build_config(n, force=True))
