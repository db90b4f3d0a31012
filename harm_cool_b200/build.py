"""Build libharm_b200.so in-tree for sm_100a.

The CUDA translation unit is compiled with -fmad=false: every multiply and
add stays a separate IEEE operation, as in the reference's SSE2 build, which
is what lets the FP64 path reproduce the reference bit for bit.  The host
set-up code is compiled by g++ with the reference's own -O2 and
-ffp-contract=off so that its libm calls and arithmetic match set_grid().
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libharm_b200.so")
BUILD = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _sources():
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))] + [
        os.path.join(ROOT, "include", "harm_b200.h")]


def _includes(path, seen=None):
    """The file and every local header it includes, transitively."""
    import re
    seen = set() if seen is None else seen
    if path in seen or not os.path.exists(path):
        return seen
    seen.add(path)
    for name in re.findall(r'^#include "([^"]+)"', open(path).read(), re.M):
        for d in (CSRC, os.path.join(ROOT, "include")):
            if os.path.exists(os.path.join(d, name)):
                _includes(os.path.join(d, name), seen)
                break
    return seen


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


# translation unit -> extra nvcc flags
UNITS = {
    "harm_api.cu": ["-fmad=false"],     # shared kernels and the C ABI
    "harm_exact.cu": ["-fmad=false"],   # the FP64 step, bit-compatible with the reference
    "harm_mixed.cu": ["-fmad=true"],    # the mixed-precision step
    "harm_noalloc.cu": ["-fmad=false"],  # batch inversion on a fixed device buffer
    "harm_tracers.cu": ["-fmad=false"],  # tracer particles
    "harm_diag.cu": ["-fmad=false"],     # diag() integrals and div B
    "harm_restart.cu": ["-fmad=false"],  # restart files in the reference's format
    "harm_eos.cu": ["-fmad=false"],      # run-time COOL_EOS tables and batch calls
    "harm_cool.cu": ["-fmad=false"],     # the COOL_EOS step and Utoprim_5d
    "harm_dump.cu": ["-fmad=false"],     # the ASCII dump format
    "harm_adjoint.cu": ["-fmad=false"],  # the discrete adjoint (values identical to the step's)
    "harm_peak.cu": ["-fmad=false"],     # measured FP64 pipe rates (roofline denominators)
    "harm_nu.cu": ["-fmad=false"],       # COOL_EOS table generator on the device
}

# host-only units, compiled by g++ with the reference's -O2 and no contraction
HOST_UNITS = ["host_setup.cpp", "harm_nu_host.cpp"]


def build(force=False, verbose=False):
    """Compile the library if any source is newer than it; return its path."""
    if (not force and os.path.exists(LIB)
            and os.path.getmtime(LIB) >= max(os.path.getmtime(s) for s in _sources())):
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    inc = ["-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
    objs = []
    for unit in HOST_UNITS:
        host_o = os.path.join(BUILD, unit.replace(".cpp", ".o"))
        _run(["g++", "-O2", "-ffp-contract=off", "-fPIC", "-std=c++17", "-c",
              os.path.join(CSRC, unit), "-o", host_o] + inc)
        objs.append(host_o)

    # a unit is recompiled when its object is older than the unit or any header it includes
    def compile_unit(item):
        unit, flags = item
        o = os.path.join(BUILD, unit.replace(".cu", ".o"))
        src = os.path.join(CSRC, unit)
        newest = max(os.path.getmtime(f) for f in _includes(src))
        if not force and os.path.exists(o) and os.path.getmtime(o) >= newest:
            return o, ""
        out = _run([NVCC] + ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xptxas", "-v", "-Xcompiler", "-fPIC",
                                    "-Xcompiler", "-ffp-contract=off", "-c", os.path.join(CSRC, unit),
                                    "-o", o] + flags + inc)
        return o, out

    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as pool:
        for o, out in pool.map(compile_unit, UNITS.items()):
            if verbose:
                print(out)
            objs.append(o)
    tmp = LIB + ".tmp"
    _run([NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart", "-lpthread"])
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose=True)
    print(LIB)
