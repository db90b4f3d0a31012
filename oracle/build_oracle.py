"""Compile the CPU oracle (harm_oracle.c, cooleos_oracle.c) into oracle/_build/libharm_oracle.so.

TEST INFRASTRUCTURE ONLY.  -ffp-contract=off keeps every multiply and add
separate, as the reference compiled for SSE2 does, so the restatement can be
compared with the reference bit for bit.
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_build", "libharm_oracle.so")


def build(force=False):
    srcs = [os.path.join(HERE, f) for f in ("harm_oracle.c", "cooleos_oracle.c", "eos_standin.c")]
    hdr = os.path.join(HERE, "harm_oracle.h")
    if (not force and os.path.exists(OUT)
            and os.path.getmtime(OUT) > max(os.path.getmtime(f) for f in srcs + [hdr])):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-std=c99",
                    "-Wall", "-Wno-unused-variable"] + srcs + ["-o", OUT, "-lm"], check=True)
    return OUT


if __name__ == "__main__":
    print(build(force=True))
