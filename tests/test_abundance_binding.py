"""CPU: harm_cool_b200/shim/harm_abundance.cpp gives the reference's Fortran
entry point abundance_(rho, T, HdFac, e, p, Qnu, tau, xnee, xnep)
(cooleos.c:58-59) over libharm_b200: a C caller built against that prototype
gets the library's node values, in the reference's argument order."""
import os
import subprocess

import numpy as np

import harm_cool_b200 as hc
from harm_cool_b200 import eos_tables as et

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CALLER = r"""
#include <stdio.h>
#include <stdlib.h>
void abundance_(double *rho, double *T, double *HdFac, double *e, double *p, double *Qnu, double *tau,
                double *xnee, double *xnep);
int main(int argc, char **argv)
{
  for (int k = 1; k + 2 < argc; k += 3) {
    double rho = atof(argv[k]), T = atof(argv[k + 1]), hd = atof(argv[k + 2]);
    double e, p, qnu, tau, xnee, xnep;
    abundance_(&rho, &T, &hd, &e, &p, &qnu, &tau, &xnee, &xnep);
    printf("%.17g %.17g %.17g %.17g %.17g %.17g\n", e, p, qnu, tau, xnee, xnep);
  }
  return 0;
}
"""


def test_abundance_entry_point_matches_the_library(harm_lib, tmp_path):
    src = tmp_path / "caller.c"
    src.write_text(CALLER)
    exe = tmp_path / "caller"
    libdir = os.path.join(ROOT, "harm_cool_b200")
    obj = tmp_path / "harm_abundance.o"
    subprocess.run(["g++", "-O2", "-c", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(libdir, "shim", "harm_abundance.cpp"), "-o", str(obj)], check=True)
    subprocess.run(["gcc", "-O2", str(src), str(obj), "-o", str(exe), "-L" + libdir, "-lharm_b200", "-lstdc++",
                    "-Wl,-rpath," + libdir], check=True)
    rho = np.array([1e6, 1e10, 1e13])
    T = np.array([5e9, 3e10, 2e11])
    hd = np.full(3, et.hdfac(8.0))
    args = [repr(float(v)) for k in range(3) for v in (rho[k], T[k], hd[k])]
    out = subprocess.run([str(exe)] + args, capture_output=True, text=True, check=True).stdout.split("\n")
    got = np.array([[float(x) for x in line.split()] for line in out if line.strip()])
    want = hc.nu_abundance(rho, T, hd)
    for i, k in enumerate(("e", "p", "qnu", "tau", "nee", "nep")):
        assert np.array_equal(got[:, i], want[k]), k
