"""CPU: the drop-in build (the reference's host code with harm_cool_b200/shim/
harm_gpu.cpp linked in place of step_ch.c, bounds.c, fixup.c, utoprim_2d.c)
defines the reference's own C++ symbols for the replaced routines, takes them
from the shim rather than from the reference, and loads libharm_b200."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# decs.h:548-610 compiled as C++ (Makefile:17-29)
REPLACED = {"_Z7step_chv": "step_ch()", "_Z10bound_primPd": "bound_prim(double*)", "_Z5fixupPd": "fixup(double*)",
            "_Z13fixup_utoprimPd": "fixup_utoprim(double*)", "_Z10fixup1zoneiiiPd": "fixup1zone(int,int,int,double*)",
            "_Z8set_Katmv": "set_Katm()", "_Z10Utoprim_2dPdPA4_dS1_dS_": "Utoprim_2d(U, gcov, gcon, gdet, prim)"}
# defined only in the replaced reference files
GONE = ("_Z7advancePdS_dS_i", "_Z8fluxcalcPdS_ii", "_Z12inflow_checkPdiiii", "_Z15get_rho_u_floordddPdS_")


@pytest.mark.parametrize("cfg", ["g2d", "g3d"])
def test_drop_in_build_takes_the_replaced_routines_from_the_shim(cfg):
    lib = os.path.join(ROOT, "oracle", "_ref", cfg, "libharmref.so")
    if not os.path.exists(lib):
        pytest.skip("drop-in build not made here (needs the reference tree)")
    shim_o = os.path.join(ROOT, "oracle", "_ref", cfg, "obj", "harm_gpu.o")
    defined = set(l.split()[-1] for l in subprocess.run(["nm", "--defined-only", lib], capture_output=True,
                                                         text=True).stdout.splitlines() if l.strip())
    from_shim = set(l.split()[-1] for l in subprocess.run(["nm", "--defined-only", shim_o], capture_output=True,
                                                          text=True).stdout.splitlines() if l.strip())
    for sym, name in REPLACED.items():
        assert sym in defined, name
        assert sym in from_shim, name
    for sym in GONE:
        assert sym not in defined, sym
    deps = subprocess.run(["ldd", lib], capture_output=True, text=True).stdout
    assert "libharm_b200.so" in deps and "not found" not in deps
