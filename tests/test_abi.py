"""CPU: the C-ABI library loads and exports every entry point include/harm_b200.h declares."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    text = open(os.path.join(ROOT, "include", "harm_b200.h")).read()
    return sorted(set(re.findall(r"\b(harm_[a-z0-9_]+)\s*\(", text)))


def test_exports_every_declared_symbol(harm_lib):
    from harm_cool_b200 import LIB_PATH
    names = declared()
    assert len(names) >= 20
    out = subprocess.run(["nm", "-D", "--defined-only", LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (harm_[a-z0-9_]+)\b", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    for n in names:
        assert hasattr(harm_lib, n)


def test_library_is_not_linked_to_the_oracle(harm_lib):
    from harm_cool_b200 import LIB_PATH
    out = subprocess.run(["nm", "-D", LIB_PATH], capture_output=True, text=True).stdout
    assert "ora_" not in out and "ref_" not in out
    deps = subprocess.run(["ldd", LIB_PATH], capture_output=True, text=True).stdout
    assert "oracle" not in deps and "harmref" not in deps


def test_create_reports_missing_gpu(harm_lib):
    import harm_cool_b200 as hc
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("a GPU is present")
    pr = hc.torus_problem(16, 16, 1)
    with pytest.raises(hc.HarmError) as e:
        hc.Context(pr)
    assert e.value.code == -3


def test_grid_arguments_are_checked(harm_lib):
    import harm_cool_b200 as hc
    with pytest.raises(hc.HarmError):
        hc.torus_problem(16, 16, 3)   # odd n3 > 1 is rejected like the reference (mpi.c:357-360)
    with pytest.raises(hc.HarmError):
        hc.torus_problem(2, 16, 1)
