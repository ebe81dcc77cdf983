"""CPU: the device division code (up_dev.cuh: reciprocal_u32, Knuth D with
FP64 quotient-digit estimates, the reference's divide rule) compiled for the
host through tests/devarith/host_shims.h and run on seeded inputs by
tests/devarith/divcheck.cpp: exact reciprocals, x == q*b + r with r < b on
random, structured and constructed operands, and div_round against the C
oracle on the precision-sweep shapes."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "devarith", "divcheck.cpp")
ORACLE = os.path.join(ROOT, "oracle", "_build")

pytestmark = pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")


def test_device_division_on_the_host(tmp_path):
    exe = str(tmp_path / "divcheck")
    subprocess.run(["g++", "-std=c++17", "-O2", "-frounding-math", "-ffp-contract=off", "-Wno-unknown-pragmas",
                    "-o", exe, SRC, f"-L{ORACLE}", "-loracle", f"-Wl,-rpath,{ORACLE}"], check=True)
    r = subprocess.run([exe, "200000", "20261203"], capture_output=True, text=True, timeout=300)
    lines = [ln.split() for ln in r.stdout.splitlines() if ln and not ln.startswith(("divmod<", "div_round p"))
             or len(ln.split()) == 3]
    checks = {ln[0]: (int(ln[1]), int(ln[2])) for ln in lines if len(ln) == 3 and ln[1].isdigit()}
    assert r.returncode == 0, r.stdout
    assert len(checks) >= 15
    assert all(bad == 0 and n > 0 for n, bad in checks.values()), checks
