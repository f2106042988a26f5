"""The fixed-divisor division of k_rhs (div_fixed, mit_jax_b200/csrc/cg2d_pressure.cu) restated in C
(tests/div_fixed_check.c) and compared bit for bit with the IEEE quotient on about 3 million dividends: the
method the kernel uses in place of dividing by deltaTMom. ISO C (no FMA contraction), glibc's fma."""

import shutil
import subprocess
from pathlib import Path

import pytest

HERE = Path(__file__).resolve().parent


def test_div_fixed_matches_ieee_division(tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    exe = tmp_path / "div_fixed_check"
    subprocess.run([cc, "-std=c11", "-O2", "-ffp-contract=off", "-o", str(exe), str(HERE / "div_fixed_check.c"),
                    "-lm"], check=True)
    out = subprocess.run([str(exe), "50000"], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout
    assert out.stdout.startswith("0 of "), out.stdout
