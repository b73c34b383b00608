"""The device code's quotient shortcuts against IEEE division, on the CPU:
div_rn (a / b from one reciprocal of b per temperature with two FMA
corrections, the CEA curve terms) and quotient_below (the shock detector's
compression test without the division outside a 2^-49 band).  Both claim the
division's exact outcome; tests/div_rn_check.c restates them in C and checks
millions of operands, the CEA divisors and values next to the thresholds."""
import os
import shutil
import subprocess
import tempfile

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_quotient_shortcuts_match_ieee_division():
    with tempfile.TemporaryDirectory() as tmp:
        exe = os.path.join(tmp, "div_rn_check")
        # -ffp-contract=off: every multiply and add rounded on its own, as the
        # device units are built (-fmad=false); fma() stays fused
        subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-o", exe,
                        os.path.join(HERE, "div_rn_check.c"), "-lm"], check=True)
        out = subprocess.run([exe, "4000000"], capture_output=True, text=True)
        assert out.returncode == 0, out.stdout + out.stderr
        assert "div_rn mismatches 0 quotient_below mismatches 0" in out.stdout
