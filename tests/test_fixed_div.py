"""The fixed-divisor quotient of the ray cast's leaf set-up
(voxviz_b200/csrc/fixed_div.h) against IEEE division, exhaustively over a's
significands for every brick-pool texel dimension.  The kernels use it in
place of the division, so their bit-exact parity rests on this."""
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_fixed_div_equals_ieee_division(tmp_path):
    exe = tmp_path / "fixed_div_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-mfma", "-fopenmp",
                    str(ROOT / "tests" / "fixed_div_check.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    checks, bad = map(int, r.stdout.split()[-2:])
    assert bad == 0 and checks == 102 * 3 * (1 << 23)
