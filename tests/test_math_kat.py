"""Known-answer checks of the product's arithmetic (tb_common.cuh built for the host), no GPU:

- Time::GetSeconds (Q64.64 times the inverse of 10^12, x87 sum): identical to long double;
- MRG32k3a: the division-free residue equals RngStream's division form on every draw;
- pow: correctly rounded, so it differs from glibc's pow (which ns-3 calls) only where glibc is
  not (about 0.08% of inputs, by one ulp); the truncated cubes Cubic uses never differ, and the
  cube roots of Cubic's integer inputs, where some do differ, are tabulated from the host libm
  by the library (tb_capi.cu), so Cubic's K equals ns-3's.
"""
import subprocess
from pathlib import Path

from conftest import ROOT


def test_math_kat(tmp_path):
    exe = tmp_path / "math_kat"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-o", str(exe), str(ROOT / "tests" / "kat" / "math_kat.cpp")],
                   check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    v = {out[i]: (int(out[i + 1]), int(out[i + 2])) for i in range(0, len(out), 3)}
    assert v["seconds"][0] == 0 and v["seconds"][1] == 2000000
    assert v["rng"][0] == 0 and v["rng"][1] == 4000000
    assert v["trunc"][0] == 0
    assert v["root"][0] < 0.002 * v["root"][1]
    assert v["cube"][0] < 0.002 * v["cube"][1]
    assert v["kinputs"][0] < 0.005 * v["kinputs"][1]
