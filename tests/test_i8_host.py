"""CPU test of the mixed plans' tensor-core M2L arithmetic (csrc/i8_ops.h): the
dense per-offset operator reproduces direct sums of the potential and the
field to truncation accuracy; four 8-bit slices with exact integer sums
reproduce the FP64 operator to ~1e-9 of the largest coefficient; the int32
sums cannot overflow up to the highest order the library uses them at."""
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
CSRC = ROOT / "simplefmm_b200" / "csrc"


def test_i8_arithmetic(tmp_path):
    exe = tmp_path / "i8_test"
    subprocess.run(["g++", "-std=c++17", "-O2", f"-I{CSRC}", f"-I{ROOT / 'include'}", str(ROOT / "tests/native/i8_test.cpp"),
                    str(CSRC / "tables.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout
    assert "i8 ok" in r.stdout
