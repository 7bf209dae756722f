"""CPU test of the CSR size guard: interaction-list and near-field totals
are summed in 64 bits and refused past INT32_MAX (no GPU needed)."""
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_csr_guard(tmp_path):
    exe = tmp_path / "csr_limits_test"
    subprocess.run(["g++", "-std=c++17", "-O1", f"-I{ROOT / 'simplefmm_b200' / 'csrc'}",
                    str(ROOT / "tests/native/csr_limits_test.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout
    assert "csr limits ok" in r.stdout
