"""The C++ side of the boundary: tests/native/ffvils_gpu_parity.cpp drives the
solve through FFVILSGpu (the FFVILS-shaped C++ mirror) and the C ABI, as
FFV's Solver::UpdateP would, and compares every residual and pressure value
with the oracle."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.gpu
def test_cpp_ffvils_mirror_bitwise(tmp_path):
    exe = str(tmp_path / "ffvils_gpu_parity")
    lib = os.path.join(ROOT, "ffv-hc_b200")
    orc = os.path.join(ROOT, "oracle")
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", exe,
                    os.path.join(ROOT, "tests", "native", "ffvils_gpu_parity.cpp"),
                    f"-L{lib}", "-lffvhc_b200", f"-L{orc}", "-lffvoracle",
                    f"-Wl,-rpath,{lib}:{orc}"], check=True)
    out = subprocess.run([exe, "2"], capture_output=True, text=True, timeout=600)
    print(out.stdout)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "mismatches 0/0" in out.stdout


def test_cpp_ffvils_mirror_compiles(tmp_path):
    """The C++ mirror and the driver build against the C ABI header alone."""
    exe = str(tmp_path / "ffvils_gpu_parity")
    lib = os.path.join(ROOT, "ffv-hc_b200")
    orc = os.path.join(ROOT, "oracle")
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", exe,
                    os.path.join(ROOT, "tests", "native", "ffvils_gpu_parity.cpp"),
                    f"-L{lib}", "-lffvhc_b200", f"-L{orc}", "-lffvoracle",
                    f"-Wl,-rpath,{lib}:{orc}"], check=True)
    assert os.path.exists(exe)
