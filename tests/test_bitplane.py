"""CPU test of the bit-plane transposes shared by the encoder and decoder."""
import os
import subprocess
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "sc25-lscomp_b200", "csrc")


def test_bitplane_transposes():
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "bitplane_check")
        subprocess.run(["g++", "-O2", "-std=c++17", "-I", CSRC, "-o", exe, os.path.join(HERE, "bitplane_check.cpp")],
                       check=True)
        out = subprocess.run([exe], capture_output=True, text=True)
        assert out.returncode == 0, out.stdout + out.stderr
        assert "mismatches 0" in out.stdout
