"""Host check of the device index arithmetic (mcpi_b200/csrc/fock.cuh).

tests/cpp/fock_check.cpp includes the same header the kernels use and checks,
on the CPU, the decode of every configuration and the index of every one- and
two-particle jump against a brute-force enumeration in the reference's order,
including that each jump index stays inside its target space (the kernels
gather through these indices). No GPU needed."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_fock_index_arithmetic(tmp_path):
    exe = tmp_path / "fock_check"
    subprocess.run(["g++", "-O2", "-std=c++17", os.path.join(ROOT, "tests", "cpp", "fock_check.cpp"),
                    "-o", str(exe)], check=True)
    r = subprocess.run([str(exe), "large"], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr

