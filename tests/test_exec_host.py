"""The device step function (z80_exec.cuh) compiled for the host agrees
with the CPU oracle on every opcode (all A x F pairs, random other state)."""
import os
import subprocess

from conftest import ROOT


def test_exec_header_matches_oracle(tmp_path):
    exe = tmp_path / "exec_check"
    srcs = [os.path.join(ROOT, "tests", "native", "exec_check.cpp"),
            os.path.join(ROOT, "oracle", "z80_oracle_isa_cpu.cpp"),
            os.path.join(ROOT, "oracle", "z80_oracle_search.cpp")]
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", str(exe)] + srcs + ["-lpthread"], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("OK")


def test_bitsliced_step_matches_scalar(tmp_path):
    """The bit-sliced step (z80_bits.cuh, 32 states per step) agrees with the
    scalar step on every opcode, random full states and all values of A."""
    exe = tmp_path / "bits_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", str(exe),
                    os.path.join(ROOT, "tests", "native", "bits_check.cpp")], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("OK")


def test_bitsliced_sweep_layouts(tmp_path):
    """The planes the bit-sliced A-independent sweep builds for a group of 32
    A-blocks hold each block's decoded initial state (every sweep shape), and
    sweeping random pairs the way both bit-sliced kernels lay them out
    (A-independent: 32 blocks per word at A = 0 and 1; A-dependent: 32 values
    of A per word) reproduces the oracle's ExhaustiveCheck[Masked] verdicts."""
    exe = tmp_path / "xbits_check"
    srcs = [os.path.join(ROOT, "tests", "native", "xbits_check.cpp"),
            os.path.join(ROOT, "z80-optimizer_b200", "csrc", "z80_tables.cpp"),
            os.path.join(ROOT, "oracle", "z80_oracle_isa_cpu.cpp"),
            os.path.join(ROOT, "oracle", "z80_oracle_search.cpp")]
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", str(exe)] + srcs + ["-lpthread"], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("OK")
