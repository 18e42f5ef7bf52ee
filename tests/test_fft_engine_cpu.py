"""The Stockham engine of tara2d_b200/csrc/fft_core.cuh, run on the host.

tests/cpu_sim/fft_sim.cpp executes the same per-thread stage code
(BatchFFT::in_pos/out_pos/compute) for every thread of a batch and compares
every radix plan against a long-double DFT, both directions."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def test_stockham_engine_matches_dft(tmp_path):
    exe = tmp_path / "fft_sim"
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", str(exe), os.path.join(HERE, "cpu_sim", "fft_sim.cpp")],
                   check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL OK" in r.stdout
    # the 512-point row transforms (16 values per thread) take their last
    # exchange as the tid ^ 16 lane swap; no other plan does
    for line in r.stdout.splitlines():
        if "lane_swaps=" in line:
            want = "lane_swaps=1" if ("L=  512 B=1 P=16" in line) else "lane_swaps=0"
            assert want in line, line
