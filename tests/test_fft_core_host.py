"""The shared-memory FFT building blocks of the Hilbert kernel (csrc/fft_core.cuh) driven on the
CPU: tests/fft_paired_host.cpp runs the device passes thread by thread. The paired form (two
transforms on the lanes of float2, used for the two inverse transforms of a row pair) must equal
the scalar form bit for bit in each lane, and both must match an FP64 DFT, for every supported
power-of-two length up to 8192 and a nonzero bank skew; and the scalar transform with its exchange
arrays split into slices of 2^14 elements (one per CTA of the thread-block-cluster kernel) must
equal the single-array one bit for bit and an FP64 FFT, for 2^14 .. 2^17 points."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "cuda_ultrasound_toolkit_b200", "csrc")
CUDA_INCLUDE = "/usr/local/cuda/include"


def test_paired_fft_matches_scalar_and_fp64(tmp_path):
    exe = tmp_path / "fft_paired_host"
    subprocess.run(["g++", "-std=c++20", "-O2", "-I", CSRC, "-I", CUDA_INCLUDE,
                    os.path.join(HERE, "fft_paired_host.cpp"), "-o", str(exe)], check=True)
    res = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    print(res.stdout)
    assert res.returncode == 0, res.stdout + res.stderr
    assert res.stdout.count("bit for bit") == 34
