"""Host check of the line FFT engines: the compile-time engines (lengths 16 ...
512, radix-16 codelets) and the runtime-plan engine run sequentially on the CPU
(tests/native/fft_engine_host.cu, built with nvcc as host code) against a
direct DFT in long double, forward and inverse, float and double."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def _nvcc():
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    return None


@pytest.mark.skipif(_nvcc() is None, reason="nvcc not available")
def test_line_fft_engines_host(tmp_path):
    exe = str(tmp_path / "fft_engine_host")
    src = os.path.join(HERE, "native", "fft_engine_host.cu")
    r = subprocess.run([_nvcc(), "-std=c++17", "--expt-relaxed-constexpr", "-O2",
                        "-Wno-deprecated-gpu-targets", "-o", exe, src],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout
    assert "ALL OK" in r.stdout
    assert r.stdout.count(" ok") >= 64
