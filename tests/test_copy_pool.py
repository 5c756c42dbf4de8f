"""The Go-slice path's host copy pool (pure host C++), built with g++ and run
under a time limit: copies from a freshly created pool (workers still
starting), mixed sizes, several callers in turn, each checked byte for
byte."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_copy_pool(tmp_path):
    exe = str(tmp_path / "copy_pool_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", os.path.join(ROOT, "algo-fft_b200", "csrc"),
                    os.path.join(ROOT, "tests", "copy_pool_check.cpp"), "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "copy pool: ok" in r.stdout
