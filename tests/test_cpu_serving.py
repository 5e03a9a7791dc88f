"""The serving loop's scheduler (tidegbm_b200/csrc/serving.h), host only: admission by
memory budget and free slots in arrival order, continuous admission of requests arriving
while others run, per-request failures, refusal of oversized requests, latency quantiles.
The C++ checks in tests/cpp/test_scheduler.cpp are compiled and run here."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_scheduler(tmp_path):
    exe = tmp_path / "test_scheduler"
    subprocess.run(["g++", "-O1", "-std=c++17", "-pthread", "-Wall", "-I", os.path.join(ROOT, "tidegbm_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "test_scheduler.cpp"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == "ok"
