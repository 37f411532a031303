"""The resolver's host team (xkaapi_b200/csrc/workpool.h), compiled and run on the CPU."""
import os
import subprocess

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_workpool_runs_every_member_each_time(tmp_path):
    exe = str(tmp_path / "workpool_test")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-pthread", os.path.join(REPO, "tests", "cpp", "workpool_test.cc"),
                    "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stderr
