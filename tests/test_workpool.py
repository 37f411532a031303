"""Host-side pieces compiled and run on the CPU: the resolver's host team (xkaapi_b200/csrc/workpool.h)
and the handle map's decisions (xkaapi_b200/csrc/handles.h)."""
import os
import subprocess

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_workpool_runs_every_member_each_time(tmp_path):
    exe = str(tmp_path / "workpool_test")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-pthread", os.path.join(REPO, "tests", "cpp", "workpool_test.cc"),
                    "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stderr


def test_handle_map_decisions(tmp_path):
    """The handle map's extra-writer decisions (xkaapi_b200/csrc/handles.h) in exact and C API mode."""
    exe = str(tmp_path / "handles_test")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", os.path.join(REPO, "tests", "cpp", "handles_test.cc"),
                    "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stderr


def test_pool_arrays_and_parked_reservations(tmp_path):
    """The spawn pools (xkaapi_b200/csrc/pool.h): fixed reservations, growth by remapping, and a
    released fixed reservation reused by the next one of the same size (pages still backed)."""
    exe = str(tmp_path / "pool_test")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-pthread", os.path.join(REPO, "tests", "cpp", "pool_test.cc"),
                    "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stderr
