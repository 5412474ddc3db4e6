"""The server's matrix-cache policy (byte budget, least recently used
first, entries in use never evicted), compiled and run on the host."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_lru_budget_policy(tmp_path):
    exe = str(tmp_path / "lru_policy")
    r = subprocess.run(["/usr/bin/g++", "-O1", "-std=c++17", os.path.join(ROOT, "tests", "cpp", "lru_policy.cpp"),
                        "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout
    assert "failures 0" in r.stdout
