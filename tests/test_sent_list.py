"""The TCP sent list on the CPU: tests/sent_list.cpp, built with g++ over twins_b200/csrc/tb_tcp.cuh,
mirrors random opens (appends and splits), joins, flag changes and whole-list losses on a plain
per-item model and checks every item's flags, the byte counters, the sacked-item count and the
candidate search bound after each step, on rings whose head lies anywhere (shifts that wrap)."""
import shutil
import subprocess

import pytest

from conftest import ROOT


def test_sent_list_matches_model(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("g++ is not here")
    exe = tmp_path / "sent_list"
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wno-unknown-pragmas", f"-I{ROOT / 'twins_b200' / 'csrc'}", "-o", str(exe),
                    str(ROOT / "tests" / "sent_list.cpp")], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-500:]
