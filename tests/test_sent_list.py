"""The TCP sent list on the CPU: tests/sent_list.cpp, built with g++ over twins_b200/csrc/tb_tcp.cuh,
mirrors random opens (appends and splits), joins, flag changes and whole-list losses on a plain
per-item model and checks every item's flags, the byte counters, the sacked-item count and the
candidate search bound after each step, on rings whose head lies anywhere (shifts that wrap); ACKs
that drop and cut items too; then the RTT history's first sends, retransmissions and ACKs against
a list scanned from its oldest entry. tests/rng_ahead.cpp, over twins_b200/csrc/tb_common.cuh, checks the
random stream's look-ahead table (the spraying draws of a switch slot computed out of order) against
the stream drawn one value at a time."""
import shutil
import subprocess

import pytest

from conftest import ROOT


def run_check(tmp_path, name):
    if shutil.which("g++") is None:
        pytest.skip("g++ is not here")
    exe = tmp_path / name
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-Wno-unknown-pragmas", f"-I{ROOT / 'twins_b200' / 'csrc'}", "-o",
                    str(exe), str(ROOT / "tests" / f"{name}.cpp")], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-500:]


def test_sent_list_matches_model(tmp_path):
    run_check(tmp_path, "sent_list")


def test_rng_look_ahead_matches_stream(tmp_path):
    run_check(tmp_path, "rng_ahead")
