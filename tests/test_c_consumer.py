"""The C-ABI from plain C. tests/c_consumer/nrrs_consumer.c builds with gcc as strict C11
(-Wall -Wextra -Werror -pedantic) against include/nrrs.h and the library, and the header also
compiles as C++17. On a B200 the program runs one depth of the path through nrrs_step and checks
that nrrs_decide_emit on the step's factors emits the same queue; without a device it reports
that and runs nothing."""
from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

import nrrs_b200 as nb

REPO = Path(__file__).resolve().parents[1]
CUDA = Path("/usr/local/cuda")


def build(tmp: Path) -> Path:
    exe = tmp / "nrrs_consumer"
    lib_dir = nb.LIB_PATH.parent
    cmd = ["gcc", "-std=c11", "-O2", "-Wall", "-Wextra", "-Werror", "-pedantic",
           f"-I{REPO / 'include'}", f"-I{CUDA / 'include'}",
           str(REPO / "tests" / "c_consumer" / "nrrs_consumer.c"),
           f"-L{lib_dir}", "-lnrrs_b200", f"-L{CUDA / 'lib64'}", "-lcudart",
           f"-Wl,-rpath,{lib_dir}", f"-Wl,-rpath,{CUDA / 'lib64'}", "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_c_consumer_builds_and_header_compiles_as_cxx(tmp_path):
    exe = build(tmp_path)
    src = tmp_path / "header.cpp"
    src.write_text('#include "nrrs.h"\nint main() { nrrs_config c; nrrs_config_default(&c); '
                   'return c.n_levels == 16 ? 0 : 1; }\n')
    r = subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", f"-I{REPO / 'include'}",
                        "-c", str(src), "-o", str(tmp_path / "header.o")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    if nb.lib().nrrs_device_available() != 1:
        r = subprocess.run([str(exe), "1000"], capture_output=True, text=True, timeout=120)
        assert r.returncode == 2 and "no sm_100 device" in r.stdout


@pytest.mark.gpu
def test_c_consumer_runs_one_depth(tmp_path):
    exe = build(tmp_path)
    r = subprocess.run([str(exe), "300001"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("ok n=300001 emitted=")
