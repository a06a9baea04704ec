"""Shared test set-up: paths, the `gpu` marker, and in-tree builds of the library and oracle."""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
PKG = REPO / "nrrs-code_b200"
ORACLE = REPO / "oracle"
for p in (str(PKG), str(ORACLE), str(REPO)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU")
    config.addinivalue_line("markers", "slow: long-running CPU test")


def _ensure_built():
    lib = PKG / "lib" / "libnrrs_b200.so"
    if not lib.exists():
        subprocess.run([sys.executable, str(PKG / "build.py")], check=True)
    if not (ORACLE / "_build" / "libnrrs_oracle.so").exists():
        subprocess.run(["make", "-s", "-C", str(ORACLE)], check=True)
    ref = os.environ.get("NRRS_REFERENCE", "/root/reference")
    if not (ORACLE / "_ref" / "libnrrs_ref.so").exists() and Path(ref).is_dir():
        # builds only where the reference checkout is present (see oracle/Makefile)
        subprocess.run(["make", "-s", "-C", str(ORACLE), "ref-if-present", f"REF={ref}"],
                       check=False)


_ensure_built()


@pytest.fixture(scope="session")
def has_gpu() -> bool:
    import nrrs_b200 as nb
    return bool(nb.lib().nrrs_device_available())
