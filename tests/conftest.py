"""pytest configuration: the `gpu` marker and shared fixtures.

Tests marked `gpu` need a B200 and the built library; everything else runs
on CPU.  The oracle build (oracle/_ref) is test infrastructure: its C
restatement always builds with gcc; the host build of the reference exists
only where the reference sources were present.
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def oracle_built():
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], check=True,
                   stdout=subprocess.DEVNULL)
    return True


@pytest.fixture(scope="session")
def saru_lib():
    from saruman_b200 import build, load
    build.build()
    return load()


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture
def report(pytestconfig):
    """Writes a line to the terminal even while output is captured (the
    full-size tests' candidate counts and content hashes)."""
    tr = pytestconfig.pluginmanager.getplugin("terminalreporter")

    def write(line: str) -> None:
        if tr is not None:
            tr.write_line(line)
        else:
            print(line)
    return write
