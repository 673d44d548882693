"""Host logic of the FEL / MEME drivers on the CPU (no GPU): the lockstep loop with a fake evaluator.

tests/harness/sitefit_lockstep.cpp links the drivers' host sources with a CPU
stand-in for the device evaluator.  Every run must finish with H3G_OK (the
loop checks, per batch, that no eigensystem slot is solved twice, that no warm
start reads a slot solved in the same launch and that every request reads a
solved slot) and repeated runs must agree bit for bit.
"""
import pathlib
import shutil
import subprocess

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
CSRC = ROOT / "hyphy-3_b200" / "csrc"


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no host C++ compiler")
    exe = tmp_path_factory.mktemp("harness") / "sitefit_lockstep"
    cmd = [gxx, "-O1", "-std=c++20", f"-I{ROOT / 'include'}", f"-I{CSRC}", "-I/usr/local/cuda/include", "-o", str(exe),
           str(ROOT / "tests" / "harness" / "sitefit_lockstep.cpp"), str(CSRC / "h3g_sitefit.cpp"),
           str(CSRC / "h3g_fel_driver.cpp"), str(CSRC / "h3g_meme_driver.cpp")]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def _run(exe, *sizes):
    r = subprocess.run([str(exe), *map(str, sizes)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout.splitlines()


def test_lockstep_batches_are_consistent(harness):
    lines = _run(harness, 7, 64, 300, 1200)
    assert len(lines) == 4 and all(" checksum " in ln for ln in lines)


def test_lockstep_is_deterministic(harness):
    a = _run(harness, 300, 300)
    b = _run(harness, 300)
    assert a[0] == a[1] == b[0]
