import pathlib
import subprocess
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
for p in (ROOT / "oracle" / "_build", ROOT / "hyphy-3_b200" / "python", ROOT):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _ensure_oracle():
    try:
        import h3oracle  # noqa: F401
    except ImportError:
        subprocess.run(["make", "-C", str(ROOT / "oracle")], check=True, capture_output=True)


_ensure_oracle()


@pytest.fixture(scope="session")
def oracle():
    import h3oracle
    return h3oracle


@pytest.fixture(scope="session")
def known():
    import json
    return json.loads((GOLDEN / "known_answers.json").read_text())


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN
