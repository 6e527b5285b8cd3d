import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: full-size workloads")


def _gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session", autouse=True)
def built_library():
    """The product library (and, where its sources are present, the checker
    libraries) are built before any test runs; a missing library fails loudly."""
    from msa_b200 import build
    build.build()
    import subprocess
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], check=True)
    from oracle.oracle import REFERENCE_ROOT
    built = all((ROOT / "oracle/_ref" / f).exists() for f in ("libmuseqa_ref.so", "libmuseqa_b200.so"))
    if (REFERENCE_ROOT / "src").is_dir() and not built:
        subprocess.run(["make", "-s", "-j8", "-C", str(ROOT / "oracle"), "ref",
                        f"MSA_REFERENCE={REFERENCE_ROOT}"], check=True)
    yield


@pytest.fixture(scope="session")
def gpu():
    if not _gpu_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
    from msa_b200 import runtime
    return runtime.context(0)


@pytest.fixture(scope="session")
def golden():
    import json
    return json.loads((ROOT / "tests/golden/golden.json").read_text())


@pytest.fixture(scope="session")
def ref():
    from oracle import oracle as O
    lib = O.reference()
    if lib is None:
        pytest.skip("reference oracle (oracle/_ref) not built")
    return O
