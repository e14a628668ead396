import lzma
import os
import shutil
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).resolve().parent / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running")


def _ensure_oracle_built():
    lib = ROOT / "oracle" / "liboracle.so"
    if not lib.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "oracle"], check=True)


_ensure_oracle_built()


@pytest.fixture(scope="session")
def reference_tube(tmp_path_factory):
    """The reference-generated 512-element straight tube (case directory)."""
    d = tmp_path_factory.mktemp("reference_tube")
    for f in (GOLDEN / "reference_tube").glob("*.xz"):
        (d / f.name[:-3]).write_bytes(lzma.decompress(f.read_bytes()))
    return d


@pytest.fixture(scope="session")
def small_tube():
    """A generator tube small enough for exhaustive CPU checks: 4x4 core + 1 ring, 3 layers."""
    from tubularflowiga_b200 import meshgen
    return meshgen.straight_tube(1.5e-3, 6e-3, core=4, ring=1, layers=3)


@pytest.fixture(scope="session")
def cylinder_1280():
    from tubularflowiga_b200 import meshgen
    return meshgen.straight_cylinder_1280()


def have_reference_build() -> bool:
    from oracle import oracle
    return oracle.ref_available()


requires_ref = pytest.mark.skipif(not (ROOT / "oracle" / "_ref" / "libtfiga_ref.so").exists(),
                                  reason="reference element build (oracle/_ref) not present")
