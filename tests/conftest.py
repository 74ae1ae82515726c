"""Shared fixtures. GPU tests are marked `gpu`; everything else runs on the CPU."""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def reference_root():
    """The reference's source tree, for the tests that compile its examples unchanged: the
    environment variable TREESAP_REFERENCE, else the tree the oracle recipe was built from
    (recorded in oracle/_ref/reference_root.txt). None when neither exists on this machine."""
    import os

    cands = [os.environ.get("TREESAP_REFERENCE")]
    rec = ROOT / "oracle" / "_ref" / "reference_root.txt"
    if rec.exists():
        cands.append(rec.read_text().strip())
    for c in cands:
        if c and (Path(c) / "examples").is_dir() and (Path(c) / "src" / "treesap").is_dir():
            return Path(c)
    return None


REFERENCE_SKIP = ("reference sources not found: set TREESAP_REFERENCE to the treesap source tree "
                  "(or build the oracle recipe, which records it)")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


@pytest.fixture(scope="session")
def ctx():
    from treesap_b200 import Context

    c = Context(0)
    yield c
    c.close()


@pytest.fixture(scope="session")
def oracle():
    """The CPU checker: the reference build when present, else the plain-C restatement."""
    from oracle import pyoracle

    if not pyoracle.available("port"):
        pyoracle.build()
    return pyoracle.Oracle("ref" if pyoracle.available("ref") else "port")


@pytest.fixture(scope="session")
def port_oracle():
    from oracle import pyoracle

    if not pyoracle.available("port"):
        pyoracle.build()
    return pyoracle.Oracle("port")
