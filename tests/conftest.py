import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "structures.json")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def golden():
    with open(GOLDEN) as fh:
        return json.load(fh)


@pytest.fixture(scope="session")
def golden_table(golden):
    from remcdockingsimulator_b200.model import AminoAcidTable
    t = golden["table"]
    table = AminoAcidTable(t["names"], t["snames"], t["symbols"], np.array(t["vdw"], np.float32),
                           np.array(t["charge"], np.float32), np.array(t["pairs"], np.float32))
    return table


def golden_system(golden, table, k):
    from remcdockingsimulator_b200.model import Molecule, System
    st = golden["structures"][k]
    mols = [Molecule.from_beads(c["types"], np.array(c["pos"], np.float32)) for c in st["chains"]]
    return System(mols, golden["box"], table)


@pytest.fixture(scope="session")
def built_lib():
    from remcdockingsimulator_b200 import build
    return build.build()


@pytest.fixture(scope="session")
def oracle_built():
    from oracle import build
    build.build_oracle()
    return True
