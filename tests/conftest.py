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


def crowder_lattice(n, spacing=8.0, seed=5, side=None):
    """n one-bead crowders on a jittered cubic lattice of `side` sites per
    edge (spacing 8 A, inside the 15 A cutoff of the reference's (6/r)^6
    crowder term), in a box of side * spacing."""
    from remcdockingsimulator_b200 import synth
    from remcdockingsimulator_b200.model import CROWDER_TYPE, Molecule, System
    rng = np.random.default_rng(seed)
    side = side or int(np.ceil(n ** (1.0 / 3.0)))
    assert side ** 3 >= n
    box = side * spacing
    g = np.stack(np.meshgrid(np.arange(side), np.arange(side), np.arange(side), indexing="ij"),
                 axis=-1).reshape(-1, 3)[:n]
    xyz = g * spacing + 1.0 + rng.uniform(-0.4, 0.4, size=(n, 3))  # inside [0, box)
    mols = []
    for c in xyz:
        m = Molecule.from_beads([CROWDER_TYPE], np.zeros((1, 3), np.float32))
        m.crowder = True
        m.set_position(c.astype(np.float32))
        mols.append(m)
    table = synth.contact_table(np.random.default_rng(seed))
    return System(mols, float(np.float32(box)), table, crowder_radius=3.0)


@pytest.fixture(scope="session")
def built_lib():
    from remcdockingsimulator_b200 import build
    return build.build()


@pytest.fixture(scope="session")
def oracle_built():
    from oracle import build
    build.build_oracle()
    return True
