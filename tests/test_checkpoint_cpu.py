"""Checkpoint text layout (saveSimulation, main.cpp:89-117) and exact-state
round trip, on CPU."""
import os

import numpy as np

from remcdockingsimulator_b200 import remc


def test_checkpoint_layout_and_round_trip(tmp_path):
    a = remc.Args(file="cfg/run.conf", prefix="demo", pid=4321, mcsteps=1000, resteps=10,
                  replicas=3, noncrowders=2)
    R, n_mol, n_b = 3, 4, 7
    rng = np.random.default_rng(1)
    state = (rng.normal(size=(R * n_b, 3)).astype(np.float32),
             rng.normal(size=(R * n_b, 3)).astype(np.float32),
             rng.normal(size=(R * n_mol, 3)).astype(np.float32),
             rng.normal(size=(R * n_mol, 4)))
    acc = {k: np.arange(R, dtype=np.int64) + i for i, k in enumerate(remc._CK_ARRAYS)}
    acc["sens"] = rng.normal(size=(R, 4))
    E, ecc, tmap = rng.normal(size=R), rng.normal(size=R), np.array([2, 0, 1], np.int32)
    path = str(tmp_path / "ck" / "demo_4321")
    remc.save_simulation(a, path, 3, 98765, state, E, ecc, tmap, acc, 5, 9)
    lines = open(path).read().splitlines()
    assert lines[0] == "#Saved simulation state file, prependage string, original pid"
    assert lines[1:4] == ["cfg/run.conf", "demo_4321", "4321"]
    assert lines[5].split()[-1] == "300"           # currentStep = 3 blocks x 100 steps
    assert lines[6:10] == ["#molecules", "4", "#replicas", "3"]
    assert lines[10].startswith("#replica 0, molecules:")
    assert len(lines[11].split()) == 7 and lines[15].startswith("#replica 0, stats")
    assert len(lines[16].split()) == 9
    ck = remc.load_simulation(path)
    assert ck["pid"] == 4321 and ck["file"] == "cfg/run.conf" and int(ck["blocks"]) == 3
    assert int(ck["seed"]) == 98765 and int(ck["total_tests"]) == 9
    for k, v in zip(("pos", "rel", "centre", "quat"), state):
        assert np.array_equal(ck[k], v) and ck[k].dtype == v.dtype
    assert np.array_equal(ck["energies"], E) and np.array_equal(ck["tmap"], tmap)
    for k in remc._CK_ARRAYS:
        assert np.array_equal(ck[k], acc[k])


def test_resume_flag_reads_config_and_pid(tmp_path):
    a = remc.parse_cli(["-z", "x/ck", "--checkpoint-every", "500"])
    assert a.resume == "x/ck" and a.checkpoint_every == 500


def test_autotune_flag():
    assert remc.parse_cli(["--autotune"]).autotune is True
    assert remc.parse_cli([]).autotune is False
