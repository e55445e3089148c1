"""CPU pins of the post-processing oracle (pdbgen's pose reconstruction,
pdbgen.cpp:166-215; DRMS, drms.cpp:7-57 and main.cpp:789-836) against
independent numpy restatements, and of the pdbgen file readers."""
import math
import os

import numpy as np

from remcdockingsimulator_b200 import post
from remcdockingsimulator_b200.model import rotate_vectors


def _np_drms(sim, ref, ms, reverse):
    sim = sim.astype(np.float32)
    ref = ref.astype(np.float32)

    def dist(a, b):
        d = (a[:, None, :] - b[None, :, :]).astype(np.float32)
        return np.sqrt((d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]) + d[..., 2] * d[..., 2])

    tot, tot2, N = 0.0, 0.0, 0
    n = len(ms) - 1
    for I in range(n):
        for J in range(I + 1, n):
            a, b = slice(ms[I], ms[I + 1]), slice(ms[J], ms[J + 1])
            ds = dist(sim[a], sim[b])
            tot += np.abs(ds - dist(ref[a], ref[b])).astype(np.float64).sum()
            N += ds.size
            if reverse:
                ra, rb = ref[ms[J]:ms[J] + (ms[I + 1] - ms[I])], ref[ms[I]:ms[I] + (ms[J + 1] - ms[J])]
                tot2 += np.abs(ds - dist(ra, rb)).astype(np.float64).sum()
    d = tot / N
    return min(d, tot2 / N) if reverse else d


def test_oracle_drms_matches_numpy(oracle_built):
    from oracle import bindings as ob
    rng = np.random.default_rng(4)
    ms = np.array([0, 12, 24, 36], np.int32)
    ref = rng.normal(scale=8.0, size=(36, 3)).astype(np.float32)
    sim = (ref + rng.normal(scale=2.0, size=ref.shape)).astype(np.float32)
    for reverse in (False, True):
        d, cnt = ob.post_drms(sim, ref, ms, reverse, 12.0, 15.0)
        assert abs(d - _np_drms(sim, ref, ms, reverse)) <= 1e-12 * abs(d)
    # identical frames: zero; counts as defined
    d0, c0 = ob.post_drms(ref, ref, ms)
    assert d0 == 0.0 and c0[0] == c0[2] and c0[1] == c0[0]


def _np_rebuild(rel0, ms, shift, c0, box, quat, centre):
    def norm(q):
        m = math.sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3])
        return [v / m for v in q]

    def img(c, p):
        out = []
        for k in range(3):
            v = np.float32(np.float32(c[k]) - np.float32(p[k]))
            x = float(np.float32(v / np.float32(box)))
            r = math.copysign(math.floor(abs(x) + 0.5), x)  # roundf: half away from zero
            out.append(np.float32(np.float32(c[k]) - np.float32(np.float32(box) * np.float32(r))))
        return np.array(out, np.float32)

    p0 = np.array(centre[0], np.float32)
    if shift[0]:
        p0 = img(p0, c0)
    pos = np.zeros((ms[-1], 3), np.float32)
    for m in range(len(ms) - 1):
        q = norm(norm(list(quat[m])))
        c = p0 if m == 0 else (img(centre[m], p0) if shift[m] else np.array(centre[m], np.float32))
        r = rotate_vectors(q[0], q[1], q[2], q[3], rel0[ms[m]:ms[m + 1]])
        pos[ms[m]:ms[m + 1]] = (r + c[None, :]).astype(np.float32)
    return pos


def test_oracle_rebuild_matches_numpy(oracle_built):
    from oracle import bindings as ob
    rng = np.random.default_rng(9)
    ms = np.array([0, 7, 13, 14, 15], np.int32)
    rel0 = rng.normal(scale=5.0, size=(15, 3)).astype(np.float32)
    shift = np.array([1, 1, 0, 1], np.int32)
    c0 = np.array([50.0, 40.0, 60.0], np.float32)
    box = 100.0
    for _ in range(5):
        quat = rng.normal(size=(4, 4))
        centre = rng.uniform(-120, 220, size=(4, 3)).astype(np.float32)
        got = ob.post_rebuild(rel0, ms, shift, c0, box, quat, centre)
        assert np.array_equal(got, _np_rebuild(rel0, ms, shift, c0, box, quat, centre))


def test_readers(tmp_path):
    idx = tmp_path / "run_repulsive_7_fileindex"
    idx.write_text("index molecule_file_path crowder(Y/N)\n 0 a.pdb N\n 1 b.pdb N\n 2 c.pdb Y\n")
    assert post.read_index(str(idx)) == [("a.pdb", False), ("b.pdb", False), ("c.pdb", True)]
    bc = tmp_path / "run_repulsive_7_boundconformations"
    bc.write_text("# iteration; complex free energy (replica free energy); temperature;\n"
                  "# molecule: rotation(w,x,y,z) position(x,y,z) 1 line per other molecule\n"
                  "500; -3.25000 (-1.50000); 300.0\n"
                  "0  0: 1.000000 0.000000 0.000000 0.000000 1.000000 2.000000 3.000000\n"
                  "0  1: 0.500000 0.500000 0.500000 0.500000 4.000000 5.000000 6.000000\n"
                  "1  2: 1.000000 0.000000 0.000000 0.000000 7.000000 8.000000 9.000000\n")
    s = post.read_bound_conformations(str(bc))
    assert len(s) == 1 and s[0][:4] == (500, -3.25, -1.5, 300.0) and len(s[0][4]) == 3
    assert s[0][4][1] == (0, 1, 0.5, 0.5, 0.5, 0.5, 4.0, 5.0, 6.0)
