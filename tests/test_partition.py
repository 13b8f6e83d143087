"""Grid planner parity with the reference's own src/partition.c (CPU)."""
import ctypes as C
import json
import os
import random

import pytest

import ca3dmm_b200 as cb

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GOLD = json.load(open(os.path.join(HERE, "golden", "grid_cases.json")))


def test_cannon_grid_matches_reference_golden():
    bad = [c for c in GOLD["cannon"] if list(cb.calc_3d_decomposition_cannon(*c[:4])) != c[4:]]
    assert not bad, bad[:5]


def test_nk_grid_matches_reference_golden():
    bad = [c for c in GOLD["nk"] if list(cb.calc_3d_decomposition_nk(*c[:3])) != c[3:]]
    assert not bad, bad[:5]


def test_block_split_matches_reference_golden():
    bad = [c for c in GOLD["split"] if list(cb.calc_block_spos_size(*c[:3])) != c[3:]]
    assert not bad, bad[:5]


def test_readme_configuration():
    # README.md:66-67: 8000^3 on 24 ranks -> 4 x 2 x 3, cuboid 2000 x 4000 x 2667
    assert cb.calc_3d_decomposition_cannon(24, 8000, 8000, 8000) == (4, 2, 3, 0)
    assert cb.calc_3d_decomposition_cannon(4, 2048, 2048, 2048) == (2, 1, 2, 0)
    assert cb.calc_3d_decomposition_nk(32, 512, 1 << 20) == (1, 32, 0)


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref_partition.so")),
                    reason="reference planner not compiled here")
def test_random_cases_against_compiled_reference():
    L = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_partition.so"))
    ip = C.POINTER(C.c_int)
    L.calc_3d_decomposition_cannon.argtypes = [C.c_int] * 4 + [ip] * 4
    rnd = random.Random(99)
    for _ in range(3000):
        p = rnd.randint(1, 4096)
        m, n, k = (int(round(2 ** rnd.uniform(0, 22))) for _ in range(3))
        o = [C.c_int() for _ in range(4)]
        L.calc_3d_decomposition_cannon(p, m, n, k, *[C.byref(x) for x in o])
        assert cb.calc_3d_decomposition_cannon(p, m, n, k) == tuple(x.value for x in o), (p, m, n, k)
