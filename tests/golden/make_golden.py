"""Generate tests/golden/grid_cases.json from the reference's own grid planner.

Runs the unmodified src/partition.c + src/utils.c of the reference, compiled
by oracle/build_oracle.py into oracle/_ref/libref_partition.so, over a seeded
set of (p, m, n, k) cases and records its decisions.  The product's planner
must reproduce every one (tests/test_partition.py).

    python tests/golden/make_golden.py
"""
import ctypes as C
import json
import os
import random

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def ref_lib():
    path = os.path.join(ROOT, "oracle", "_ref", "libref_partition.so")
    L = C.CDLL(path)
    ip = C.POINTER(C.c_int)
    L.calc_3d_decomposition_cannon.argtypes = [C.c_int] * 4 + [ip] * 4
    L.calc_3d_decomposition_nk.argtypes = [C.c_int] * 3 + [ip] * 3
    L.calc_block_spos_size.argtypes = [C.c_int] * 3 + [ip] * 2
    return L


def cases(seed=20221111, n=3000):
    rnd = random.Random(seed)
    out = [(24, 8000, 8000, 8000), (4, 2048, 2048, 2048), (1, 1, 1, 1), (16, 50000, 50000, 50000),
           (32, 512, 512, 1 << 20), (2048, 6000, 6000, 1200000), (3072, 100000, 100000, 5000)]
    for _ in range(n):
        p = rnd.choice([1, 2, 3, 4, 6, 8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256, 1000, 3072])
        dims = [int(round(2 ** rnd.uniform(0, 20))) for _ in range(3)]
        out.append((p, dims[0], dims[1], dims[2]))
    return out


def main():
    L = ref_lib()
    rec = {"source": "reference src/partition.c + src/utils.c, compiled unmodified",
           "cannon": [], "nk": [], "split": []}
    for p, m, n, k in cases():
        o = [C.c_int() for _ in range(4)]
        L.calc_3d_decomposition_cannon(p, m, n, k, *[C.byref(x) for x in o])
        rec["cannon"].append([p, m, n, k] + [x.value for x in o])
        o3 = [C.c_int() for _ in range(3)]
        L.calc_3d_decomposition_nk(p, n, k, *[C.byref(x) for x in o3])
        rec["nk"].append([p, n, k] + [x.value for x in o3])
    rnd = random.Random(7)
    for _ in range(500):
        ln, nb = rnd.randint(0, 100000), rnd.randint(1, 64)
        ib = rnd.randint(0, nb)
        s, z = C.c_int(), C.c_int()
        L.calc_block_spos_size(ln, nb, ib, C.byref(s), C.byref(z))
        rec["split"].append([ln, nb, ib, s.value, z.value])
    with open(os.path.join(HERE, "grid_cases.json"), "w") as f:
        json.dump(rec, f, separators=(",", ":"))


if __name__ == "__main__":
    main()
