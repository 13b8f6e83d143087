"""Cost-model features of the autotuner's configurations (host code, no GPU):
the tile shape each GEMM kernel really computes, the modulus count the
engine resolves, and the tile count of one slab."""
import math

import ca3dmm_b200 as cb


def feats(m, n, k, cfg, spread=3.0, ta=0, tb=1):
    return [float(x) for x in cb.tune_features(m, n, k, ta, tb, cfg, spread)]


def test_feature_layout():
    assert cb.NFEAT == 14
    f = feats(1000, 3000, 8000, (0, 0, 2, 16, 0))
    want = [math.log2(1000), math.log2(3000), math.log2(8000), 0.0, 1.0]
    assert all(abs(a - b) < 1e-5 for a, b in zip(f[:5], want))
    assert f[5:9] == [0.0, 0.0, 0.0, 1.0]
    assert f[9] == 4.0 and f[10:12] == [128.0, 128.0]
    assert abs(f[12] - math.log2(8 * 24)) < 1e-6
    assert f[13] == 3.0


def test_tile_shapes_and_counts():
    oz = feats(1000, 3000, 8000, (1, 7, 1, 8, 0))
    assert oz[5:8] == [1.0, 0.0, 7.0] and oz[10:12] == [128.0, 64.0]
    assert abs(oz[12] - math.log2(8 * 47)) < 1e-6
    wide = feats(1000, 3000, 8000, (2, 0, 1, 32, 256))
    narrow = feats(1000, 3000, 8000, (2, 0, 1, 8, 128))
    assert wide[5:7] == [0.0, 1.0] and wide[11] == 256.0 and narrow[11] == 128.0
    assert wide[9] == 5.0 and narrow[9] == 3.0
    assert abs(wide[12] - math.log2(8 * 12)) < 1e-6 and abs(narrow[12] - math.log2(8 * 24)) < 1e-6
    # 0 moduli: the engine's automatic count (fewest with 51-bit integers)
    auto = wide[7]
    assert 8 <= auto <= 18
    L = cb.lib()
    assert L.ca3dmm_crt_bits(int(auto), 8000) >= 51 and L.ca3dmm_crt_bits(int(auto) - 1, 8000) < 51
    assert feats(1000, 3000, 8000, (2, 17, 1, 32, 256))[7] == 17.0


def test_plain_tile_widths():
    """The plain DMMA GEMM's two tiles: 128 x 128 (tile_n 0 or 128) and 128 x 64."""
    full = feats(1000, 3000, 8000, (0, 0, 1, 8, 0))
    half = feats(1000, 3000, 8000, (0, 0, 1, 8, 64))
    assert full[10:12] == [128.0, 128.0] and half[10:12] == [128.0, 64.0]
    assert abs(full[12] - math.log2(8 * 24)) < 1e-6 and abs(half[12] - math.log2(8 * 47)) < 1e-6
