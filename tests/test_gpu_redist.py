"""Folded redistribution between arbitrary layouts (mat_redist_layouts_*): all
ranks' source and required rectangles in one call, one batched device copy.
Checked bit for bit against the reference's own mat_redist run on vmpi rank
threads over the same layouts (where the reference's one-rectangle-per-rank
form applies) and against direct slicing of the global matrix."""
import numpy as np
import pytest

import ca3dmm_b200 as cb
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _grid_rects(R, Cc, pr, pc):
    rs = [R * i // pr for i in range(pr + 1)]
    cs = [Cc * j // pc for j in range(pc + 1)]
    return [(rs[i], cs[j], rs[i + 1] - rs[i], cs[j + 1] - cs[j]) for i in range(pr) for j in range(pc)]


def _run(G, src, req, pad=0, stream=None):
    """Source blocks cut from G (row-major, ld = ncol + pad), required blocks
    returned as row-major arrays."""
    import torch
    srcs, slds, dsts, dlds = [], [], [], []
    for r in src:
        ld = r[3] + pad
        buf = np.zeros((max(r[2], 1), max(ld, 1)))
        buf[:r[2], :r[3]] = G[r[0]:r[0] + r[2], r[1]:r[1] + r[3]]
        srcs.append(torch.from_numpy(buf.ravel()).cuda())
        slds.append(max(ld, 1))
    for r in req:
        ld = r[3] + pad
        dsts.append(torch.full((max(r[2], 1) * max(ld, 1),), -7.0, dtype=torch.float64,
                               device="cuda"))
        dlds.append(max(ld, 1))
    L = cb.RedistLayouts(src, req)
    assert L.ok
    s = None
    if stream is not None:
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())      # the uploads above
        with torch.cuda.stream(s):
            assert L.exec(srcs, slds, dsts, dlds, s.cuda_stream) == 0
        s.synchronize()
    else:
        assert L.exec(srcs, slds, dsts, dlds) == 0
    out = []
    for r, d, ld in zip(req, dsts, dlds):
        out.append(d.cpu().numpy().reshape(max(r[2], 1), ld)[:r[2], :r[3]])
    return out, L.pieces()


@pytest.mark.parametrize("R,Cc,src,req", [
    (37, 53, (2, 3), (3, 2)),
    (300, 257, (1, 6), (6, 1)),      # 1D column blocks (the example drivers' layout) -> row blocks
    (1000, 800, (4, 1), (2, 2)),
    (129, 64, (3, 3), (3, 3)),
])
def test_layouts_match_reference_mat_redist(cuda, R, Cc, src, req):
    G = orc.gen_uniform(31, R, Cc)
    sr, rr = _grid_rects(R, Cc, *src), _grid_rects(R, Cc, *req)
    got, _ = _run(G, sr, rr)
    want = orc.ref_redist(sr, rr, G) if orc.ref_lib() is not None else None
    for j, r in enumerate(rr):
        assert np.array_equal(got[j], G[r[0]:r[0] + r[2], r[1]:r[1] + r[3]]), j
        if want is not None:
            assert np.array_equal(got[j], want[j]), j


def test_replicated_and_partial_requirements(cuda):
    """Required blocks may overlap each other (replication, as the engine's
    allgather does) and may reach outside every source block (those elements
    stay untouched); more required blocks than source blocks; padded leading
    dimensions; an empty rectangle; a launch on a stream."""
    R, Cc = 400, 300
    G = orc.gen_uniform(32, R, Cc)
    src = _grid_rects(R, Cc, 2, 2)
    req = [(0, 0, R, 100), (50, 50, 200, 200), (0, 0, R, 100), (390, 290, 20, 20), (10, 10, 0, 5)]
    got, pieces = _run(G, src, req, pad=3, stream=True)
    assert pieces == 2 + 4 + 2 + 1                  # per required block; the empty one has none
    for j, r in enumerate(req[:3]):
        assert np.array_equal(got[j], G[r[0]:r[0] + r[2], r[1]:r[1] + r[3]]), j
    tail = got[3]                                   # rows 390..409, columns 290..309
    assert np.array_equal(tail[:10, :10], G[390:400, 290:300])
    assert np.all(tail[10:, :] == -7.0) and np.all(tail[:, 10:] == -7.0)


def test_layouts_rejects_bad_arguments(cuda):
    import torch
    L = cb.RedistLayouts([(0, 0, 4, 4)], [(0, 0, 4, 4)])
    assert L.ok
    a = torch.zeros(16, dtype=torch.float64, device="cuda")
    b = torch.zeros(16, dtype=torch.float64, device="cuda")
    assert L.exec([a], [3], [b], [4]) == cb.EINVAL          # ld below the block's width
    assert not cb.RedistLayouts([(0, 0, -1, 4)], [(0, 0, 4, 4)]).ok
