"""One engine per host thread: engines are independent (the library's only
shared state is its lazily initialised device-property cache, function
attributes and launch counter), so engines of different shapes and modes
executing at the same time from several host threads, each on its own
stream, give the results each gives alone, bit for bit."""
import threading

import numpy as np
import pytest

import ca3dmm_b200 as cb
from oracle import oracle as orc
from tests._util import dev_zeros, to_dev

pytestmark = pytest.mark.gpu

SHAPES = [(700, 500, 900, 0, 0, 6, cb.GEMM_OZAKI), (512, 640, 384, 1, 0, 4, cb.GEMM_PLAIN),
          (300, 300, 2000, 0, 1, 8, cb.GEMM_OZAKI), (1024, 256, 512, 1, 1, 2, cb.GEMM_PLAIN),
          (257, 129, 1111, 0, 0, 3, cb.GEMM_OZAKI), (640, 640, 640, 0, 0, 24, cb.GEMM_PLAIN)]


def test_engines_on_concurrent_host_threads(cuda):
    import torch
    jobs = []
    for i, (m, n, k, ta, tb, p, mode) in enumerate(SHAPES):
        A = orc.gen_signed_exp(700 + i, *((k, m) if ta else (m, k)))
        B = orc.gen_signed_exp(800 + i, *((n, k) if tb else (k, n)))
        dA, lda = to_dev(A)
        dB, ldb = to_dev(B)
        e = cb.Ca3dmmEngine(m, n, k, ta, tb, p=p)
        assert e.ok
        if mode == cb.GEMM_OZAKI:
            assert e.set_gemm_mode(mode, 7) == 0
        alone = dev_zeros(m * n)
        assert e.exec(dA, lda, dB, ldb, alone, m) == 0
        torch.cuda.synchronize()
        jobs.append((e, dA, lda, dB, ldb, m, n, alone))
    errors = []
    outs = [dev_zeros(j[5] * j[6]) for j in jobs]
    barrier = threading.Barrier(len(jobs))

    def run(i):
        e, dA, lda, dB, ldb, m, n, _ = jobs[i]
        s = torch.cuda.Stream()
        e.set_stream(s.cuda_stream, 1)
        barrier.wait()
        for _ in range(5):
            rc = e.exec(dA, lda, dB, ldb, outs[i], m)
            if rc:
                errors.append((i, rc))

    threads = [threading.Thread(target=run, args=(i,)) for i in range(len(jobs))]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=120)
    torch.cuda.synchronize()
    assert not errors, errors
    for i, j in enumerate(jobs):
        assert torch.equal(outs[i], j[7]), i
        j[0].free()
