"""The restated example drivers (examples/example_AB.c and example_BTB.c of the
reference) on the library: same command line, same output lines, parsed the
way scripts written for the reference's output parse them, and the same
validation rule (0 entries with a relative error above 1e-12 against the
closed form of the deterministic fill)."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EX = os.path.join(ROOT, "ca3dmm_b200", "examples")


def run(exe, *args, env=None):
    r = subprocess.run([os.path.join(EX, exe)] + [str(a) for a in args], capture_output=True,
                       text=True, timeout=600, env=dict(os.environ, **(env or {})))
    return r.returncode, r.stdout + r.stderr


def parse(out):
    """The fields a reference output parser reads."""
    f = {}
    m = re.search(r"Test problem size m \* n \* k : (\d+) \* (\d+) \* (\d+)", out)
    f["mnk"] = tuple(int(x) for x in m.groups()) if m else None
    m = re.search(r"Process grid mp \* np \* kp  : (\d+) \* (\d+) \* (\d+)", out)
    f["grid"] = tuple(int(x) for x in m.groups()) if m else None
    m = re.search(r"Work cuboid  mb \* nb \* kb  : (\d+) \* (\d+) \* (\d+)", out)
    f["cuboid"] = tuple(int(x) for x in m.groups()) if m else None
    m = re.search(r"Process utilization        : ([0-9.]+) %", out)
    f["util"] = float(m.group(1)) if m else None
    for key, label in (("redist", "A, B, C redist   "), ("cannon", "2D Cannon        "),
                       ("matmul", "matmul only      "), ("total", "total execution  ")):
        m = re.search(re.escape(label) + r": ([0-9 ]+)\n", out)
        f[key] = [int(x) for x in m.group(1).split()] if m else None
    m = re.search(r"CA3DMM output : (\d+) error\(s\)", out)
    f["errors"] = int(m.group(1)) if m else None
    return f


def test_help_without_gpu():
    for exe in ("example_ab", "example_btb"):
        rc, out = run(exe, "--help")
        assert rc == 0 and out.startswith("Usage:"), out


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["0", "1", "2", "auto"])
def test_example_ab_2048_on_four_ranks(cuda, mode):
    """The 2048^3 example on 4 virtual ranks: the reference's grid 2 x 1 x 2,
    cuboid 1024 x 2048 x 1024, and 0 errors in every GEMM mode (auto: tuned at
    the warm-up exec)."""
    rc, out = run("example_ab", 2048, 2048, 2048, 0, 0, 1, 3, 1,
                  env={"CA3DMM_VRANKS": "4", "CA3DMM_GEMM_MODE": mode})
    assert rc == 0, out
    f = parse(out)
    assert f["mnk"] == (2048, 2048, 2048)
    assert f["grid"] == (2, 1, 2) and f["cuboid"] == (1024, 2048, 1024)
    assert f["util"] == 100.0
    assert len(f["total"]) == 3 and len(f["matmul"]) == 3
    assert f["errors"] == 0


@pytest.mark.gpu
@pytest.mark.parametrize("ta,tb", [(1, 0), (0, 1), (1, 1)])
def test_example_ab_given_grid_and_transposes(cuda, ta, tb):
    """A given 4 x 2 x 3 grid (the README's 24-rank run) at 1200 x 1000 x 900."""
    rc, out = run("example_ab", 1200, 1000, 900, ta, tb, 1, 2, 1, 4, 2, 3,
                  env={"CA3DMM_GEMM_MODE": "2"})
    assert rc == 0, out
    f = parse(out)
    assert f["grid"] == (4, 2, 3) and f["errors"] == 0


@pytest.mark.gpu
def test_example_btb(cuda):
    rc, out = run("example_btb", 512, 40000, 1, 2, 1, env={"CA3DMM_VRANKS": "8"})
    assert rc == 0, out
    f = parse(out)
    assert f["mnk"] == (512, 512, 40000)
    assert f["grid"] is not None and f["errors"] == 0
    for mode in ("1", "2"):
        rc, out = run("example_btb", 512, 40000, 1, 2, 1,
                      env={"CA3DMM_VRANKS": "8", "CA3DMM_GEMM_MODE": mode})
        assert rc == 0 and parse(out)["errors"] == 0, out


@pytest.mark.gpu
def test_select_device_by_local_rank(cuda, monkeypatch):
    """select_cuda_device_by_mpi_local_rank (include/cuda_proxy.h), which the
    drivers call first: device (local rank mod device count) becomes current."""
    import ctypes
    import torch
    import ca3dmm_b200 as cb
    L = ctypes.CDLL(cb.LIB_PATH)
    ndev = torch.cuda.device_count()
    for n in ("MPI_LOCALRANKID", "MV2_COMM_WORLD_LOCAL_RANK", "SLURM_LOCALID", "PBS_O_VNODENUM"):
        monkeypatch.delenv(n, raising=False)
    for rank in (ndev, 2 * ndev - 1):
        monkeypatch.setenv("OMPI_COMM_WORLD_NODE_RANK", str(rank))
        L.select_cuda_device_by_mpi_local_rank()
        assert torch.cuda.current_device() == rank % ndev
    torch.cuda.set_device(0)
