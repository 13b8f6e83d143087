"""The C-ABI library loads and exports every function include/*.h declares."""
import ctypes
import os
import re

import ca3dmm_b200 as cb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if not f.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", f)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"#define[^\n]*(\\\n[^\n]*)*", "", text)
        for m in re.finditer(r"^\s*[A-Za-z_][\w\s\*]*?\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text, flags=re.M):
            name = m.group(1)
            if name not in ("if", "while", "for", "sizeof", "return"):
                names.add(name)
    return sorted(names)


def test_headers_declare_the_reference_api():
    names = set(declared_functions())
    for n in ("ca3dmm_engine_init", "ca3dmm_engine_init_BTB", "ca3dmm_engine_attach_workbuf",
              "ca3dmm_engine_free", "ca3dmm_engine_exec", "ca3dmm_engine_reset_stat",
              "ca3dmm_engine_print_stat", "cannon_engine_init", "cannon_engine_exec",
              "calc_3d_decomposition_cannon", "calc_3d_decomposition_nk",
              "mat_redist_engine_init", "mat_redist_engine_exec", "dev_type_malloc"):
        assert n in names, n


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(cb.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_static_archive_defines_every_symbol_and_links():
    """libca3dmm_b200.a (installed beside the .so, as the reference installs
    libca3dmm.a and .so) defines every declared function, and a C caller links
    statically against it and runs a host-only entry point."""
    import subprocess
    from ca3dmm_b200 import build
    arc = build.ARCHIVE
    assert os.path.exists(arc)
    nm = subprocess.run(["nm", "--defined-only", arc], capture_output=True, text=True).stdout
    defined = {ln.split()[-1] for ln in nm.splitlines() if " T " in ln}
    missing = [n for n in declared_functions() if n not in defined]
    assert not missing, missing
    src = os.path.join(build.OBJ, "static_caller.c")
    exe = os.path.join(build.OBJ, "static_caller")
    with open(src, "w") as f:
        f.write('#include "ca3dmm.h"\n'
                "int main(void) { int mp, np, kp, rp;\n"
                "  calc_3d_decomposition_cannon(24, 8000, 8000, 8000, &mp, &np, &kp, &rp);\n"
                "  return (mp == 4 && np == 2 && kp == 3 && rp == 0) ? 0 : 1; }\n")
    cuda_lib = os.path.join(build.CUDA, "lib64")
    r = subprocess.run(["gcc", "-O2", "-I", os.path.join(ROOT, "include"), src, arc, "-L", cuda_lib,
                        "-lcudart_static", "-lstdc++", "-ldl", "-lpthread", "-lrt", "-lm", "-o", exe],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    assert subprocess.run([exe]).returncode == 0


def test_local_rank_env_precedence(monkeypatch):
    """select_cuda_device_by_mpi_local_rank's local rank: the first set of the
    launchers' variables, in the reference's order (src/cuda_proxy.cu), -1 when
    none is set, 0 for a value that is not a non-negative number."""
    L = ctypes.CDLL(cb.LIB_PATH)
    names = ["MPI_LOCALRANKID", "MV2_COMM_WORLD_LOCAL_RANK", "OMPI_COMM_WORLD_NODE_RANK",
             "SLURM_LOCALID", "PBS_O_VNODENUM"]
    for n in names:
        monkeypatch.delenv(n, raising=False)
    assert L.ca3dmm_mpi_local_rank_env() == -1
    monkeypatch.setenv("PBS_O_VNODENUM", "9")
    assert L.ca3dmm_mpi_local_rank_env() == 9
    monkeypatch.setenv("SLURM_LOCALID", "5")
    assert L.ca3dmm_mpi_local_rank_env() == 5
    monkeypatch.setenv("OMPI_COMM_WORLD_NODE_RANK", "3")
    assert L.ca3dmm_mpi_local_rank_env() == 3
    monkeypatch.setenv("MV2_COMM_WORLD_LOCAL_RANK", "2")
    assert L.ca3dmm_mpi_local_rank_env() == 2
    monkeypatch.setenv("MPI_LOCALRANKID", "x")
    assert L.ca3dmm_mpi_local_rank_env() == 0
