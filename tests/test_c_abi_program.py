"""A plain C program (tests/c_abi_smoke.c) built against include/ffs_lbm.h and
libffs_lbm.so alone: the header compiles as C11 with warnings on, the program
links (CPU), and on a B200 it steps a D2Q9 channel with a cylinder through the
C ABI without Python or torch in the process (GPU)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "freeflow_b200")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def _build(tmp_path):
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    if not os.path.exists(os.path.join(LIBDIR, "libffs_lbm.so")):
        pytest.skip("libffs_lbm.so not built")
    exe = str(tmp_path / "c_abi_smoke")
    cmd = ["gcc", "-std=c11", "-O2", "-Wall", "-Wextra", "-Werror",
           "-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(CUDA, "include"),
           os.path.join(ROOT, "tests", "c_abi_smoke.c"), "-o", exe,
           "-L" + LIBDIR, "-lffs_lbm", "-L" + os.path.join(CUDA, "lib64"), "-lcudart", "-lm",
           "-Wl,-rpath," + LIBDIR]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    return exe


def test_c_program_compiles_and_links(tmp_path):
    _build(tmp_path)


@pytest.mark.gpu
def test_c_program_steps_a_channel(tmp_path, cuda):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "c abi smoke ok" in r.stdout
