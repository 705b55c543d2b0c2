"""The kernels' own per-item logic, compiled for the host, against the oracle
(no GPU).  fdp_item.cuh and fdp_core.cuh are host+device code: the same source
the sm_100a cell and growth kernels run is built here with g++ and checked on
every cell of small widths, in every visiting order the kernel may use.  The
row-k initialiser's automaton and fill plan (fdp_rowinit.cpp) are checked the
same way against the oracle's state after the first rows."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "oneesan-gpu_b200", "csrc")
CUDA_INC = "/usr/local/cuda/include"


@pytest.mark.skipif(shutil.which("g++") is None or shutil.which("gcc") is None, reason="needs gcc/g++")
@pytest.mark.skipif(not os.path.exists(os.path.join(CUDA_INC, "cuda_runtime.h")), reason="needs CUDA headers")
def test_kernel_item_logic_matches_oracle(tmp_path):
    oracle_o = tmp_path / "fdp_oracle.o"
    subprocess.run(["gcc", "-O2", "-c", os.path.join(ROOT, "oracle", "fdp_oracle.c"), "-o", str(oracle_o)],
                   check=True)
    exe = tmp_path / "kernel_logic_check"
    subprocess.run(["g++", "-O2", "-std=c++17", f"-I{CSRC}", f"-I{CUDA_INC}",
                    os.path.join(ROOT, "tests", "host", "kernel_logic_check.cpp"),
                    os.path.join(CSRC, "fdp_host.cpp"), str(oracle_o), "-o", str(exe), "-lpthread"], check=True)
    out = subprocess.run([str(exe), "11", "10"], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip().endswith("bad=0"), out.stdout


@pytest.mark.skipif(shutil.which("g++") is None or shutil.which("gcc") is None, reason="needs gcc/g++")
@pytest.mark.skipif(not os.path.exists(os.path.join(CUDA_INC, "cuda_runtime.h")), reason="needs CUDA headers")
def test_row_automaton_and_fill_match_oracle(tmp_path):
    oracle_o = tmp_path / "fdp_oracle.o"
    subprocess.run(["gcc", "-O2", "-c", os.path.join(ROOT, "oracle", "fdp_oracle.c"), "-o", str(oracle_o)],
                   check=True)
    exe = tmp_path / "row_automaton_check"
    subprocess.run(["g++", "-O2", "-std=c++17", f"-I{CSRC}", f"-I{CUDA_INC}",
                    os.path.join(ROOT, "tests", "host", "row_automaton_check.cpp"),
                    os.path.join(CSRC, "fdp_rowinit.cpp"), os.path.join(CSRC, "fdp_host.cpp"), str(oracle_o),
                    "-o", str(exe), "-lpthread"], check=True)
    out = subprocess.run([str(exe), "10"], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip().endswith("bad=0"), out.stdout
