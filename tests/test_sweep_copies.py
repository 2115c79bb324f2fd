"""The bulk copies of the MILU sweeps (sweep_lane in csrc/kernels.h, host
and device code alike), checked on the CPU: a host-only harness
(tests/native/sweep_copies.cu) walks every tile, mode, step and copy of a
set of grids and tile shapes and checks bounds, 16-byte alignment, that the
copies of a step do not overlap, and that every ring entry a column reads
at a step was copied for it.  The checks are the ones the kernel relies on
(a bulk copy that starts off a 16-byte boundary faults)."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
CSRC = ROOT / "multiscale-and-multiphysics-integrated-simulator-for-tsunami_b200" / "csrc"


def test_sweep_copies_bounds_alignment_and_coverage(tmp_path):
    nvcc = shutil.which("nvcc") or ("/usr/local/cuda/bin/nvcc" if Path("/usr/local/cuda/bin/nvcc").exists() else None)
    if nvcc is None:
        pytest.skip("nvcc not found")
    exe = tmp_path / "sweep_copies"
    subprocess.run([nvcc, "-std=c++17", "-O1", "-Wno-deprecated-gpu-targets", f"-I{CSRC}", "-o", str(exe),
                    str(ROOT / "tests" / "native" / "sweep_copies.cu")], check=True, capture_output=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:]
    assert " 0 failures" in r.stdout, r.stdout
