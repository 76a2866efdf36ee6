"""The persistent kernels' footprint, read from ptxas's resource report (CPU only: nvcc
cross-compiles sm_100a here).

An update is two cooperative launches of occupancy x 148 blocks: the batch applier (k_apply,
graph.cu) and the sssp kernel (k_sssp, sssp.cu).  Both are written for three blocks of 256
threads per SM (444 blocks), and the serving loop's lanes cap their grids at shares of those
three slots (the large lane two per SM, the small lanes one), so any three blocks of the two
kernels must fit one SM together: at most 80 registers a thread (a warp's registers are
allocated in units of 256, so 80 x 256 x 3 = 61,440 of the SM's 65,536) and at most 228 KB of
shared memory for three blocks, counting the 1 KB the hardware reserves per block.
"""
import os
import re
import shutil
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from dyng_b200 import build as B  # noqa: E402

THREADS = 256
BLOCKS_PER_SM = 3
SM_REGISTERS = 65536
SM_SHARED = 228 * 1024
RESERVED_PER_BLOCK = 1024
STATIC_SHARED_LIMIT = 48 * 1024

# mangled names carry the identifier's length before it: "7k_applyE", "6k_ssspE"
KERNELS = {"k_apply": ("graph.cu", re.compile(r"7k_applyE")),
           "k_sssp": ("sssp.cu", re.compile(r"6k_ssspE"))}

ENTRY = re.compile(r"Compiling entry function '([^']+)'")
USED = re.compile(r"Used (\d+) registers.*?(\d+) bytes smem")


def _nvcc():
    return B.NVCC if os.path.exists(B.NVCC) else shutil.which("nvcc")


def _report(text, pattern):
    """(registers, static shared bytes) of the entry function whose name matches `pattern`."""
    current = None
    for line in text.splitlines():
        m = ENTRY.search(line)
        if m:
            current = m.group(1)
            continue
        m = USED.search(line)
        if m and current is not None and pattern.search(current):
            return int(m.group(1)), int(m.group(2))
    raise AssertionError(f"no ptxas report for {pattern.pattern}")


@pytest.fixture(scope="module")
def footprints(tmp_path_factory):
    nvcc = _nvcc()
    if nvcc is None:
        pytest.skip("nvcc not found")
    out = tmp_path_factory.mktemp("ptxas")
    procs = {}
    for name, (src, _) in KERNELS.items():
        cmd = [nvcc, "-c", os.path.join(B.CSRC, src), "-o", str(out / (name + ".o"))]
        cmd += B.flags() + ["-Xptxas", "-v"]
        procs[name] = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    result = {}
    for name, p in procs.items():
        text, _ = p.communicate()
        assert p.returncode == 0, text.decode()[-2000:]
        result[name] = _report(text.decode(), KERNELS[name][1])
    return result


def test_each_persistent_kernel_fits_three_blocks_per_sm(footprints):
    for name, (regs, smem) in footprints.items():
        per_warp = -(-regs * 32 // 256) * 256  # registers are allocated per warp in 256s
        assert per_warp * (THREADS // 32) * BLOCKS_PER_SM <= SM_REGISTERS, (name, regs)
        assert smem <= STATIC_SHARED_LIMIT, (name, smem)
        assert BLOCKS_PER_SM * (smem + RESERVED_PER_BLOCK) <= SM_SHARED, (name, smem)


def test_any_three_blocks_of_the_two_kernels_fit_one_sm(footprints):
    largest = max(smem for _, smem in footprints.values())
    assert BLOCKS_PER_SM * (largest + RESERVED_PER_BLOCK) <= SM_SHARED, footprints
    most = max(regs for regs, _ in footprints.values())
    assert most <= 80, footprints
