"""The C++17 face (include/dyng/dyng.hpp): the reference's C++ quickstart compiles against it and
links to the library (CPU); on a GPU it prints the quickstart's output and maps statuses to the
reference's exception classes.  The same for dyng::mosp (tests/cpp/mosp_quickstart.cpp: the
two-objective case of the reference's mosp_test.cpp:249-269 and one update)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_DIR = os.path.join(ROOT, "dyng_b200")


def _build(tmp_path, name="quickstart"):
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    if not os.path.exists(os.path.join(LIB_DIR, "libdyngb200.so")):
        pytest.skip("library not built")
    exe = str(tmp_path / name)
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror",
           "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", name + ".cpp"),
           "-L", LIB_DIR, "-ldyngb200", f"-Wl,-rpath,{LIB_DIR}", "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_quickstart_compiles_and_links(tmp_path):
    exe = _build(tmp_path)
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_quickstart_runs(tmp_path):
    exe = _build(tmp_path)
    out = subprocess.run([exe], check=True, capture_output=True, text=True, timeout=120).stdout
    assert out.splitlines() == ["0 4 1 2 | invalidated 2", "stale_result_error",
                                "not_supported_error"]


def test_mosp_program_compiles_and_links(tmp_path):
    assert os.path.exists(_build(tmp_path, "mosp_quickstart"))


@pytest.mark.gpu
def test_mosp_program_runs(tmp_path):
    exe = _build(tmp_path, "mosp_quickstart")
    out = subprocess.run([exe], check=True, capture_output=True, text=True, timeout=120).stdout
    assert out.splitlines() == ["0 1 1 3 | -1 0 0 1 | 2 10 | L 1",
                                "0 3 3 7 | -1 0 0 2 | 10 2 | L 2",
                                "0 1 1 2 | -1 0 0 2 | 10 2 | L 1",
                                "affected 1 objectives 2"]
