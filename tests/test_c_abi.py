"""The C ABI from a plain C program: it compiles against include/ausaxs_b200.h alone and links
against the shared library (CPU), and on a GPU it reproduces the SimpleCube known answer."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "ausaxs_b200", "_lib")


def _build(tmp_path):
    exe = str(tmp_path / "c_abi_consumer")
    subprocess.check_call(["gcc", "-std=c99", "-Wall", "-Werror", "-O1", os.path.join(ROOT, "tests", "c_abi_consumer.c"),
                           "-I", os.path.join(ROOT, "include"), "-L", LIBDIR, "-lausaxs_b200",
                           f"-Wl,-rpath,{LIBDIR}", "-lm", "-o", exe])
    return exe


def test_c_consumer_compiles_and_links(tmp_path):
    assert os.path.exists(_build(tmp_path))


@pytest.mark.gpu
def test_c_consumer_simple_cube(tmp_path):
    r = subprocess.run([_build(tmp_path)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.startswith("ok")
