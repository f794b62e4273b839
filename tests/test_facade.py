"""The C++ facade include/interface.hpp: code written against the
reference's IBFMM_Mat<3> interface compiles unchanged and runs."""
import os
import re
import shutil
import subprocess

import pytest

from oracle import refsrc

REF = refsrc.reference_dir()
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "defmm_b200")


def compile_driver(src, out, incdir):
    cmd = ["g++", "-std=c++17", "-O2", src, "-I", incdir, f"-L{LIBDIR}", "-ldefmm_b200",
           f"-Wl,-rpath,{LIBDIR}", "-o", out]
    cp = subprocess.run(cmd, capture_output=True, text=True)
    assert cp.returncode == 0, cp.stderr


def test_facade_driver_compiles(tmp_path):
    compile_driver(os.path.join(ROOT, "tests", "cpp", "facade_driver.cpp"), str(tmp_path / "drv"),
                   os.path.join(ROOT, "include"))


@pytest.mark.skipif(not REF or not os.path.isfile(os.path.join(REF, "test", "testinterface.cpp")),
                    reason="reference checkout absent")
def test_reference_driver_compiles_unchanged(tmp_path):
    # the reference's driver includes "../include/interface.hpp"
    (tmp_path / "test").mkdir()
    shutil.copy(os.path.join(REF, "test", "testinterface.cpp"), tmp_path / "test")
    os.symlink(os.path.join(ROOT, "include"), tmp_path / "include")
    compile_driver(str(tmp_path / "test" / "testinterface.cpp"), str(tmp_path / "testinterface"),
                   str(tmp_path / "include"))


@pytest.mark.gpu
def test_facade_driver_runs(tmp_path, gpu):
    exe = str(tmp_path / "drv")
    compile_driver(os.path.join(ROOT, "tests", "cpp", "facade_driver.cpp"), exe, os.path.join(ROOT, "include"))
    cp = subprocess.run([exe, str(tmp_path / "pts.inp")], capture_output=True, text=True, timeout=600)
    assert cp.returncode == 0, cp.stderr
    out = re.sub(r"\x1b\[[0-9;]*m", "", cp.stdout)
    l2 = float(re.search(r"L\^2  norm: ([0-9.eE+-]+)", out).group(1))
    assert l2 < 1e-2
