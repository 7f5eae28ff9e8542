"""The C ABI from compiled C: abt_b200/examples/c_drop_in.c built with gcc."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def build_c_caller(tmp_path):
    exe = str(tmp_path / "c_drop_in")
    libdir = os.path.join(ROOT, "abt_b200")
    subprocess.check_call(["gcc", "-O2", "-std=c99", "-I", os.path.join(ROOT, "include"),
                           os.path.join(libdir, "examples", "c_drop_in.c"), "-o", exe,
                           "-L", libdir, "-lpbt_b200", "-Wl,-rpath," + libdir, "-lm"])
    return exe


def test_c_caller_builds(tmp_path):
    assert os.path.exists(build_c_caller(tmp_path))


@pytest.mark.gpu
def test_c_caller_runs(tmp_path):
    exe = build_c_caller(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("ok ")


def build_batch_caller(tmp_path):
    exe = str(tmp_path / "c_batch_beamlist")
    libdir = os.path.join(ROOT, "abt_b200")
    subprocess.check_call(["gcc", "-O2", "-std=c99", "-Wall", "-I", os.path.join(ROOT, "include"),
                           os.path.join(libdir, "examples", "c_batch_beamlist.c"), "-o", exe,
                           "-L", libdir, "-lpbt_b200", "-Wl,-rpath," + libdir, "-lm"])
    return exe


def test_c_batch_caller_file_steps_without_gpu(tmp_path):
    """The beam-list writer/reader and the far-field bins from C need no GPU."""
    exe = build_batch_caller(tmp_path)
    r = subprocess.run([exe, str(tmp_path / "o.pbtb")], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("ok")


@pytest.mark.gpu
def test_c_batch_caller_runs(tmp_path):
    exe = build_batch_caller(tmp_path)
    r = subprocess.run([exe, str(tmp_path / "o.pbtb")], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("ok ")
