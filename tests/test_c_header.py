"""Binary compatibility with the reference's C users: a C99 program written
against the reference's own public header (include/fastprox.h) compiles with
-Werror, links to libfastprox_b200.so in place of libfastprox and runs (here
without a GPU: operators, parameters, error codes and FP_EDEVICE for a
solve); the same program against this library's header solves a batch on the
GPU (-m gpu). This library's header compiles as strict C99 on its own."""

import pathlib
import subprocess

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "c" / "header_caller.c"
LIBDIR = ROOT / "fastprox_b200"


def _compile(tmp_path, include, header):
    exe = tmp_path / "caller"
    cmd = ["gcc", "-std=c99", "-pedantic", "-Wall", "-Wextra", "-Werror", f"-DFP_HEADER=\"{header}\"",
           f"-I{include}", str(SRC), "-o", str(exe), f"-L{LIBDIR}", "-lfastprox_b200", f"-Wl,-rpath,{LIBDIR}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return exe


def _reference_include():
    r = subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "have-ref"], capture_output=True)
    if r.returncode != 0:
        return None
    out = subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "ref-include"], capture_output=True, text=True)
    return out.stdout.strip()


def test_own_header_is_strict_c99():
    r = subprocess.run(["gcc", "-std=c99", "-pedantic", "-Wall", "-Wextra", "-Werror", "-fsyntax-only", "-x", "c",
                        str(ROOT / "include" / "fastprox_b200.h")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_reference_header_caller_links_and_runs(tmp_path):
    inc = _reference_include()
    if inc is None:
        pytest.skip("the reference's sources are not present")
    exe = _compile(tmp_path, inc, "fastprox.h")
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("ok"), r.stdout


@pytest.mark.gpu
def test_caller_solves_on_the_gpu(cuda, tmp_path):
    exe = _compile(tmp_path, ROOT / "include", "fastprox_b200.h")
    r = subprocess.run([str(exe), "gpu"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "solved" in r.stdout and r.stdout.strip().endswith("ok"), r.stdout
