"""The tribit CLI keeps the reference's argument contract
(src/single_gpu/tribit.cu:282-315) -- checked here without a GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "tribit_b200", "bin", "tribit")


def run(*args):
    return subprocess.run([CLI, *args], capture_output=True, text=True, timeout=60)


def test_cli_built():
    assert os.access(CLI, os.X_OK)


def test_no_args_usage():
    r = run()
    assert r.returncode == 1
    assert "Usage:" in r.stderr and "-i <input_file>" in r.stderr
    assert r.stdout.startswith("Thrust version: ")
    assert "CUB version: " in r.stdout


def test_unknown_option():
    r = run("-z")
    assert r.returncode == 1
    assert "Error: unknown option or missing argument" in r.stderr


def test_missing_input():
    r = run("-v")
    assert r.returncode == 1
    assert "Error: input file is required (-i option)" in r.stderr


def test_missing_file():
    r = run("-i", "/nonexistent/x.mtx")
    assert r.returncode == 1
    assert "Reading data from /nonexistent/x.mtx..." in r.stdout
    assert "cannot open" in r.stderr


def test_extra_args_warning(tmp_path):
    p = tmp_path / "g.mtx"
    p.write_text("%%MatrixMarket matrix coordinate pattern general\n3 3 3\n1 2\n2 3\n3 1\n")
    r = run("-i", str(p), "extra")
    assert "Warning: extra arguments ignored" in r.stderr
