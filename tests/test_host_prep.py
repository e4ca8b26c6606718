"""The engine's host-side layout preparation (csrc/host_prep.hpp) checked on CPU under
AddressSanitizer and UBSan: CSR sorting and padding, weight classification, plastic plans and the
carry-over of per-instance weights and in-flight plastic input when the plastic set grows."""

import os
import shutil
import subprocess

import pytest

from conftest import ROOT


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_host_prep_under_sanitizers(tmp_path):
    exe = tmp_path / "host_prep_check"
    csrc = os.path.join(ROOT, "can-the-fly-play-f-zero-_b200", "csrc")
    subprocess.run(["g++", "-std=c++17", "-O1", "-g", "-fsanitize=address,undefined", "-fno-sanitize-recover=all",
                    "-I", csrc, os.path.join(ROOT, "tests", "host_prep_check.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL OK" in r.stdout
