"""The HGP kernel's shared-memory carve-up, checked on the host for every
Fock class, FP64 and FP32 recurrence sizes, every CTA width, forced slot
counts 0-2 and contraction degrees to 121 x 121: every region 16-byte
aligned, disjoint, inside the 216 KiB budget and as large as the kernel
reads (tests/layout_harness.cpp); a class that cannot fit is refused, never
laid out short."""

import os
import shutil
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_every_layout_fits_what_the_kernel_reads(tmp_path):
    exe = tmp_path / "layout_harness"
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(REPO, "include"),
                    "-I", os.path.join(REPO, "felizjueves_b200", "csrc"),
                    os.path.join(REPO, "tests", "layout_harness.cpp"),
                    os.path.join(REPO, "felizjueves_b200", "csrc", "hgp_tables.cpp"), "-o", str(exe)],
                   check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-2000:]
    assert "violations 0" in r.stdout
