"""The drop-in headers: a GSAP-style C++ caller (tests/dropin_main.cpp)
compiled against include/ gets the same labels as the Python binding."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp_path):
    exe = tmp_path / "dropin"
    lib = os.path.join(ROOT, "gsap_b200")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "dropin_main.cpp"), os.path.join(lib, "libsbp.so"),
                    f"-Wl,-rpath,{lib}", "-o", str(exe)], check=True)
    return exe


def _write_tsv(g, path):
    src, dst, w = g.edges()
    with open(path, "w") as f:
        for a, b, c in zip(src, dst, w):
            f.write(f"{a + 1}\t{b + 1}\t{c}\n")


def test_dropin_headers_compile(tmp_path):
    assert _build(tmp_path).exists()


@pytest.mark.gpu
def test_dropin_partition_matches_binding(sbp, tmp_path):
    exe = _build(tmp_path)
    g = sbp.dcsbm_variant("LH", 1000, 11, seed=3)
    tsv = tmp_path / "g.tsv"
    _write_tsv(g, tsv)
    out = tmp_path / "labels.bin"
    r = subprocess.run([str(exe), str(tsv), str(out)], capture_output=True, text=True, check=True)
    assert f"N={g.N} E={g.E}" in r.stdout
    lab = np.fromfile(out, dtype=np.int32)
    sbp.partition(g, seed=0)
    assert np.array_equal(lab, g.partitions)
