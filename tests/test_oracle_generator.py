"""The oracle's restatement of the benchmark graph generator builds the same
graphs, bit for bit, as the library's sbp_dcsbm_generate, and the reference
arm of bench.py, which uses it, never loads the library."""
import json
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KEYS = ("out_ptr", "out_idx", "out_w", "in_ptr", "in_idx", "in_w", "deg_out", "deg_in",
        "true_partitions")


@pytest.mark.parametrize("variant,N,B,seed", [
    ("LL", 1000, 11, 0), ("LH", 1000, 11, 4), ("HL", 5000, 20, 2), ("HH", 20000, 32, 3),
    ("HH", 200000, 71, 0)])
def test_oracle_generator_matches_library(sbp, orc, variant, N, B, seed):
    a = orc.dcsbm_variant(variant, N, B, seed=seed)
    b = sbp.dcsbm_variant(variant, N, B, seed=seed)
    assert a.N == b.N and a.E == b.E
    for k in KEYS:
        assert np.array_equal(getattr(a, k), getattr(b, k)), k


def test_oracle_generator_other_parameters(sbp, orc):
    # alpha < 1 (the boosted gamma draw), a narrow degree law, a single block
    for kw in (dict(N=3000, B=40, alpha=0.3, p_in=0.7, seed=9),
               dict(N=500, B=1, alpha=2.0, p_in=0.0, seed=1, deg_min=1, deg_max=3),
               dict(N=800, B=800, alpha=5.0, p_in=1.0, seed=2, exponent=1.5)):
        a, b = orc.dcsbm(**kw), sbp.dcsbm(**kw)
        for k in KEYS:
            assert np.array_equal(getattr(a, k), getattr(b, k)), (kw, k)
    with pytest.raises(ValueError):
        orc.dcsbm(N=10, B=20, alpha=1.0, p_in=0.5)


def test_reference_arm_never_loads_the_library(tmp_path):
    # a stand-in for oracle/_ref/gsap_ref that answers with the planted-free
    # labels v mod 71, so the arm's scoring path runs without a GPU
    fake = tmp_path / "gsap_ref"
    fake.write_text(textwrap.dedent(f"""\
        #!{sys.executable}
        import struct, sys
        import numpy as np
        hdr = np.fromfile(sys.argv[1], dtype=np.int32, count=4)
        N = int(hdr[1])
        (np.arange(N, dtype=np.int32) % 71).tofile(sys.argv[3])
        print('{{"run": 0, "ms": 1234.5, "B": 71, "cuda": "no error"}}')
        """))
    fake.chmod(0o755)
    code = textwrap.dedent(f"""\
        import json, sys
        sys.path.insert(0, {ROOT!r})
        import bench
        class A: pass
        a = A(); a.ref_steps = 2; a.ref_warmup = 0; a.ref_timeout = 60; a.steps = 20
        a.ref_max_steps = 3
        line = bench.run_reference(a, 0, 1, 0)
        maps = open("/proc/self/maps").read()
        print(json.dumps({{"line": line, "libsbp": "libsbp.so" in maps,
                          "module": "gsap_b200.sbp" in sys.modules}}))
        """)
    env = dict(os.environ, GSAP_REF_EXE=str(fake), CUDA_VISIBLE_DEVICES="")
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env,
                       timeout=600, cwd=ROOT)
    assert p.returncode == 0, p.stderr[-2000:]
    out = json.loads(p.stdout.strip().splitlines()[-1])
    assert not out["libsbp"] and not out["module"]
    line = out["line"]
    assert line["impl"] == "reference" and line["steps"] == 2 and not line["same_steps"]
    assert abs(line["ms_per_step"] - 1234.5) < 1e-9
    q = line["quality"]
    assert q["B"] == 71 and len(q["runs"]) == 2 and q["S"] > 0
