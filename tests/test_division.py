"""CPU check of the exact division by a small count used by the smoothers
(div_by_count in smokesim_b200/csrc/common.cuh): the same bits as IEEE
division, signed zeros included, for f = 1..6 and every finite float.  The
full sweep over all 2^32 bit patterns (`division_check 1`) found no mismatch;
this test runs a strided subset plus the signed zeros, subnormal and
threshold neighbourhoods."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def test_division_by_count_matches_ieee(tmp_path):
    exe = tmp_path / "division_check"
    env = dict(os.environ)
    env.pop("CC", None)
    subprocess.run(["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-march=x86-64-v3",
                    os.path.join(HERE, "division_check.c"), "-o", str(exe), "-lm"], check=True, env=env)
    r = subprocess.run([str(exe), "4093"], stdout=subprocess.PIPE, text=True)
    assert r.returncode == 0, r.stdout
    assert " 0 bit mismatches" in r.stdout
