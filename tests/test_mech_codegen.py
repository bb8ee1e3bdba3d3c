"""The compiled mechanism header (opencfd-comb_b200/csrc/ocfd_mech_h2air9.cuh) is what its
generator writes from the mechanism data file today, and its structure is that file's."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GEN = os.path.join(ROOT, "opencfd-comb_b200", "csrc", "gen_mech.py")


def test_generated_header_is_current():
    r = subprocess.run([sys.executable, GEN, "--check"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr


def test_generated_terms_follow_the_stoichiometry():
    sys.path.insert(0, os.path.dirname(GEN))
    import gen_mech
    text = gen_mech.generate()
    with open(gen_mech.DATA) as fh:
        kin = json.load(fh)["kinetics"]
    for j, r in enumerate(kin["reactions"]):
        # the second block of reaction j (Reaction_rate_and_Matrix) adds one Jacobian column per
        # species with a part in it, one row per species whose amount it changes
        block = text.split("  {  // %d: " % j)[2]
        cols = sum(1 for a, b in zip(r["vf"], r["vr"]) if a or b)
        block = block.split("  {  // ")[0]
        assert block.count("const double dA") == cols
        rows = sum(1 for a, b in zip(r["vf"], r["vr"]) if b - a)
        assert block.count("Ar[") == 2 * rows * cols
