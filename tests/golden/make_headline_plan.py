"""Write the headline workload's plan text to tests/golden/headline/matching_n70_w30_plan.txt.

    python tests/golden/make_headline_plan.py

The workload is the n = 70, depth-70 random-matching circuit (seed 2) with a Haar U3 layer, on the width-30 order the
native order search finds (seed 12).  The benchmark's reference arm reads this file, so that timing the reference
executor needs nothing from this repository's package or library; tests/test_host.py checks that the file equals
what the package builds.
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "headline", "matching_n70_w30_plan.txt")


def main():
    sys.path.insert(0, os.path.join(ROOT, "exact-graphstate-sampling_b200"))
    import workloads
    w = workloads.matching_n70_w30()
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    with open(OUT, "w") as f:
        f.write(w["plan"])
    print(f"wrote {OUT}: n = {w['n']}, width {w['width']}, {len(w['steps'])} steps")


if __name__ == "__main__":
    main()
