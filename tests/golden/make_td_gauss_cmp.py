"""Copy the reference testsuite's td-gauss final-value references (testsuite/td-gauss-*/ref/
test.<tag>.cmp.ref: name, value, tolerance per line) into tests/golden/td_gauss_cmp/, the golden
values of tests/test_gpu_driver.py (the reference's own TD drivers linked against this library).

    WSLDA_REFERENCE=<reference tree> python tests/golden/make_td_gauss_cmp.py
"""
import glob
import os
import shutil

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REFERENCE = os.environ.get("WSLDA_REFERENCE", os.path.join(REPO, os.pardir, "reference"))
OUT = os.path.join(HERE, "td_gauss_cmp")

if __name__ == "__main__":
    os.makedirs(OUT, exist_ok=True)
    for fam in ("bdg", "slda", "aslda", "sldae", "sldae-a1"):
        for src in sorted(glob.glob(os.path.join(REFERENCE, "testsuite", f"td-gauss-{fam}", "ref", "*.cmp.ref"))):
            dst = os.path.join(OUT, f"td-gauss-{fam}.{os.path.basename(src)}")
            shutil.copyfile(src, dst)
            print(dst)
