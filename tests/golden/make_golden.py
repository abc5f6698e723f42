"""Regenerate the golden input fixtures of tests/golden from the reference's own
initial-data scripts (inipar/briowu-test12.py, inipar/riemann-test11.py,
inipar/strongshock-test11.py of drewleonard42/SAC).

Run with the reference tree's root in the environment variable SAC_REFERENCE
(required); each script is executed unmodified in a scratch directory and the
.ini file it writes is copied here.  The tests read only the copies.

    SAC_REFERENCE=<path to the SAC tree> python tests/golden/make_golden.py

The scripts were written for Python 2, whose list comprehensions leak their loop
variable: line 37 of each uses `p`, the last entry of `nprocs` (1 for the `_np01`
file names).  Under Python 3 that name must be supplied, which is all
`init_globals` does here.
"""
import os
import runpy
import shutil
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
SCRIPTS = {
    "briowu-test12.py": "data/briowu-test12_np01_000.ini",
    "riemann-test11.py": "data/riemann-test11_np01_000.ini",
    "strongshock-test11.py": "data/strongshock-test11_np01_000.ini",
}


def main():
    ref = os.environ.get("SAC_REFERENCE")
    if not ref or not os.path.isdir(os.path.join(ref, "inipar")):
        raise SystemExit("set SAC_REFERENCE to the root of the SAC tree (the directory holding inipar/)")
    for script, out in SCRIPTS.items():
        src = os.path.join(ref, "inipar", script)
        with tempfile.TemporaryDirectory() as tmp:
            os.makedirs(os.path.join(tmp, "data"))
            cwd = os.getcwd()
            try:
                os.chdir(tmp)
                runpy.run_path(src, init_globals={"p": 1}, run_name="__main__")
            finally:
                os.chdir(cwd)
            shutil.copy(os.path.join(tmp, out), os.path.join(HERE, os.path.basename(out)))
            print("wrote", os.path.basename(out))


if __name__ == "__main__":
    main()
