"""Regenerate tests/golden/ffs_job/: the reference's chicken forward-facing-step job
(examples/chicken/forward-facing-step/ffs.py), prepared by the reference's own
chkn_prep.py exactly as examples/chicken/test_chicken.py prepares it (max_time edited
to 1.0e-3 s), so that the GPU path and the oracle run the reference's job unchanged on
machines without the reference tree.

Run from the repository root with the reference tree at $GDTK_RMHD_REFERENCE (default:
a sibling directory named `reference`):
    python tests/golden/make_ffs_job.py
The job: 5 x 5 x 1 lattice of 60 x 20 x 2-cell blocks (10 mm cells), 21 active and
4 inactive (below the step), M=3 inflow of air at 101.325 kPa, 300 K; gzipped text
grid and flow files.
"""
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("GDTK_RMHD_REFERENCE") or os.path.join(os.path.dirname(ROOT), "reference")


def main():
    src = os.path.join(REF, "examples", "chicken", "forward-facing-step", "ffs.py")
    out = os.path.join(HERE, "ffs_job")
    with tempfile.TemporaryDirectory() as tmp:
        with open(src) as f:
            text = f.read()
        assert "config.max_time = 5.0e-3" in text
        with open(os.path.join(tmp, "ffs.py"), "w") as f:
            f.write(text.replace("config.max_time = 5.0e-3", "config.max_time = 1.0e-3"))
        env = dict(os.environ, PYTHONPATH=os.pathsep.join([os.path.join(REF, "src", "lib"),
                                                           os.path.join(REF, "src", "chicken")]))
        subprocess.run([sys.executable, os.path.join(REF, "src", "chicken", "chkn_prep.py"), "-f", "ffs"],
                       cwd=tmp, env=env, check=True, stdout=subprocess.DEVNULL)
        shutil.rmtree(out, ignore_errors=True)
        shutil.copytree(os.path.join(tmp, "ffs"), out)


if __name__ == "__main__":
    main()
