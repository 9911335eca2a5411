"""Install the reference for the benchmark's reference arm.

The reference is Fortran 90 and this image has no Fortran compiler (nor does
`pip install --target baseline/_ref <reference tree>` apply: the tree has no Python build).  Its
repository ships a prebuilt Linux x86-64 executable (src/fastspec_Linux_x86_64, OpenMP); this
recipe copies that executable, unmodified, to baseline/_ref/ so that `bench.py --impl reference`
runs the reference's own stock build on the host cores of the machine it runs on.  The executable
is only run (decks in, fs_*.bin out), never inspected.

    python oracle/install_reference.py [reference tree]
The tree: the argument, else $FASTSPEC_REFERENCE, else the read-only mount the build machine keeps it
at (MOUNT); when none exists nothing is installed.
"""
import os
import shutil
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DEST = os.path.join(REPO, "baseline", "_ref")
NAME = "fastspec_Linux_x86_64"
MOUNT = "/root/reference"


def install(ref_tree=None):
    ref_tree = ref_tree or os.environ.get("FASTSPEC_REFERENCE") or MOUNT
    src = os.path.join(ref_tree, "src", NAME)
    if not os.path.exists(src):
        return None
    os.makedirs(DEST, exist_ok=True)
    dst = os.path.join(DEST, NAME)
    if not os.path.exists(dst) or os.path.getsize(dst) != os.path.getsize(src):
        shutil.copy2(src, dst)
    os.chmod(dst, 0o755)
    return dst


if __name__ == "__main__":
    print(install(*sys.argv[1:]) or "reference executable not found")
