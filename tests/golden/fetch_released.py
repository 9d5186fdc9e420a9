"""Copy the released 16x16 Pfaffian-backflow state (parameters and equilibrated chains) from a
checkout of the reference into tests/golden/released/, checking the parameter file's md5.

    python tests/golden/fetch_released.py REFERENCE_ROOT [NAME ...]

REFERENCE_ROOT is the root of a ChenAo-Phys/NeuralHubbard checkout (it holds weights/); NAME
defaults to tpm02_L16_pfaffian.  The copies are not
committed (tests/golden/released/ is git-ignored: 5 MB of weights); tests that need them skip
when they are absent.
"""

import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from neuralhubbard_b200 import checkpoint  # noqa: E402


def main(argv):
    if len(argv) < 2:
        raise SystemExit(__doc__)
    root = argv[1]
    names = argv[2:] or ["tpm02_L16_pfaffian"]
    out = os.path.join(HERE, "released")
    os.makedirs(out, exist_ok=True)
    for name in names:
        for suffix in (".eqx", "_spins.npz"):
            src = os.path.join(root, "weights", name + suffix)
            dst = os.path.join(out, name + suffix)
            shutil.copyfile(src, dst)
            print(dst)
        md5 = checkpoint.file_md5(os.path.join(out, name + ".eqx"))
        if md5 != checkpoint.RELEASED[name].md5:
            raise SystemExit(f"{name}.eqx: md5 {md5}, released {checkpoint.RELEASED[name].md5}")


if __name__ == "__main__":
    main(sys.argv)
