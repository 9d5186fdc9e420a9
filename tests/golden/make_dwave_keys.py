"""Golden key orders of the packed d-wave measurement, generated by the reference's own
``code/measure/observables.py`` (``SquareGeometry``, ``dwave_keys``; the module imports only
numpy, so it loads without JAX).

    python tests/golden/make_dwave_keys.py REFERENCE_ROOT

REFERENCE_ROOT is the root of a ChenAo-Phys/NeuralHubbard checkout.  Writes
``tests/golden/dwave_keys.npz``; for case k of CASES (LX, LY, R, primary_only):

* ``F_k``: the F keys as int rows (bx, by, bax, oL, cx, cy, cax, oR), the reference's
  ``F_keys_to_int`` layout (``code/measure/observables.py:152-154``);
* ``G_k``: the G keys as int rows (ix, iy, jx, jy, spin), spin up 0 and down 1
  (``G_keys_to_int``, ``:157-159``);
* ``left_k``: the left bonds (bx, by, bax) in the reference's order;
* ``strings_k``: (site index of c+_up, site index of c+_dn) of A+(bond, o) for every bond of
  ``all_bonds`` and o = 0, 1 in that order (``string_sites``), i.e. the packed pair term t =
  2 bond + o that a connected configuration is binned into (``dwave_packed.py:50-56``).
"""

import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = [(4, 4, (0, 0), True), (8, 8, (1, 2), True), (6, 4, (5, 3), False),
         (16, 16, (0, 0), True)]


def load_reference_observables(root):
    path = os.path.join(root, "code", "measure", "observables.py")
    spec = importlib.util.spec_from_file_location("reference_measure_observables", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def main(argv):
    if len(argv) != 2:
        raise SystemExit(__doc__)
    ref = load_reference_observables(argv[1])
    out = {}
    for k, (LX, LY, R, primary) in enumerate(CASES):
        geo = ref.SquareGeometry(LX, LY)
        left_bonds, _left_sites, F_keys, G_keys = ref.dwave_keys(geo, R, primary)
        out[f"F_{k}"] = ref.F_keys_to_int(F_keys)
        out[f"G_{k}"] = ref.G_keys_to_int(G_keys)
        out[f"left_{k}"] = np.array(left_bonds, np.int32)
        out[f"strings_{k}"] = np.array(
            [[geo.index(p) for p in geo.string_sites(b, o)] for b in geo.all_bonds
             for o in (0, 1)], np.int32)
    out["cases"] = np.array([(LX, LY, R[0], R[1], int(p)) for LX, LY, R, p in CASES], np.int32)
    dst = os.path.join(HERE, "dwave_keys.npz")
    np.savez_compressed(dst, **out)
    print(dst, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main(sys.argv)
