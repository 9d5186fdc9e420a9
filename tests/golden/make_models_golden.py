"""Golden vectors of the einsum paths of ``code/backflow/models.py``, computed by the reference's
own code: the tables of ``_einsum_tables`` (distances and the d-wave form factor F^d,
``models.py:69-84``), ``PfaffianBackflow.pairing_matrix`` (feature split of the network output,
spin blocks, envelope, ``models.py:163-196``) and ``BCSBackflow.pairing_matrix`` (up x down
block plus delta_d F^d, ``models.py:272-281``).

    python tests/golden/make_models_golden.py REFERENCE_ROOT

The module is loaded as in ``make_pairing_golden.py`` (numpy in place of JAX where JAX is
missing), with empty stand-ins for the libraries it imports at module level that are missing
(equinox, quantax, fermix): their names only have to exist for the module to load, and none of
them is called by the functions run here.  The models are made with ``object.__new__`` and their fields set directly (no quantax
lattice); the Pfaffian model's network is the identity, so ``pairing_matrix(x)`` starts from a
given network output x (2 d, LX, LY), and the BCS model's ``features`` returns the given (2, N, d)
features.  Writes ``tests/golden/models_golden.npz``; for case k of CASES (LX, LY, d):

* ``dist_k``, ``fd_k`` (N, N): the pair tables (FP32, as the reference stores them);
* ``x_k`` (B, 2 d, LX, LY), ``W_k`` (3, N, d), ``theta_k``, ``Fpf_k`` (B, 2N, 2N): the Pfaffian
  model's antisymmetric pairing matrix;
* ``y_k`` (B, 2, N, d), ``Wb_k`` (N, d), ``thetab_k``, ``delta_k``, ``Fbcs_k`` (B, N, N): the
  BCS model's pairing matrix f_ud + delta_d F^d.
"""

import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from make_pairing_golden import install_jax_stand_in, load_reference_kernels  # noqa: E402

CASES = [(4, 4, 16), (6, 4, 8), (8, 8, 16)]
BATCH = 1


def install_library_stand_ins():
    import importlib.util

    if all(importlib.util.find_spec(m) is not None for m in ("equinox", "quantax", "fermix")):
        return

    class _Any(types.ModuleType):
        def __getattr__(self, name):
            return lambda *a, **k: None

    eqx = _Any("equinox")
    eqx.Module = type("Module", (), {})
    mods = {"equinox": eqx, "fermix": _Any("fermix"), "quantax": _Any("quantax")}
    for sub in ("model", "nn", "symmetry", "utils"):
        mods[f"quantax.{sub}"] = _Any(f"quantax.{sub}")
    mods["quantax.model"].ResConv = type("ResConv", (), {})
    mods["quantax.symmetry"].Identity = type("Identity", (), {})
    mods["quantax.utils"].LogArray = type("LogArray", (), {})
    sys.modules.update(mods)


def load_reference_models(root):
    import importlib.util

    pfk, bcs = load_reference_kernels(root)
    spec = importlib.util.spec_from_file_location(
        "reference_backflow.models", os.path.join(root, "code", "backflow", "models.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod
    spec.loader.exec_module(mod)
    return pfk, bcs, mod


def main(argv):
    if len(argv) != 2:
        raise SystemExit(__doc__)
    install_jax_stand_in()
    install_library_stand_ins()
    pfk, bcs, models = load_reference_models(argv[1])
    rng = np.random.default_rng(77)
    out = {"cases": np.array(CASES, np.int32)}
    for k, (LX, LY, d) in enumerate(CASES):
        N = LX * LY
        tables = models._einsum_tables(LX, LY)
        # fields set with object.__setattr__: equinox modules are frozen dataclasses
        pf = object.__new__(models.PfaffianBackflow)
        W, theta = rng.normal(0.0, 0.5, size=(3, N, d)), np.float64(rng.normal(0.0, 0.5))
        for name, v in (("net", lambda s: s), ("d", d), ("W", W), ("theta", theta),
                        ("geom", pfk.PairGeometry(LX, LY, d, 0, 0))):
            object.__setattr__(pf, name, v)
        x = rng.normal(0.0, 1.0, size=(BATCH, 2 * d, LX, LY))
        Fpf = np.stack([np.asarray(pf.pairing_matrix(x[b])) for b in range(BATCH)])
        bm = object.__new__(models.BCSBackflow)
        Wb, thetab = rng.normal(0.0, 0.5, size=(N, d)), np.float64(rng.normal(0.0, 0.5))
        delta = np.float64(rng.normal(0.0, 0.3))
        for name, v in (("features", lambda s: s), ("W", Wb), ("theta", thetab),
                        ("delta_d", delta), ("geom", bcs.UDGeometry(LX, LY, d, 0, 0))):
            object.__setattr__(bm, name, v)
        y = rng.normal(0.0, 1.0, size=(BATCH, 2, N, d))
        Fbcs = np.stack([np.asarray(bm.pairing_matrix(y[b])) for b in range(BATCH)])
        out.update({f"dist_{k}": tables.dist, f"fd_{k}": tables.fd, f"x_{k}": x,
                    f"W_{k}": W, f"theta_{k}": theta, f"Fpf_{k}": Fpf, f"y_{k}": y,
                    f"Wb_{k}": Wb, f"thetab_{k}": thetab, f"delta_{k}": delta,
                    f"Fbcs_{k}": Fbcs})
    dst = os.path.join(HERE, "models_golden.npz")
    np.savez_compressed(dst, **out)
    print(dst, os.path.getsize(dst), "bytes")


if __name__ == "__main__":
    main(sys.argv)
