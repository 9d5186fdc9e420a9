"""Golden vectors of the pairing tables and occupied gathers, computed by the reference's own
functions in ``code/backflow/pf_kernel.py`` (``displacement_tables``, ``build_wtilde``,
``pairing_matrix_occ`` with ``reference=True``, i.e. ``pairing_occ_reference``) and
``code/backflow/bcs_kernel.py`` (``build_wt_ud``, ``pairing_block_ud`` with
``reference=True``, i.e. ``pairing_ud_reference``).

    python tests/golden/make_pairing_golden.py REFERENCE_ROOT

Where JAX is installed it is used, with 64-bit types enabled.  Where it is not, the two modules
are loaded with a stand-in ``jax`` module whose ``jax.numpy`` is numpy (``einsum``'s
``precision`` argument dropped), ``jax.nn.softplus`` is log(1 + e^x) and ``jax.custom_vjp``
passes calls through; these reference functions use nothing else of JAX, so they run unchanged
in FP64.  The package ``__init__`` (which imports equinox, quantax and fermix) is not executed.
Writes ``tests/golden/pairing_golden.npz``; for case k of CASES (LX, LY, d, n_up, n_dn), with
seeded inputs stored beside the outputs:

* ``disp_k``, ``neg_k``, ``dist_k``: the displacement tables (``dist`` in FP32, as the
  reference stores it);
* ``W_k`` (3, N, d), ``theta_k``, ``Wt_k`` (4, N, d): ``build_wtilde``;
* ``y_k`` (B, 2, N, d) features, ``s_k`` (B, 2N) int8 configurations, ``F_k`` (B, n, n):
  ``pairing_matrix_occ(y, idx, W, theta, geom, reference=True)`` with idx the occupied modes
  in ascending order (the reference's ``fermion_idx`` order);
* ``Wud_k`` (N, d): ``build_wt_ud(W[0], theta)``; ``Fud_k`` (B, n_up, n_dn):
  ``pairing_block_ud(y, iu, idn, W[0], theta, geom, reference=True)`` with iu, idn the
  occupied up and down sites in ascending order (no d-wave term: the reference adds it
  outside this function).
"""

import importlib.util
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = [(4, 4, 16, 7, 7), (6, 4, 8, 10, 10), (8, 8, 16, 28, 28)]
BATCH = 3


def install_jax_stand_in():
    if importlib.util.find_spec("jax") is not None:
        import jax

        jax.config.update("jax_enable_x64", True)
        return

    class _NumpyAsJnp(types.ModuleType):
        def __getattr__(self, name):
            return getattr(np, name)

    jnp = _NumpyAsJnp("jax.numpy")
    jnp.einsum = lambda *a, precision=None, **k: np.einsum(*a, **k)
    lax = types.ModuleType("jax.lax")
    lax.Precision = types.SimpleNamespace(HIGHEST="highest")

    class custom_vjp:
        def __init__(self, fun, nondiff_argnums=()):
            self.fun = fun

        def defvjp(self, fwd, bwd):
            pass

        def __call__(self, *args, **kwargs):
            return self.fun(*args, **kwargs)

    jax = types.ModuleType("jax")
    jax.numpy, jax.lax, jax.Array, jax.custom_vjp = jnp, lax, np.ndarray, custom_vjp
    jax.nn = types.SimpleNamespace(softplus=lambda x: np.logaddexp(0.0, x))
    jax.default_backend = lambda: "cpu"
    sys.modules.update({"jax": jax, "jax.numpy": jnp, "jax.lax": lax})


def load_reference_kernels(root):
    pkg = types.ModuleType("reference_backflow")
    pkg.__path__ = [os.path.join(root, "code", "backflow")]
    sys.modules[pkg.__name__] = pkg
    mods = []
    for name in ("pf_kernel", "bcs_kernel"):
        spec = importlib.util.spec_from_file_location(
            f"reference_backflow.{name}", os.path.join(pkg.__path__[0], name + ".py"))
        mod = importlib.util.module_from_spec(spec)
        sys.modules[spec.name] = mod
        spec.loader.exec_module(mod)
        mods.append(mod)
    return mods


def random_configs(rng, B, N, n_up, n_dn):
    s = -np.ones((B, 2 * N), np.int8)
    for b in range(B):
        s[b, rng.choice(N, n_up, replace=False)] = 1
        s[b, N + rng.choice(N, n_dn, replace=False)] = 1
    return s


def main(argv):
    if len(argv) != 2:
        raise SystemExit(__doc__)
    install_jax_stand_in()
    pfk, bcs = load_reference_kernels(argv[1])
    rng = np.random.default_rng(2024)
    out = {"cases": np.array(CASES, np.int32)}
    for k, (LX, LY, d, n_up, n_dn) in enumerate(CASES):
        N = LX * LY
        geom = pfk.PairGeometry(LX, LY, d, n_up, n_dn)
        disp, neg, dist = pfk.displacement_tables(geom)
        W = rng.normal(0.0, 0.5, size=(3, N, d))
        theta = np.float64(rng.normal(0.0, 0.5))
        y = rng.normal(0.0, 1.0, size=(BATCH, 2, N, d))
        s = random_configs(rng, BATCH, N, n_up, n_dn)
        F, Fud = [], []
        ugeom = bcs.UDGeometry(LX, LY, d, n_up, n_dn)
        for b in range(BATCH):
            idx = np.flatnonzero(s[b] > 0)
            F.append(pfk.pairing_matrix_occ(y[b], idx, W, theta, geom, reference=True))
            iu, idn = np.flatnonzero(s[b, :N] > 0), np.flatnonzero(s[b, N:] > 0)
            Fud.append(bcs.pairing_block_ud(y[b], iu, idn, W[0], theta, ugeom, reference=True))
        out.update({f"disp_{k}": disp.astype(np.int32), f"neg_{k}": neg.astype(np.int32),
                    f"dist_{k}": dist, f"W_{k}": W, f"theta_{k}": theta,
                    f"Wt_{k}": pfk.build_wtilde(W, theta, geom), f"y_{k}": y, f"s_{k}": s,
                    f"F_{k}": np.stack(F), f"Wud_{k}": bcs.build_wt_ud(W[0], theta, ugeom),
                    f"Fud_{k}": np.stack(Fud)})
    dst = os.path.join(HERE, "pairing_golden.npz")
    np.savez_compressed(dst, **out)
    print(dst, os.path.getsize(dst), "bytes")


if __name__ == "__main__":
    main(sys.argv)
