"""Chain statistics on the host: integrated autocorrelation time, effective sample rate and
block-jackknife errors (the error analysis of ``code/measure/assemble.py:48-84``).

tau_int follows A. Sokal, "Monte Carlo methods in statistical mechanics: foundations and new
algorithms" (Cargese lectures, 1996): the normalised autocorrelation averaged over chains,
summed up to the smallest window W with W >= c tau(W).
"""

from __future__ import annotations

import numpy as np


def autocorrelation(x: np.ndarray) -> np.ndarray:
    """Normalised autocorrelation rho(t), t = 0 .. T-1, of a series (T,) or of chains (T, B)
    (each chain centred on its own mean, the autocovariances averaged over chains)."""
    x = np.asarray(x, np.float64)
    if x.ndim == 1:
        x = x[:, None]
    T = x.shape[0]
    xc = x - x.mean(0, keepdims=True)
    f = np.fft.rfft(xc, n=2 * T, axis=0)
    acov = np.fft.irfft(f * np.conj(f), n=2 * T, axis=0)[:T].mean(1)
    if acov[0] <= 0:
        out = np.zeros(T)
        out[0] = 1.0
        return out
    return acov / acov[0]


def tau_int_window(x: np.ndarray, c: float = 5.0):
    """(tau, W): tau = 1/2 + sum_{t=1}^{W} rho(t) and Sokal's window W (the smallest W with
    W >= c tau(W))."""
    rho = autocorrelation(x)
    tau = 0.5
    W = 0
    for W in range(1, len(rho)):
        tau += rho[W]
        if W >= c * tau:
            break
    return float(max(tau, 0.5)), int(W)


def tau_int(x: np.ndarray, c: float = 5.0) -> float:
    """Integrated autocorrelation time tau = 1/2 + sum_{t=1}^{W} rho(t) with Sokal's window."""
    return tau_int_window(x, c)[0]


def tau_int_error(x: np.ndarray, c: float = 5.0, groups: int = 8) -> dict:
    """tau_int of a (T, B) chain series with two error bars: Sokal's variance estimate
    var(tau) = 2 (2W + 1) / (T B) tau^2 (independent chains averaged), and the spread of tau over
    ``groups`` disjoint sets of chains divided by sqrt(groups) (empirical; needs B >= 2 groups)."""
    x = np.asarray(x, np.float64)
    if x.ndim == 1:
        x = x[:, None]
    T, B = x.shape
    tau, W = tau_int_window(x, c)
    out = {"tau": tau, "window": W, "err_sokal": float(np.sqrt(2.0 * (2 * W + 1) / (T * B)) * tau)}
    if B >= 2 * groups:
        taus = [tau_int(x[:, g::groups], c) for g in range(groups)]
        out["err_groups"] = float(np.std(taus, ddof=1) / np.sqrt(groups))
    else:
        out["err_groups"] = None
    return out


def effective_rate(n_chains: int, n_steps: int, tau: float, seconds: float) -> float:
    """Effective samples per second: chains x steps / (2 tau_int x time).  With tau_int in the
    convention above an uncorrelated series has tau = 1/2 and counts every step."""
    return float(n_chains) * float(n_steps) / (2.0 * float(tau) * float(seconds))


def jackknife_mean(x: np.ndarray, blocks=(1, 2, 4, 8), min_blocks: int = 8):
    """Mean and the largest block-jackknife error over the given block sizes."""
    x = np.asarray(x, np.float64)
    val = float(x.mean())
    errs = []
    for b in blocks:
        nb = x.shape[0] // b
        if nb < min_blocks:
            continue
        xb = x[: nb * b].reshape(nb, b).mean(1)
        reps = (xb.sum() - xb) / (nb - 1)
        errs.append(np.sqrt(nb - 1) * reps.std())
    return val, float(max(errs)) if errs else float("nan")
