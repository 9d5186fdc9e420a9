#!/usr/bin/env python
"""Benchmark of the Pfaffian-backflow amplitude path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step is one projected-amplitude call ``state(spins)`` on the 16x16 lattice (N = 256,
112 + 112 electrons, 224 x 224 Pfaffians) for 8192 configurations x 8 symmetry images =
65,536 amplitudes, with seeded N(0, 0.02) weights of the 4-layer, 32-channel backflow CNN and
synthetic uniformly random configurations (no dataset is involved).  ``value`` is amplitude
evaluations per second over all ranks with the inputs resident in HBM; ``e2e`` is the same
metric through the public API with the configurations copied from pinned host memory and the
amplitudes read back every step.

``sampling`` (1 GPU) compares the plain form (FP32 CNN, uniform-hop Metropolis) with the
chosen form (tcgen05 BF16x3 CNN, learned hop proposal with the exact Hastings correction,
trained on 2^20 records of the plain chains): acceptance, tau_int of the log|psi| series,
effective samples per second and the energy per site of each, on 1024 chains that start from
the same configurations after 6000 equilibration steps.  ``local_energy`` (1 GPU) times the
ragged local energy at 8x8, 16x16 and 24x24, one CUDA-graph replay each; ``large_lattice``
(1 GPU) times Metropolis steps at 32x32 (n = 896) with the uniform hop and the learned proposal.
``precision`` (1 GPU) reports each precision form's |delta log|psi_P|| and sign mismatches
against the library's all-FP64 path, and near-nodal log-Pfaffians at the slogpf boundary.
``resconv`` (1 GPU) times the released states' residual network (16 blocks x 64 channels) on
CUDA cores and on the tensor cores, with E/N of the released 16x16 state on 512 of its chains.
``extensions`` (1 GPU) times the per-sample Jacobian of log|psi_P|, the BCS-backflow ansatz (with
its error against the BCS all-FP64 form) and the packed observables.  ``--config5`` (opt-in,
several minutes) trains the learned proposal at 32x32 on records of plain chains and compares
its tau_int and effective samples/s with the uniform hop there.

Under torchrun each rank evaluates its own 8192 configurations (weak scaling); the time is the
maximum over ranks of the summed per-step CUDA-event durations.  ``--impl reference`` times the
compiled CPU restatement of the same path (oracle/c/nh_port.c; the reference's JAX stack cannot
be installed here) on all host cores, on rank 0 only.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "effective samples/s + amplitude evals/s, 16x16 Pfaffian; chosen vs plain, 1 B200"
UNIT = "amplitude evals/s"
L, NE, BATCH, IMAGES, CHANNELS, LAYERS = 16, 112, 8192, 8, 32, 4
N_SITES = L * L
N_OCC = 2 * NE
D_FEAT = CHANNELS // 2
# Algorithmic work per amplitude (one image): CNN 2 * 9 * (2*32 + 3*32*32) FLOP per site,
# occupied gather 2 n^2 d, Pfaffian n^3 / 3 (the Table S3 convention of the reference).
CNN_FLOP = 2 * 9 * (2 * CHANNELS + (LAYERS - 1) * CHANNELS * CHANNELS) * N_SITES
GATHER_FLOP = 2 * N_OCC * N_OCC * D_FEAT
PFAFFIAN_FLOP = N_OCC ** 3 / 3.0
FP32_CORE_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12  # nominal FMA rate of the CUDA cores
# DRAM bytes per amplitude from ncu captures (dram__bytes_read.sum + dram__bytes_write.sum of a
# 2048-matrix launch, divided by 2048: traffic grows in proportion to the matrices), keyed by
# kernel; the figures are those of the summaries under profiles/.
TRAFFIC_BYTES = {"pfaffian": 31.3e6 / 2048}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), float(p["bf16_tflops"]), "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- CPU restatement (oracle)

def _cpu_worker(args):
    spins, params = args
    from oracle import projection

    t0 = time.perf_counter()
    projection.projected_amplitude(spins, params, symm=True)
    return time.perf_counter() - t0


def cpu_baseline(target_s: float = 12.0, fp32: bool = True) -> dict:
    """Projected amplitudes of the same workload by the CPU restatement on all host cores, on a
    bounded sample sized for ~target_s seconds: the compiled restatement (oracle/c/nh_port.c,
    gcc -O3, OpenMP across configurations; its FP32 build by default, the arithmetic of the
    reference's own path, or the FP64 build) when it builds, else the numpy oracle (FP64) in a
    spawn pool (one numpy thread per core)."""
    import multiprocessing as mp

    from neuralhubbard_b200.backflow import init_params
    from neuralhubbard_b200.sampler import random_spins

    try:
        cores = len(os.sched_getaffinity(0))
    except Exception:
        cores = os.cpu_count() or 1
    p = init_params(L, L, CHANNELS, LAYERS, seed=0)
    params = dict(conv_w=[w.astype(np.float64) for w in p["conv_w"]],
                  conv_b=[b.astype(np.float64) for b in p["conv_b"]],
                  W=p["W"].astype(np.float64), theta=float(p["theta"]), Lx=L, Ly=L)
    rng = np.random.default_rng(123)
    try:
        from oracle import port

        port.load(fp32)
    except Exception:
        port = None
    if port is not None:
        warm = random_spins(rng, cores, N_SITES, NE, NE)
        t0 = time.perf_counter()
        port.projected_amplitude(warm, params, threads=cores, fp32=fp32)
        t_batch = time.perf_counter() - t0
        n_cfg = max(cores, int(cores * target_s / max(t_batch, 1e-3)))
        sample = random_spins(rng, n_cfg, N_SITES, NE, NE)
        t0 = time.perf_counter()
        port.projected_amplitude(sample, params, threads=cores, fp32=fp32)
        wall = time.perf_counter() - t0
        n_amp = n_cfg * IMAGES
        prec = "FP32" if fp32 else "FP64"
        return {"value": n_amp / wall, "unit": UNIT, "cores": cores, "kind": "port",
                "sample": f"{n_cfg} configurations x {IMAGES} images at 16x16 ({n_amp} "
                          f"amplitudes, compiled {prec} restatement, gcc -O3 + OpenMP, "
                          f"{wall:.1f} s)",
                "seconds": wall}
    for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[k] = "1"
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        one = random_spins(rng, 1, N_SITES, NE, NE)
        pool.map(_cpu_worker, [(one, params)] * cores)  # warm the workers
        t_one = max(pool.map(_cpu_worker, [(one, params)] * cores))
        per_worker = max(1, int(target_s / max(t_one, 1e-3)))
        jobs = [(random_spins(rng, per_worker, N_SITES, NE, NE), params) for _ in range(cores)]
        t0 = time.perf_counter()
        pool.map(_cpu_worker, jobs)
        wall = time.perf_counter() - t0
    n_amp = cores * per_worker * IMAGES
    return {"value": n_amp / wall, "unit": UNIT, "cores": cores, "kind": "numpy",
            "sample": f"{cores * per_worker} configurations x {IMAGES} images at 16x16 "
                      f"({n_amp} amplitudes, FP64 numpy restatement, {wall:.1f} s)",
            "seconds": wall}


# ---------------------------------------------------------------- GPU arm

def time_amplitudes(state, spins, steps, warmup, flush, st, profile=False):
    """Warm-up, then ``steps`` timed calls of ``state(spins)`` with L2 flushed between them
    (outside the events).  Returns (summed step milliseconds, per-kernel profile or {})."""
    import torch

    from neuralhubbard_b200 import _lib

    for _ in range(warmup):
        state(spins)
    torch.cuda.synchronize()
    if profile:
        _lib.profile_read()
        _lib.profile_enable(True)
    ev = []
    for _ in range(steps):
        flush.fill_(1)  # evict L2 between steps (not timed)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        state(spins)
        e1.record(st)
        ev.append((e0, e1))
    torch.cuda.synchronize()
    kern = {}
    if profile:
        _lib.profile_enable(False)
        kern = _lib.profile_read()
    return sum(a.elapsed_time(b) for a, b in ev), kern


def run_chains(smp, steps, st):
    """``steps`` Metropolis steps, one call each, recording log|psi| of every chain; returns
    (log|psi| series (steps, B) on the host, device milliseconds, acceptance)."""
    import torch

    B = smp.nsamples
    series = torch.empty((steps, B), dtype=torch.float64, device=smp.spins.device)
    a0 = int(smp.accepted.sum().item())
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for t in range(steps):
        smp.run(1)
        series[t].copy_(smp.psi.logabs)
    e1.record(st)
    torch.cuda.synchronize()
    acc = (int(smp.accepted.sum().item()) - a0) / (B * steps)
    return series.cpu().numpy(), e0.elapsed_time(e1), acc


def measure_sampling(args, dev, st, seed) -> dict:
    """Effective samples/s of the plain form (FP32 CNN, uniform-hop sampler) and the chosen form
    (tcgen05 BF16x3 CNN, learned proposal trained on 2^20 records of plain chains), plus the
    chosen amplitudes under the uniform-hop sampler and under the reference's MixSampler (hop and
    site-exchange chains, half each).  All chains start from the same
    configurations, equilibrated by ``burn`` plain steps; tau_int is that of the log|psi| series
    over the ``steps`` measured steps; energies per site from the final configurations."""
    import torch

    import neuralhubbard_b200 as nh
    from neuralhubbard_b200 import stats

    B, steps, burn = args.chains, args.sampler_steps, args.burn
    params = nh.init_params(L, L, CHANNELS, LAYERS, std=0.02, seed=0)
    forms = {
        "plain": nh.PfaffianBackflow(L, L, NE, NE, params=params, device=dev, cnn_mode=0),
        "chosen": nh.PfaffianBackflow(L, L, NE, NE, params=params, device=dev, cnn_mode=2,
                                      pf_mode=args.pf_mode),
    }
    states = {k: nh.Variational(m, symm=True, max_parallel=8192) for k, m in forms.items()}
    init = nh.random_spins(np.random.default_rng(seed), B, N_SITES, NE, NE)
    eq = nh.ParticleHop(states["chosen"], B, n_neighbor=(1, 2), initial_spins=init, seed=seed)
    n_snap = min(burn, max(1, (1 << 20) // B))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    eq.run(burn - n_snap)
    snaps = []
    for _ in range(n_snap):  # training records: the chains' last 2^20 / B configurations
        eq.run(1)
        snaps.append(eq.spins.clone())
    torch.cuda.synchronize()
    t_burn = time.perf_counter() - t0
    start = eq.spins.clone()
    t0 = time.perf_counter()
    rec = nh.training_records(states["chosen"], torch.cat(snaps), seed=seed + 2,
                              weight="barker")
    torch.cuda.synchronize()
    t_rec = time.perf_counter() - t0
    del snaps
    q = nh.HopProposal(L, L, 8, seed=seed + 3, std=0.05, device=dev)
    t0 = time.perf_counter()
    losses = q.train(rec, args.train_steps, batch=512, lr=3e-3, seed=seed + 4)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    train = {"records": int(rec[0].shape[0]), "steps": args.train_steps, "batch": 512,
             "target": "barker r/(1+r)", "record_seconds": t_rec, "train_seconds": t_train,
             "loss_first": float(np.mean(losses[:20])), "loss_last": float(np.mean(losses[-20:]))}
    del rec

    out = {}
    H = nh.Hubbard(8.0, [1.0, -0.2], [1, 2])
    ne = min(B, args.energy_samples)
    runs = [("plain", "plain", lambda s: nh.ParticleHop(states["plain"], B, n_neighbor=(1, 2),
                                                        initial_spins=s, seed=seed + 5)),
            ("chosen", "chosen", lambda s: nh.LearnedHop(states["chosen"], B, q,
                                                         initial_spins=s, seed=seed + 6)),
            ("chosen_uniform_hop", "chosen",
             lambda s: nh.ParticleHop(states["chosen"], B, n_neighbor=(1, 2), initial_spins=s,
                                      seed=seed + 7)),
            # the reference's own sampler: MixSampler of hop and site-exchange chains, half each
            ("chosen_mix", "chosen",
             lambda s: nh.MixSampler([nh.ParticleHop(states["chosen"], B // 2, n_neighbor=(1, 2)),
                                      nh.SiteExchange(states["chosen"], B - B // 2,
                                                      n_neighbor=(1, 2))],
                                     initial_spins=s, seed=seed + 8))]
    for name, form, make in runs:
        smp = make(start)
        series, ms, acc = run_chains(smp, steps, st)
        te = stats.tau_int_error(series)
        tau = te["tau"]
        err = te["err_groups"] if te["err_groups"] is not None else te["err_sokal"]
        rate = stats.effective_rate(B, steps, tau, ms / 1e3)
        e = H.Oloc(states[form], nh.Samples(smp.spins[:ne].contiguous(), smp.psi[:ne]))
        e = e.cpu().numpy() / N_SITES
        out[name] = {"acceptance": acc, "tau_int_logpsi": tau, "tau_int_logpsi_err": err,
                     "tau_int_logpsi_err_sokal": te["err_sokal"], "tau_window": te["window"],
                     "ms_per_step": ms / steps, "effective_samples_per_s": rate,
                     "effective_samples_per_s_err": rate * err / tau,
                     "energy_per_site": float(e.mean()),
                     "energy_per_site_err": float(e.std(ddof=1) / np.sqrt(ne))}
        del smp
    out["chosen"]["proposal_training"] = train
    out["_proposal"] = q
    d = out["chosen"]["energy_per_site"] - out["plain"]["energy_per_site"]
    sig = float(np.hypot(out["chosen"]["energy_per_site_err"], out["plain"]["energy_per_site_err"]))
    out["energy_difference_sigma"] = abs(d) / sig if sig > 0 else None
    out["chosen_vs_plain"] = (out["chosen"]["effective_samples_per_s"]
                              / out["plain"]["effective_samples_per_s"])
    out["chosen_uniform_hop_vs_plain"] = (out["chosen_uniform_hop"]["effective_samples_per_s"]
                                          / out["plain"]["effective_samples_per_s"])
    out["chosen_mix_vs_plain"] = (out["chosen_mix"]["effective_samples_per_s"]
                                  / out["plain"]["effective_samples_per_s"])
    out["setup"] = {"chains": B, "burn_in_steps": burn, "burn_in_seconds": t_burn,
                    "measured_steps": steps,
                    "start": "all runs from the same configurations after the burn-in",
                    "tau_convention": "Sokal tau = 1/2 + sum rho (window c = 5); effective = "
                                      "B steps / (2 tau seconds); tau error = spread of tau over "
                                      "8 disjoint sets of chains / sqrt(8) (Sokal's variance "
                                      "formula beside it)",
                    "energy_samples": ne, "seconds_are": "CUDA-event time of the measured steps"}
    return out


def measure_local_energy(args, dev, st) -> dict:
    """Ragged local energy (unprojected amplitudes, CUDA-core Pfaffian; FP32 CNN, and at 16x16
    also the tcgen05 BF16x3 CNN) of ``eloc_samples`` configurations per lattice: the chunk size
    is tuned on 256 of them, then one call is recorded in a CUDA graph and its replay timed with
    CUDA events."""
    import torch

    import neuralhubbard_b200 as nh

    out = {}
    H = nh.Hubbard(8.0, [1.0, -0.2], [1, 2])
    for Lk, cnn_mode in ((8, 0), (16, 0), (16, 2), (24, 0)):
        Nk = Lk * Lk
        nek = 7 * Nk // 16
        params = nh.init_params(Lk, Lk, CHANNELS, LAYERS, std=0.02, seed=0)
        model = nh.PfaffianBackflow(Lk, Lk, nek, nek, params=params, device=dev,
                                    cnn_mode=cnn_mode)
        state = nh.Variational(model, symm=False, max_parallel=8192)
        B = args.eloc_samples if Lk <= 16 else args.eloc_samples_large
        spins = torch.from_numpy(nh.random_spins(np.random.default_rng(500 + Lk), B, Nk, nek,
                                                 nek)).to(dev)
        psi = state(spins)
        sub = nh.Samples(spins[:256].contiguous(), psi[:256])
        chunk = H.autotune(state, sub, candidates=(0, 4096, 16384, 65536), repeats=1)
        counts = H.hop_list(spins, Lk, Lk)[0]
        n_conn = int(counts.sum().item())
        samples = nh.Samples(spins, psi)
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            H.Oloc(state, nh.Samples(spins[:64].contiguous(), psi[:64]), chunk_configs=chunk,
                   count_connections=False)
        torch.cuda.current_stream().wait_stream(side)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            e = H.Oloc(state, samples, chunk_configs=chunk, count_connections=False)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        graph.replay()
        e1.record(st)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        ev = e.cpu().numpy() / Nk
        out[f"{Lk}x{Lk}" + ("" if cnn_mode == 0 else " tcgen05 BF16x3 CNN")] = {
            "samples": B, "connections": n_conn, "pfaffian_n": 2 * nek, "chunk_configs": chunk,
            "ms": ms, "samples_per_s": B / (ms / 1e3),
            "amplitudes_per_s": n_conn / (ms / 1e3),
            "energy_per_site": float(ev.mean()),
            "energy_per_site_err": float(ev.std(ddof=1) / np.sqrt(B))}
        del graph, e, state, model
        torch.cuda.empty_cache()
    out["setup"] = ("4096 uniformly random configurations at 8x8 and 16x16, 256 at 24x24 (n = "
                    "504, large-lattice path: 40 ms of amplitudes per sample), unprojected "
                    "amplitudes, t = 1, t' = -0.2, U = 8; one CUDA-graph replay of the whole call")
    return out


def measure_config1(args, dev, st) -> dict:
    """Config 1: 8x8 lattice (Pfaffians of 56 x 56), 1024 seeded configurations, no symmetry
    projection: log|psi|, sign and local energy (U = 8, t' = -0.2).  GPU: one amplitude call and
    one local-energy call per step, CUDA events, 3 steps after a warm-up.  CPU: the compiled
    restatement (FP32 build, all host cores) on a bounded sample of the same configurations,
    amplitudes of the samples and of every connected configuration; its local energies are
    compared with the GPU's on that sample."""
    import torch

    import neuralhubbard_b200 as nh
    from oracle import hubbard as ohub
    from oracle import port

    Lk, B = 8, 1024
    Nk = Lk * Lk
    nek = 7 * Nk // 16
    params = nh.init_params(Lk, Lk, CHANNELS, LAYERS, std=0.02, seed=0)
    state = nh.Variational(nh.PfaffianBackflow(Lk, Lk, nek, nek, params=params, device=dev),
                           symm=False, max_parallel=B)
    H = nh.Hubbard(8.0, [1.0, -0.2], [1, 2])
    s_np = nh.random_spins(np.random.default_rng(11), B, Nk, nek, nek)
    s = torch.from_numpy(s_np).to(dev)
    e = H.Oloc(state, nh.Samples(s, state(s)), count_connections=False)
    torch.cuda.synchronize()
    ev = []
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        psi = state(s)
        e = H.Oloc(state, nh.Samples(s, psi), count_connections=False)
        e1.record(st)
        ev.append((e0, e1))
    torch.cuda.synchronize()
    ms = sum(a.elapsed_time(b) for a, b in ev) / len(ev)
    e_gpu = e.cpu().numpy()
    out = {"lattice": "8x8", "configurations": B, "projected": False,
           "gpu_ms_per_call": ms, "gpu_samples_per_s": B / (ms / 1e3),
           "E_per_site": float(e_gpu.mean() / Nk)}
    try:
        cores = len(os.sched_getaffinity(0))
    except Exception:
        cores = os.cpu_count() or 1
    hp = dict(conv_w=[w.astype(np.float64) for w in params["conv_w"]],
              conv_b=[b.astype(np.float64) for b in params["conv_b"]],
              W=params["W"].astype(np.float64), theta=float(params["theta"]), Lx=Lk, Ly=Lk)
    amp = lambda c: port.projected_amplitude(c, hp, symm=False, threads=cores, fp32=True)  # noqa
    n_cpu = 16
    t0 = time.perf_counter()
    e_cpu = ohub.local_energy(s_np[:n_cpu], amp, Lk, Lk, 1.0, -0.2, 8.0)
    wall = time.perf_counter() - t0
    rate = n_cpu / wall
    out["cpu"] = {"samples_per_s": rate, "cores": cores, "kind": "port (FP32 build)",
                  "sample": f"{n_cpu} of the configurations ({wall:.1f} s)"}
    out["gpu_over_cpu"] = out["gpu_samples_per_s"] / rate
    out["eloc_max_rel_diff_vs_cpu_fp32"] = float(
        np.max(np.abs(e_gpu[:n_cpu] - e_cpu) / np.maximum(1.0, np.abs(e_cpu))))
    return out


def _err_stats(la, l0, sg, s0) -> dict:
    e = np.abs(la - l0)
    return {"max": float(e.max()), "p99.9": float(np.quantile(e, 0.999)),
            "p99": float(np.quantile(e, 0.99)), "mean": float(e.mean()),
            "count_above_1e-4": int((e > 1e-4).sum()), "sign_mismatches": int((sg != s0).sum())}


def measure_precision(dev, st, spins, flush) -> dict:
    """Config 3: |delta log|psi_P|| and sign mismatches against the all-FP64 path for each
    precision form on the benchmark's 8192 configurations (projected), with each form's step
    time; and the log-Pfaffian of 8192 FP32 matrices of 224 x 224, 1% of them near-nodal (one
    pivot 1e-6 of the others), against FP64 factorisation of the same matrices."""
    import torch

    import neuralhubbard_b200 as nh

    params = nh.init_params(L, L, CHANNELS, LAYERS, std=0.02, seed=0)
    forms = [("all FP64 (cond_tau 1, reference)", dict(cnn_mode=0, cond_tau=1.0)),
             ("plain (defaults): FP32 CNN; FP64 features + static-pivot FP64 refinement of "
              "images with |share| x pivot ratio > 5 and of cancelling configurations",
              dict(cnn_mode=0)),
             ("chosen (defaults): tcgen05 BF16x3 CNN, same policy", dict(cnn_mode=2)),
             ("tcgen05 BF16x3 CNN, threshold 10", dict(cnn_mode=2, cond_tau=10.0)),
             ("tcgen05 BF16x3 CNN, threshold 5 + FP32-block refinement of every image",
              dict(cnn_mode=2, refine_tau=1.0)),
             ("tcgen05 BF16x3 CNN, no FP64 work", dict(cnn_mode=2, cond_tau=0.0,
                                                       cancel_tau=0.0)),
             ("tcgen05 CNN + tensor-memory 3xTF32 Pfaffian (pf_mode 1)",
              dict(cnn_mode=2, pf_mode=1))]
    out = {}
    ref = None
    for name, kw in forms:
        model = nh.PfaffianBackflow(L, L, NE, NE, params=params, device=dev, **kw)
        state = nh.Variational(model, symm=True, max_parallel=BATCH)
        ms, _ = time_amplitudes(state, spins, 3, 1, flush, st)
        psi = state(spins)
        sg, la = psi.sign.cpu().numpy(), psi.logabs.cpu().numpy()
        fl = psi.flags.cpu().numpy()
        if ref is None:
            ref = (sg, la)
        out[name] = {"amplitudes_per_s": BATCH * IMAGES / (ms / 3 / 1e3),
                     "refined_configurations": float(((fl & 8) != 0).mean()),
                     **_err_stats(la, ref[1], sg, ref[0])}
        del model, state, psi
    # near-nodal pairing matrices at the slogpf boundary
    g = torch.Generator(device=dev)
    g.manual_seed(3)
    B, n = 8192, N_OCC
    A = torch.randn((B, n, n), generator=g, device=dev)
    A = A - A.transpose(1, 2)
    nn_idx = torch.arange(0, B, 100, device=dev)  # 1% near-nodal
    Q, _ = torch.linalg.qr(torch.randn((len(nn_idx), n, n), generator=g, device=dev,
                                       dtype=torch.float64))
    a = (torch.rand((len(nn_idx), n // 2), generator=g, device=dev, dtype=torch.float64) * 1.5
         + 0.5) * torch.where(torch.rand((len(nn_idx), n // 2), generator=g, device=dev) < 0.5,
                              -1.0, 1.0).double()
    a[:, 7] *= 1e-6
    Bm = torch.zeros((len(nn_idx), n, n), dtype=torch.float64, device=dev)
    k = torch.arange(n // 2, device=dev)
    Bm[:, 2 * k, 2 * k + 1] = a
    Bm[:, 2 * k + 1, 2 * k] = -a
    An = Q.transpose(1, 2) @ Bm @ Q
    A[nn_idx] = (0.5 * (An - An.transpose(1, 2))).float()
    s0, l0, _ = nh.slogpf(A, cond_tau=1.0)
    s1, l1, f1 = nh.slogpf(A)
    s2, l2, _ = nh.slogpf(A, cond_tau=0.0)
    refined = (f1.cpu().numpy() & 8) != 0
    near = np.zeros(B, bool)
    near[nn_idx.cpu().numpy()] = True
    out["near-nodal slogpf, 8192 x 224x224 (1% seeded, pivot 1e-6)"] = {
        "default (FP64 refinement of pivot ratio > 5)":
            _err_stats(l1.cpu().numpy(), l0.cpu().numpy(), s1.cpu().numpy(), s0.cpu().numpy()),
        "FP32 only": _err_stats(l2.cpu().numpy(), l0.cpu().numpy(), s2.cpu().numpy(),
                                s0.cpu().numpy()),
        "near-nodal refined": int(refined[near].sum()), "near-nodal": int(near.sum()),
        "refined fraction": float(refined.mean())}
    del A
    torch.cuda.empty_cache()
    out["reference"] = ("all-FP64 path of the library (FP64 CNN, gather and Pfaffian), which "
                        "matches the numpy oracle to 1e-9 in the parity tests")
    return out


def measure_extensions(args, dev, st, spins, flush) -> dict:
    """The rows beyond the amplitude: the per-sample Jacobian of log|psi_P| (16x16, 1024
    configurations x 8 images, benchmark weights), the BCS-backflow ansatz on the benchmark's
    8192 configurations x 8 images (throughput of the chosen CNN form, and its |delta log|psi_P||
    against the BCS all-FP64 form), and the packed observables (transverse spin at one
    reference site, the d-wave F and G families at R = (0, 0)) on 1024 configurations."""
    import torch

    import neuralhubbard_b200 as nh
    from neuralhubbard_b200 import _lib
    from neuralhubbard_b200.observables import PackedDwave, transverse_terms

    out = {}
    params = nh.init_params(L, L, CHANNELS, LAYERS, std=0.02, seed=0)
    model = nh.PfaffianBackflow(L, L, NE, NE, params=params, device=dev)
    state = nh.Variational(model, symm=True, max_parallel=1024)
    sj = spins[:1024]
    state.jacobian(sj)
    torch.cuda.synchronize()
    _lib.profile_read()
    _lib.profile_enable(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(2):
        psi, J = state.jacobian(sj)
    e1.record(st)
    torch.cuda.synchronize()
    _lib.profile_enable(False)
    kern = _lib.profile_read()
    ms = e0.elapsed_time(e1) / 2
    out["jacobian"] = {"lattice": "16x16", "configurations": 1024, "images": 8,
                       "parameters": int(J.shape[1]), "ms_per_call": ms,
                       "samples_per_s": 1024 / (ms / 1e3),
                       "kernels_ms_per_call": {k: v[0] / 2 for k, v in kern.items()}}
    del J, psi
    # BCS ansatz
    bp = dict(params)
    bp["W"] = params["W"][0]
    bp["delta_d"] = 0.1
    bcs = {}
    ref = None
    for name, kw in (("all FP64 (cond_tau 1, reference)", dict(cond_tau=1.0)),
                     ("chosen (defaults): tcgen05 BF16x3 CNN", dict(cnn_mode=2)),
                     ("plain (defaults): FP32 CNN", dict(cnn_mode=0))):
        m = nh.BCSBackflow(L, L, NE, NE, params=bp, device=dev, **kw)
        sb = nh.Variational(m, symm=True, max_parallel=BATCH)
        bms, bk = time_amplitudes(sb, spins, 3, 1, flush, st, True)
        ps = sb(spins)
        sg, la = ps.sign.cpu().numpy(), ps.logabs.cpu().numpy()
        if ref is None:
            ref = (sg, la)
        bcs[name] = {"amplitudes_per_s": BATCH * IMAGES / (bms / 3 / 1e3),
                     "kernels_ms_per_step": {k: v[0] / 3 for k, v in bk.items()},
                     **_err_stats(la, ref[1], sg, ref[0])}
        del m, sb, ps
    out["bcs"] = {"lattice": "16x16", "configurations": BATCH, "images": IMAGES,
                  "n_up x n_dn": f"{NE} x {NE}", "delta_d": 0.1, "forms": bcs}
    # packed observables
    so = spins[:1024]
    samples = nh.Samples(so, state(so))
    transverse_terms(state, samples, (0, 0))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    T = transverse_terms(state, samples, (0, 0))
    torch.cuda.synchronize()
    t_tr = time.perf_counter() - t0
    dw = PackedDwave(L, L, R=(0, 0))
    t0 = time.perf_counter()
    F, G = dw.measure(state, samples)
    t_dw = time.perf_counter() - t0
    out["observables"] = {
        "lattice": "16x16", "configurations": 1024, "projected": True,
        "transverse_spin_s": t_tr, "transverse_terms": int(T.numel()),
        "dwave_s": t_dw, "dwave_F_terms": len(F), "dwave_G_terms": len(G),
        "sum_rule_Sz0": float(T[0, 0].item() + T[1, 0].item()),
        "note": "wall-clock seconds of one call each (each call reads its connection count back "
                "once); the terms' connections run through the amplitude pipeline"}
    return out


def measure_large(args, dev, st, q) -> dict:
    """Config 5 shapes: Metropolis at 32x32 (n = 896, large-lattice path) with 4096 chains x 8
    images, uniform hop against the learned proposal (the 16x16-trained weights: the proposal
    network is translation-equivariant); one untimed and ``large_steps`` timed steps each."""
    import torch

    import neuralhubbard_b200 as nh

    Lk, B = 32, args.large_chains
    Nk = Lk * Lk
    nek = 7 * Nk // 16
    params = nh.init_params(Lk, Lk, CHANNELS, LAYERS, std=0.02, seed=0)
    model = nh.PfaffianBackflow(Lk, Lk, nek, nek, params=params, device=dev)
    state = nh.Variational(model, symm=True, max_parallel=8192)
    init = nh.random_spins(np.random.default_rng(31), B, Nk, nek, nek)
    out = {"lattice": "32x32", "pfaffian_n": 2 * nek, "chains": B, "images": IMAGES,
           "timed_steps": args.large_steps}
    q32 = None
    if q is not None:
        q32 = nh.HopProposal(Lk, Lk, 8, params=q.numpy(), device=dev)
    for name, make in (("uniform_hop", lambda: nh.ParticleHop(state, B, n_neighbor=(1, 2),
                                                              initial_spins=init, seed=32)),
                       ("learned", lambda: nh.LearnedHop(state, B, q32, initial_spins=init,
                                                         seed=33) if q32 else None)):
        smp = make()
        if smp is None:
            continue
        smp.run(1)
        a0 = int(smp.accepted.sum().item())
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        smp.run(args.large_steps)
        e1.record(st)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.large_steps
        out[name] = {"ms_per_step": ms,
                     "acceptance": (int(smp.accepted.sum().item()) - a0) / (B * args.large_steps)}
        del smp
    t = torch.from_numpy(init[:512]).to(dev)
    state(t)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(st)
    state(t)
    e1.record(st)
    torch.cuda.synchronize()
    out["amplitudes_per_s"] = 512 * IMAGES / (e0.elapsed_time(e1) / 1e3)
    out["note"] = ("tau_int is not measured at 32x32 within the bench (about 2.4 s per step with "
                   "4096 chains); the proposal is trained at 16x16 (its backward kernel holds "
                   "the activations of up to 559 sites in shared memory) and transferred")
    return out


def measure_config5(args, dev, st) -> dict:
    """Config 5 at 32x32 (n = 896): the learned proposal trained at 32x32 on records of plain
    chains, against the uniform hop.  Reduced from the stated 4096 chains, 2^20 records and a
    tau_int over >= 50 tau to what one GPU does in minutes (a projected 32x32 amplitude costs
    ~0.7 ms): ``c5_chains`` chains equilibrated by ``c5_burn`` plain steps, ``c5_records``
    training records (Barker weight) from their last configurations, 2000 Adam steps, then
    ``c5_steps`` measured steps per sampler from the same start; tau_int of log|psi| with its
    chain-group error, effective samples/s, and E/N on 16 final configurations each."""
    import torch

    import neuralhubbard_b200 as nh
    from neuralhubbard_b200 import stats

    Lk = 32
    Nk = Lk * Lk
    nek = 7 * Nk // 16
    B, burn, steps = args.c5_chains, args.c5_burn, args.c5_steps
    params = nh.init_params(Lk, Lk, CHANNELS, LAYERS, std=0.02, seed=0)
    model = nh.PfaffianBackflow(Lk, Lk, nek, nek, params=params, device=dev)
    state = nh.Variational(model, symm=True, max_parallel=4096)
    init = nh.random_spins(np.random.default_rng(51), B, Nk, nek, nek)
    eq = nh.ParticleHop(state, B, n_neighbor=(1, 2), initial_spins=init, seed=52)
    n_snap = max(1, min(burn, args.c5_records // B))
    t0 = time.perf_counter()
    eq.run(burn - n_snap)
    snaps = []
    for _ in range(n_snap):
        eq.run(1)
        snaps.append(eq.spins.clone())
    torch.cuda.synchronize()
    t_burn = time.perf_counter() - t0
    start = eq.spins.clone()
    t0 = time.perf_counter()
    rec = nh.training_records(state, torch.cat(snaps), seed=53, weight="barker")
    torch.cuda.synchronize()
    t_rec = time.perf_counter() - t0
    del snaps
    q = nh.HopProposal(Lk, Lk, 8, seed=54, std=0.05, device=dev)
    t0 = time.perf_counter()
    losses = q.train(rec, args.train_steps, batch=512, lr=3e-3, seed=55)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    out = {"lattice": "32x32", "pfaffian_n": 2 * nek, "chains": B, "burn_in_steps": burn,
           "burn_in_seconds": t_burn, "measured_steps": steps,
           "proposal_training": {"records": int(rec[0].shape[0]), "steps": args.train_steps,
                                 "batch": 512, "target": "barker r/(1+r)",
                                 "record_seconds": t_rec, "train_seconds": t_train,
                                 "loss_first": float(np.mean(losses[:20])),
                                 "loss_last": float(np.mean(losses[-20:]))}}
    del rec
    H = nh.Hubbard(8.0, [1.0, -0.2], [1, 2])
    for name, make in (("uniform_hop", lambda: nh.ParticleHop(state, B, n_neighbor=(1, 2),
                                                              initial_spins=start, seed=56)),
                       ("learned", lambda: nh.LearnedHop(state, B, q, initial_spins=start,
                                                         seed=57))):
        smp = make()
        series, ms, acc = run_chains(smp, steps, st)
        te = stats.tau_int_error(series)
        tau = te["tau"]
        err = te["err_groups"] if te["err_groups"] is not None else te["err_sokal"]
        rate = stats.effective_rate(B, steps, tau, ms / 1e3)
        e = H.Oloc(state, nh.Samples(smp.spins[:16].contiguous(), smp.psi[:16]))
        e = e.cpu().numpy() / Nk
        out[name] = {"acceptance": acc, "tau_int_logpsi": tau, "tau_int_logpsi_err": err,
                     "tau_window": te["window"], "ms_per_step": ms / steps,
                     "effective_samples_per_s": rate,
                     "effective_samples_per_s_err": rate * err / tau,
                     "energy_per_site": float(e.mean()),
                     "energy_per_site_err": float(e.std(ddof=1) / np.sqrt(16))}
        del smp
    out["learned_vs_uniform"] = (out["learned"]["effective_samples_per_s"]
                                 / out["uniform_hop"]["effective_samples_per_s"])
    return out


def measure_resconv(args, dev, st) -> dict:
    """The released states' residual network (16 blocks x 64 channels, d = 32) at 16x16: projected
    amplitudes of 1024 configurations x 8 images on CUDA cores (FP32) and on the tensor cores
    (BF16 x3), each against the all-FP64 path; with the released tpm02_L16_pfaffian weights
    (tests/golden/released/, copied by tests/golden/fetch_released.py) the configurations are
    its stored chains and E/N on 512 of them is measured with the tensor-core form."""
    import torch

    import neuralhubbard_b200 as nh
    from neuralhubbard_b200 import _lib, checkpoint

    here = os.path.dirname(os.path.abspath(__file__))
    eqx = os.path.join(here, "tests", "golden", "released", "tpm02_L16_pfaffian.eqx")
    ne = 7 * N_SITES // 16
    released = os.path.exists(eqx)
    if released:
        params = checkpoint.load_pfaffian_backflow(
            eqx, L, expect_md5=checkpoint.RELEASED["tpm02_L16_pfaffian"].md5)
        spins = checkpoint.load_spins(eqx.replace(".eqx", "_spins.npz"), N_SITES, NE, NE)
    else:
        rng = np.random.default_rng(61)
        params = dict(net="resconv", embed=rng.normal(size=(64, 4)).astype(np.float32),
                      conv_w=[(rng.normal(size=(64, 64, 3, 3)) * 0.04).astype(np.float32)
                              for _ in range(32)],
                      conv_b=[(rng.normal(size=64) * 0.1).astype(np.float32) for _ in range(32)],
                      W=(rng.normal(size=(3, N_SITES, 32)) / np.sqrt(32)).astype(np.float32),
                      theta=0.55)
        spins = nh.random_spins(np.random.default_rng(62), 1024, N_SITES, ne, ne)
    B = 1024
    s = torch.from_numpy(spins[:B]).to(dev)
    ref = nh.Variational(nh.PfaffianBackflow(L, L, ne, ne, params=params, cond_tau=1.0,
                                             device=dev))(s)
    out = {"weights": "released tpm02_L16_pfaffian" if released else "random (LeCun-sized)",
           "network": "16 residual blocks x 64 channels, d = 32 (code/backflow/models.py:319-329)",
           "configurations": B, "images": IMAGES,
           "reference_a100_us_per_amplitude": {
               "cnn_tf32": 16.0, "pfaffian_3xtf32_n256": 3.39,
               "source": "data/supplement/tableS3_amplitude_cost/amplitude_cost.csv rows "
                         "'16,256,Normal CNN' and '16,256,Pfaffian' (A100, half filling)"}}
    for name, mode in (("cuda_cores_fp32", 0), ("tensor_cores_bf16x3", 2)):
        state = nh.Variational(nh.PfaffianBackflow(L, L, ne, ne, params=params, cnn_mode=mode,
                                                   device=dev))
        for _ in range(2):
            state(s)
        torch.cuda.synchronize()
        _lib.profile_enable(True)
        _lib.profile_read()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        psi = state(s)
        e1.record(st)
        torch.cuda.synchronize()
        kern = _lib.profile_read()
        _lib.profile_enable(False)
        d = (psi.logabs - ref.logabs).abs().cpu().numpy()
        out[name] = {"amplitudes_per_s": B * IMAGES / (e0.elapsed_time(e1) / 1e3),
                     "kernels_ms": {k: v[0] for k, v in kern.items()},
                     "max_abs_dlog": float(d.max()), "mean_abs_dlog": float(d.mean()),
                     "sign_mismatches": int((psi.sign != ref.sign).sum().item())}
    if released:
        info = checkpoint.RELEASED["tpm02_L16_pfaffian"]
        state = nh.Variational(nh.PfaffianBackflow(L, L, ne, ne, params=params, cnn_mode=2,
                                                   device=dev))
        H = nh.Hubbard(8.0, [1.0, info.tprime], [1, 2])
        sc = torch.from_numpy(spins[1024:1536]).to(dev)
        t0 = time.time()
        e = H.Oloc(state, nh.Samples(sc, state(sc))).cpu().numpy() / N_SITES
        out["energy"] = {"chains": 512, "E_per_site": float(e.mean()),
                         "E_per_site_err": float(e.std(ddof=1) / math.sqrt(len(e))),
                         "published": info.energy, "published_err": info.energy_err,
                         "seconds": time.time() - t0}
    return out


def measure_released_sampling(args, dev, st) -> dict:
    """Sampling on a physical state: the released tpm02_L16_pfaffian (tensor-core residual
    network) with the uniform hop and with the learned proposal trained on records drawn from the
    released equilibrated chains (spins 1024..8191, ``released_repeats`` moves each, Barker
    weight).  Both runs start from the stored chains 0..B-1 (already equilibrated under the
    projected state) and measure ``released_steps`` steps: acceptance, tau_int of log|psi|,
    effective samples/s and E/N on ``energy_samples`` final configurations."""
    import torch

    import neuralhubbard_b200 as nh
    from neuralhubbard_b200 import checkpoint, stats

    here = os.path.dirname(os.path.abspath(__file__))
    eqx = os.path.join(here, "tests", "golden", "released", "tpm02_L16_pfaffian.eqx")
    if not os.path.exists(eqx):
        return {"skipped": "released weights not fetched (tests/golden/fetch_released.py)"}
    params = checkpoint.load_pfaffian_backflow(
        eqx, L, expect_md5=checkpoint.RELEASED["tpm02_L16_pfaffian"].md5)
    spins = checkpoint.load_spins(eqx.replace(".eqx", "_spins.npz"), N_SITES, NE, NE)
    info = checkpoint.RELEASED["tpm02_L16_pfaffian"]
    ne = 7 * N_SITES // 16
    state = nh.Variational(nh.PfaffianBackflow(L, L, ne, ne, params=params, cnn_mode=2,
                                               device=dev), symm=True)
    B, steps = args.chains, args.released_steps
    pool = torch.from_numpy(spins[B:]).to(dev)
    t0 = time.perf_counter()
    psi_pool = state(pool)
    recs = [nh.training_records(state, pool, psi=psi_pool, seed=900 + r, weight="barker")
            for r in range(args.released_repeats)]
    rec = tuple(torch.cat([r[i] for r in recs]) for i in range(len(recs[0])))
    torch.cuda.synchronize()
    t_rec = time.perf_counter() - t0
    q = nh.HopProposal(L, L, 8, seed=901, std=0.05, device=dev)
    t0 = time.perf_counter()
    losses = q.train(rec, args.train_steps, batch=512, lr=3e-3, seed=902)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    out = {"state": "tpm02_L16_pfaffian (released), tensor-core residual network",
           "chains": B, "measured_steps": steps,
           "proposal_training": {"records": int(rec[0].shape[0]), "steps": args.train_steps,
                                 "record_seconds": t_rec, "train_seconds": t_train,
                                 "loss_first": float(np.mean(losses[:20])),
                                 "loss_last": float(np.mean(losses[-20:]))}}
    del rec, recs
    H = nh.Hubbard(8.0, [1.0, info.tprime], [1, 2])
    n_e = min(B, args.energy_samples)
    start = torch.from_numpy(spins[:B]).to(dev)
    for name, make in (("uniform_hop", lambda: nh.ParticleHop(state, B, n_neighbor=(1, 2),
                                                              initial_spins=start, seed=903)),
                       ("learned", lambda: nh.LearnedHop(state, B, q, initial_spins=start,
                                                         seed=904))):
        smp = make()
        series, ms, acc = run_chains(smp, steps, st)
        tau = stats.tau_int(series)
        e = H.Oloc(state, nh.Samples(smp.spins[:n_e].contiguous(), smp.psi[:n_e]))
        e = e.cpu().numpy() / N_SITES
        out[name] = {"acceptance": acc, "tau_int_logpsi": tau, "ms_per_step": ms / steps,
                     "effective_samples_per_s": stats.effective_rate(B, steps, tau, ms / 1e3),
                     "energy_per_site": float(e.mean()),
                     "energy_per_site_err": float(e.std(ddof=1) / np.sqrt(n_e))}
        del smp
    out["learned_vs_uniform"] = (out["learned"]["effective_samples_per_s"]
                                 / out["uniform_hop"]["effective_samples_per_s"])
    out["published_energy_per_site"] = info.energy
    return out


def run_ours(args) -> None:
    import torch
    import torch.distributed as dist

    import neuralhubbard_b200 as nh
    from neuralhubbard_b200.distributed import init_from_env

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    multi = init_from_env("nccl") if world > 1 else False

    params = nh.init_params(L, L, CHANNELS, LAYERS, std=0.02, seed=0)
    model = nh.PfaffianBackflow(L, L, NE, NE, params=params, device=dev, cnn_mode=args.cnn_mode,
                                pf_mode=args.pf_mode)
    state = nh.Variational(model, symm=True, max_parallel=BATCH)
    rng = np.random.default_rng(1000 + rank)
    spins_host = torch.from_numpy(nh.random_spins(rng, BATCH, N_SITES, NE, NE)).pin_memory()
    spins = spins_host.to(dev)
    flush = torch.empty(512 * 1024 * 1024, dtype=torch.uint8, device=dev)
    st = torch.cuda.current_stream(dev)

    clocks = ClockSampler(local)
    clocks.start()
    if multi:
        dist.barrier()
    total_ms, kern = time_amplitudes(state, spins, args.steps, args.warmup, flush, st, True)
    if multi:
        dist.barrier()
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    if multi:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    n_amp = world * BATCH * IMAGES * args.steps
    value = n_amp / (total_ms / 1e3)

    # the plain FP32 form on the same inputs (reported beside the chosen form)
    plain = None
    if args.cnn_mode != 0 or args.pf_mode != 0:
        m0 = nh.PfaffianBackflow(L, L, NE, NE, params=params, device=dev, cnn_mode=0)
        s0 = nh.Variational(m0, symm=True, max_parallel=BATCH)
        p_ms, p_kern = time_amplitudes(s0, spins, args.steps, args.warmup, flush, st, True)
        tp = torch.tensor([p_ms], dtype=torch.float64, device=dev)
        if multi:
            dist.all_reduce(tp, op=dist.ReduceOp.MAX)
        p_ms = float(tp.item())
        plain = {"value": n_amp / (p_ms / 1e3), "ms_per_step": p_ms / args.steps,
                 "form": "FP32 CUDA-core CNN, CUDA-core Pfaffian",
                 "kernels": {k: {"ms_per_step": v[0] / args.steps, "launches": v[1]}
                             for k, v in p_kern.items()}}
        del m0, s0

    # e2e: public API, configurations from pinned host memory, amplitudes back to the host
    sign_h = torch.empty(BATCH, dtype=torch.float32).pin_memory()
    logabs_h = torch.empty(BATCH, dtype=torch.float64).pin_memory()
    e2e_ms = []
    for _ in range(max(2, args.steps // 2)):
        flush.fill_(1)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        psi = state(spins_host)
        sign_h.copy_(psi.sign, non_blocking=True)
        logabs_h.copy_(psi.logabs, non_blocking=True)
        e1.record(st)
        e2e_ms.append((e0, e1))
    torch.cuda.synchronize(dev)
    e2e_total = sum(a.elapsed_time(b) for a, b in e2e_ms)
    te = torch.tensor([e2e_total], dtype=torch.float64, device=dev)
    if multi:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = world * BATCH * IMAGES * len(e2e_ms) / (float(te.item()) / 1e3)

    # roofline of the dominant kernel (live CUDA-event durations on the launching stream)
    hbm, bf16, peak_kind = peaks()
    dom = max(kern.items(), key=lambda kv: kv[1][0])[0] if kern else None
    roof = None
    if dom is not None:
        ms, launches = kern[dom]
        per_launch_s = ms / launches / 1e3
        amps_per_launch = BATCH * IMAGES * args.steps / launches
        flop = {"cnn": CNN_FLOP, "cnn_tc": CNN_FLOP,
                "pfaffian": PFAFFIAN_FLOP + GATHER_FLOP,
                "pfaffian_tc": PFAFFIAN_FLOP + GATHER_FLOP,
                "fused": CNN_FLOP + PFAFFIAN_FLOP + GATHER_FLOP}.get(dom, 0.0)
        achieved = flop * amps_per_launch / per_launch_s / 1e12
        tb = TRAFFIC_BYTES.get(dom)
        roof = {"kernel": dom, "bound": "tensor", "achieved": achieved, "peak": bf16,
                "unit": "TFLOP/s", "frac": achieved / bf16,
                "traffic": tb * amps_per_launch if tb else None,
                "peak_source": f"{peak_kind} bf16 dense (MEASURED_PEAKS.json)",
                "fp32_core_frac": achieved / FP32_CORE_PEAK_TFLOPS,
                "note": "gather + Pfaffian FLOP (2 n^2 d + n^3 / 3 per amplitude); "
                        "fp32_core_frac is against the nominal FP32 FMA rate of 148 SMs at "
                        "1965 MHz, the roof of the CUDA-core kernel"}
    launches = sum(n for _, n in kern.values())
    kernels = {k: {"ms_per_step": v[0] / args.steps, "launches": v[1]} for k, v in kern.items()}

    config1 = None
    if world == 1 and not args.no_config1:
        config1 = measure_config1(args, dev, st)
    sampling = None
    q16 = None
    if world == 1 and not args.no_sampling:
        sampling = measure_sampling(args, dev, st, seed=77)
        q16 = sampling.pop("_proposal")
    large = None
    if world == 1 and not args.no_large:
        large = measure_large(args, dev, st, q16)
    local_energy = None
    if world == 1 and not args.no_eloc:
        local_energy = measure_local_energy(args, dev, st)
    precision = None
    if world == 1 and not args.no_precision:
        precision = measure_precision(dev, st, spins, flush)
    resconv = None
    if world == 1 and not args.no_resconv:
        resconv = measure_resconv(args, dev, st)
    config5 = None
    if world == 1 and args.config5:
        config5 = measure_config5(args, dev, st)
    extensions = None
    if world == 1 and not args.no_extensions:
        extensions = measure_extensions(args, dev, st, spins, flush)
    released_sampling = None
    if world == 1 and args.released_sampling:
        released_sampling = measure_released_sampling(args, dev, st)

    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            # FP32 (the reference's arithmetic) is the baseline; FP64 rides along for comparison.
            cpu = cpu_baseline(fp32=True)
            c64 = cpu_baseline(target_s=8.0, fp32=False)
            cpu["fp64"] = {"value": c64["value"], "sample": c64["sample"]}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
            "config": {"workload": "projected amplitudes, 16x16 Hubbard lattice, 112+112 "
                                   "electrons, 8192 configurations x 8 images = 65536 "
                                   "Pfaffians of 224x224 per step",
                       "form": ["plain FP32 CNN", "tcgen05 BF16 CNN",
                                "tcgen05 BF16x3 CNN"][args.cnn_mode] + ", " +
                               ["CUDA-core Pfaffian",
                                "tensor-memory 3xTF32 Pfaffian"][args.pf_mode],
                       "L": L, "batch": BATCH, "images": IMAGES,
                       "cnn": "4 x periodic 3x3, 32 channels, tanh-GELU, N(0, 0.02)",
                       "l2": "512 MiB written between timed steps, outside the step events",
                       "parallelism": f"replicas x{world} (chains data-parallel)"},
            "plain": plain,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": BATCH * 2 * N_SITES,
                    "d2h_bytes_per_step": BATCH * (4 + 8)},
            "config1": config1,
            "sampling": sampling,
            "local_energy": local_energy,
            "large_lattice": large,
            "precision": precision,
            "resconv": resconv,
            "released_sampling": released_sampling,
            "extensions": extensions,
            "config5": config5,
            "roofline": roof, "kernels": kernels, "gpu_launches": launches,
            "cpu_baseline": cpu, "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    if multi:
        dist.barrier()
        dist.destroy_process_group()


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    per_step = [cpu_baseline(target_s=max(2.0, 60.0 / max(1, args.steps + args.warmup)))
                for _ in range(args.warmup + args.steps)][args.warmup:]
    secs = sum(p["seconds"] for p in per_step)
    amps = sum(p["value"] * p["seconds"] for p in per_step)
    value = amps / secs
    last = per_step[-1]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference",
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
        "data": "synthetic",
        "config": {"workload": "projected amplitudes, 16x16 Hubbard lattice, 112+112 electrons, "
                               "8 images per configuration (bounded sample per step)",
                   "form": "compiled CPU restatement of the reference path (C, FP32 like the "
                           "reference's own arithmetic, OpenMP across configurations; the JAX "
                           "stack is not installable)",
                   "L": L, "images": IMAGES},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": last["cores"], "kind": "port",
                         "sample": last["sample"]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ profiling cases
# Fixed small workloads for profiling single kernels (python bench.py --profile-case CASE
# [--repeat R]): each case builds its inputs once and runs the operation R times (default 2, so
# that a profiler can skip the first, cold launch).  Inputs exceed the 126 MB L2 where the
# kernel's DRAM rate is the figure of interest.
#   pairing            nh_pairing_occ, 16x16, 2048 matrices (F = 411 MB written)
#   hops               nh_hop_list count/scan/emit, 16x16, 16384 configurations
#   eloc               local energy, 8x8 unprojected, 32768 configurations (8.4M connections)
#   proposal_sample    learned-proposal draw, 16x16, 4096 chains
#   proposal_backward  learned-proposal loss and gradient, 16x16, 4096 records
#   resconv_tc         residual network (16 blocks x 64 channels) on tcgen05, 16x16, 64 x 8 images
#   resconv            the same network on CUDA cores (FP32)
#   refine             16x16 projected amplitudes, 512 x 8 images, every image refined in FP64
#   amplitude          16x16 projected amplitudes, 1024 x 8 images, tcgen05 CNN + staged FP32
#                      Pfaffian + default refinement (the benchmark's chosen form)
#   amplitude_plain    the same on the plain form (fused FP32 CNN + Pfaffian kernel)
#   jacobian           16x16 per-sample Jacobian of log|psi_P|, 128 x 8 images (Pfaffian adjoint,
#                      pairing VJP and CNN VJP kernels after the amplitude pipeline)
#   bcs                16x16 BCS-backflow projected amplitudes, 256 x 8 images (determinant kernels)
#   observables        16x16 transverse-spin terms of one reference site, 128 configurations

def _model(L, cnn_mode=0):
    import neuralhubbard_b200 as nh

    ne = 7 * L * L // 16
    params = nh.init_params(L, L, 32, 4, std=0.02, seed=0)
    return nh.PfaffianBackflow(L, L, ne, ne, params=params, cnn_mode=cnn_mode), ne


def case_pairing(repeat):
    import torch

    import neuralhubbard_b200 as nh

    model, ne = _model(16)
    g = model.geom
    B = 2048
    rng = np.random.default_rng(0)
    Y = torch.from_numpy(rng.normal(size=(B, 2 * ne, g.d)).astype(np.float32)).cuda()
    idx = np.sort(np.stack([rng.choice(2 * g.N, 2 * ne, replace=False) for _ in range(B)]), 1)
    idx = torch.from_numpy(idx.astype(np.int32)).cuda()
    for _ in range(repeat):
        nh.pairing_occ(Y, idx, model.Wt, g)


def case_hops(repeat):
    import torch

    import neuralhubbard_b200 as nh

    L = 16
    ne = 7 * L * L // 16
    s = torch.from_numpy(nh.random_spins(np.random.default_rng(1), 16384, L * L, ne, ne)).cuda()
    H = nh.Hubbard(8.0, [1.0, -0.2], [1, 2])
    for _ in range(repeat):
        H.hop_list(s, L, L)


def case_eloc(repeat):
    import torch

    import neuralhubbard_b200 as nh

    model, ne = _model(8)
    state = nh.Variational(model, symm=False, max_parallel=65536)
    s = torch.from_numpy(nh.random_spins(np.random.default_rng(2), 32768, 64, ne, ne)).cuda()
    psi = state(s)
    H = nh.Hubbard(8.0, [1.0, -0.2], [1, 2])
    for _ in range(repeat):
        H.Oloc(state, nh.Samples(s, psi), chunk_configs=65536, count_connections=False)


def case_proposal_sample(repeat):
    import torch

    import neuralhubbard_b200 as nh

    L = 16
    ne = 7 * L * L // 16
    q = nh.HopProposal(L, L, 8, seed=3, std=0.1)
    s = torch.from_numpy(nh.random_spins(np.random.default_rng(3), 4096, L * L, ne, ne)).cuda()
    for r in range(repeat):
        q.sample(s, 11, r)


def case_proposal_backward(repeat):
    import torch

    import neuralhubbard_b200 as nh
    from neuralhubbard_b200.proposal import valid_moves

    L = 16
    ne = 7 * L * L // 16
    q = nh.HopProposal(L, L, 8, seed=4, std=0.1)
    s = torch.from_numpy(nh.random_spins(np.random.default_rng(4), 4096, L * L, ne, ne)).cuda()
    ok = valid_moves(s, L, L)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(5)
    m = torch.rand(ok.shape, generator=gen, device="cuda").masked_fill_(~ok, -1.0).argmax(1)
    w = torch.rand(4096, generator=gen, device="cuda")
    for _ in range(repeat):
        q.loss_grad(s, m.to(torch.int32), w)


def _resconv(repeat, cnn_mode):
    import torch

    import neuralhubbard_b200 as nh

    rng = np.random.default_rng(6)
    L, C = 16, 64
    params = dict(net="resconv", embed=rng.normal(size=(C, 4)).astype(np.float32),
                  conv_w=[(rng.normal(size=(C, C, 3, 3)) * 0.04).astype(np.float32)
                          for _ in range(32)],
                  conv_b=[(rng.normal(size=C) * 0.1).astype(np.float32) for _ in range(32)],
                  W=(rng.normal(size=(3, L * L, 32)) / np.sqrt(32)).astype(np.float32),
                  theta=0.55)
    ne = 7 * L * L // 16
    model = nh.PfaffianBackflow(L, L, ne, ne, params=params, cnn_mode=cnn_mode, cond_tau=0.0,
                             cancel_tau=0.0)
    state = nh.Variational(model, symm=True)
    s = torch.from_numpy(nh.random_spins(np.random.default_rng(7), 64, L * L, ne, ne)).cuda()
    for _ in range(repeat):
        state(s)


def case_resconv_tc(repeat):
    import torch

    import neuralhubbard_b200 as nh

    _resconv(repeat, 2)


def case_resconv(repeat):
    import torch

    import neuralhubbard_b200 as nh

    _resconv(repeat, 0)


def case_refine(repeat):
    import torch

    import neuralhubbard_b200 as nh

    model, ne = _model(16)
    model.refine_tau = 1.0
    state = nh.Variational(model, symm=True)
    s = torch.from_numpy(nh.random_spins(np.random.default_rng(8), 512, 256, ne, ne)).cuda()
    for _ in range(repeat):
        state(s)


def _amplitude(repeat, cnn_mode):
    import torch

    import neuralhubbard_b200 as nh

    model, ne = _model(16, cnn_mode=cnn_mode)
    state = nh.Variational(model, symm=True)
    s = torch.from_numpy(nh.random_spins(np.random.default_rng(9), 1024, 256, ne, ne)).cuda()
    for _ in range(repeat):
        state(s)


def case_amplitude(repeat):
    _amplitude(repeat, 2)


def case_amplitude_plain(repeat):
    _amplitude(repeat, 0)


def case_jacobian(repeat):
    import torch

    import neuralhubbard_b200 as nh

    model, ne = _model(16)
    state = nh.Variational(model, symm=True)
    s = torch.from_numpy(nh.random_spins(np.random.default_rng(10), 128, 256, ne, ne)).cuda()
    for _ in range(repeat):
        state.jacobian(s)


def case_bcs(repeat):
    import torch

    import neuralhubbard_b200 as nh

    ne = 112
    params = nh.init_params(16, 16, 32, 4, std=0.02, seed=0)
    params["W"] = params["W"][0]
    params["delta_d"] = 0.1
    model = nh.BCSBackflow(16, 16, ne, ne, params=params, cnn_mode=2)
    state = nh.Variational(model, symm=True)
    s = torch.from_numpy(nh.random_spins(np.random.default_rng(11), 256, 256, ne, ne)).cuda()
    for _ in range(repeat):
        state(s)


def case_observables(repeat):
    import torch

    import neuralhubbard_b200 as nh
    from neuralhubbard_b200.observables import transverse_terms

    model, ne = _model(16, cnn_mode=2)
    state = nh.Variational(model, symm=True)
    s = torch.from_numpy(nh.random_spins(np.random.default_rng(12), 128, 256, ne, ne)).cuda()
    samples = nh.Samples(s, state(s))
    for _ in range(repeat):
        transverse_terms(state, samples, (0, 0))


CASES = {"pairing": case_pairing, "hops": case_hops, "eloc": case_eloc,
         "proposal_sample": case_proposal_sample, "proposal_backward": case_proposal_backward,
         "resconv_tc": case_resconv_tc, "resconv": case_resconv,
         "refine": case_refine, "amplitude": case_amplitude,
         "amplitude_plain": case_amplitude_plain, "jacobian": case_jacobian,
         "bcs": case_bcs, "observables": case_observables}



def main():
    global BATCH
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--profile-case", default=None,
                    help="run one fixed profiling workload instead of the benchmark (cases: "
                         "pairing, hops, eloc, proposal_sample, proposal_backward, resconv_tc, "
                         "resconv, refine, amplitude, amplitude_plain)")
    ap.add_argument("--repeat", type=int, default=2, help="repetitions of --profile-case")
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cnn-mode", type=int, default=2, choices=[0, 1, 2],
                    help="0: FP32 CUDA-core CNN (plain form); 1: tcgen05 BF16; 2: tcgen05 BF16x3")
    ap.add_argument("--pf-mode", type=int, default=0, choices=[0, 1],
                    help="0: CUDA-core Pfaffian; 1: matrix in tensor memory, tcgen05 updates")
    ap.add_argument("--no-config1", action="store_true",
                    help="skip the 8x8 amplitude + local-energy block (config 1)")
    ap.add_argument("--no-sampling", action="store_true",
                    help="skip the effective-samples comparison of the two sampler forms")
    ap.add_argument("--no-eloc", action="store_true",
                    help="skip the ragged local-energy measurement (8x8 and 16x16)")
    ap.add_argument("--eloc-samples", type=int, default=4096)
    ap.add_argument("--eloc-samples-large", type=int, default=256,
                    help="local-energy samples at 24x24 (4096 is config 4's size: ~6 minutes)")
    ap.add_argument("--no-large", action="store_true",
                    help="skip the 32x32 (n = 896) Metropolis measurement")
    ap.add_argument("--large-chains", type=int, default=4096)
    ap.add_argument("--large-steps", type=int, default=2)
    ap.add_argument("--config5", action="store_true",
                    help="the learned proposal trained and measured at 32x32 (several minutes)")
    ap.add_argument("--c5-chains", type=int, default=512)
    ap.add_argument("--c5-burn", type=int, default=200)
    ap.add_argument("--c5-steps", type=int, default=300)
    ap.add_argument("--c5-records", type=int, default=65536)
    ap.add_argument("--no-extensions", action="store_true",
                    help="skip the Jacobian, BCS and packed-observable blocks")
    ap.add_argument("--no-resconv", action="store_true",
                    help="skip the released-state residual network block")
    ap.add_argument("--released-sampling", action="store_true",
                    help="also compare uniform and learned hops on the released state")
    ap.add_argument("--released-steps", type=int, default=1000)
    ap.add_argument("--released-repeats", type=int, default=16)
    ap.add_argument("--no-precision", action="store_true",
                    help="skip the precision-form report (errors against the all-FP64 path)")
    ap.add_argument("--chains", type=int, default=1024)
    ap.add_argument("--sampler-steps", type=int, default=2000)
    ap.add_argument("--burn", type=int, default=6000)
    ap.add_argument("--train-steps", type=int, default=2000)
    ap.add_argument("--energy-samples", type=int, default=512)
    ap.add_argument("--batch", type=int, default=BATCH,
                    help="configurations per step (default 8192; smaller only for profiling)")
    args = ap.parse_args()
    if args.profile_case:
        import torch

        if args.profile_case not in CASES:
            raise SystemExit(f"unknown profiling case {args.profile_case}; one of {sorted(CASES)}")
        CASES[args.profile_case](args.repeat)
        torch.cuda.synchronize()
        print(f"{args.profile_case}: ok")
        return
    if args.warmup < 3:
        args.warmup = 3
    BATCH = args.batch
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
