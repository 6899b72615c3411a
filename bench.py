#!/usr/bin/env python
"""Throughput of the batched checkerboard Ising sampler on B200.

Workload (one "step" = one checkerboard Metropolis sweep of every chain):
2D Ising, multi-spin-coded uint32, L = 4096, beta in {0.40, 0.4406868, 0.48},
64 independent chains per beta (192 chains, 3.2e9 sites, 384 MiB of spins:
far larger than the 126 MB L2, so no L2 flush is needed), hot
random start, seeds (seed, "ising", L, beta index, chain).

Metric: attempted spin updates per ns (N site visits per sweep).  Extras in
the same JSON line: heat bath, the plain one-chain-per-launch path, L = 1024,
the HBM roofline of the half-sweep kernel, clocks, and a CPU baseline (the C
oracle on host threads).

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Multi-GPU: one process per GPU under torch.distributed.run; every rank runs
its own 192 chains (weak scaling, no collective on the data path).
"""

from __future__ import annotations

import argparse
import concurrent.futures as cf
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

# the server runs many lanes on their own streams: let them map to separate
# hardware queues (a process setting read when CUDA starts)
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

L_HEAD = 4096
BETAS = (0.40, 0.4406868, 0.48)
CHAINS_PER_BETA = 64
BYTES_PER_UPDATE = 0.25  # 1 bit read + 1 bit written per site and sweep
METRIC = "attempted spin updates/ns"


def peaks() -> tuple[float, str]:
    try:
        d = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic() -> dict | None:
    """DRAM bytes per chain and half-sweep launch from the committed ncu summary."""
    p = ROOT / "profiles" / "msc_halfsweep_L4096.json"
    try:
        return json.loads(p.read_text())
    except Exception:
        return None


class Clocks:
    """Samples the SM clock and the clock-event reasons of one GPU every 1 ms
    from a host thread (NVML queries only; no setting is changed), so that a
    timed region of a few tens of milliseconds still gets several samples.  NVML
    set-up, the maximum clock and a first (discarded) sample come before the
    region starts.

    NVML is read in-process rather than through a piped ``nvidia-smi -lms``:
    that child buffers its output and, stopped by a signal, can lose every
    sample it took.
    """

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"),
               ("hw_power_brake_slowdown", "nvmlClocksEventReasonHwPowerBrakeSlowdown"))

    def __init__(self, device, period_s: float = 0.001):
        self.device = device
        self.period = period_s
        self.samples: list[tuple[float, float, int]] = []
        self.error = None
        self._stop = None
        self._thread = None

    def _handle(self, nvml):
        import torch

        try:  # match the CUDA device to its NVML handle by PCI address (CUDA_VISIBLE_DEVICES may remap)
            p = torch.cuda.get_device_properties(self.device)
            return nvml.nvmlDeviceGetHandleByPciBusId(f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0")
        except Exception:
            return nvml.nvmlDeviceGetHandleByIndex(int(getattr(self.device, "index", 0) or 0))

    def __enter__(self):
        import threading

        try:
            import pynvml as nvml

            nvml.nvmlInit()
            h = self._handle(nvml)
        except Exception as exc:  # no NVML: the line says so instead of carrying no record
            self.error = f"NVML unavailable: {exc}"
            return self
        self._stop = threading.Event()
        ready = threading.Event()
        try:
            mx = float(nvml.nvmlDeviceGetMaxClockInfo(h, nvml.NVML_CLOCK_SM))
        except Exception as exc:
            self.error = f"NVML max clock: {exc}"
            return self

        def loop():
            get_reasons = getattr(nvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nvml.nvmlDeviceGetCurrentClocksThrottleReasons
            while not self._stop.is_set():
                try:
                    sm = nvml.nvmlDeviceGetClockInfo(h, nvml.NVML_CLOCK_SM)
                    self.samples.append((float(sm), mx, int(get_reasons(h))))
                except Exception as exc:
                    self.error = str(exc)
                ready.set()
                self._stop.wait(self.period)

        self._thread = threading.Thread(target=loop, daemon=True)
        self._thread.start()
        ready.wait(2.0)
        self.samples = []  # the warm-up sample precedes the timed region
        return self

    def __exit__(self, *exc):
        if self._thread is not None:
            self._stop.set()
            self._thread.join(timeout=5)
        return False

    def summary(self) -> dict:
        if not self.samples:
            out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
            if self.error:
                out["error"] = self.error
            return out
        try:
            import pynvml as nvml
        except Exception:
            nvml = None
        reasons = set()
        for _, _, mask in self.samples:
            for name, const in self.REASONS:
                bit = getattr(nvml, const, 0) if nvml else 0
                if bit and mask & bit:
                    reasons.add(name)
        return {"sm_mhz": statistics.median(x[0] for x in self.samples),
                "sm_max_mhz": max(x[1] for x in self.samples), "reasons": sorted(reasons),
                "samples": len(self.samples), "source": f"NVML every {self.period * 1e3:.0f} ms during the timed steps"}


def ea_bench(dev, n_bins: int = 16, peak: float = 6650.0) -> dict:
    """3D EA +-J campaign: L in {6, 8, 10, 12, 16}, 512 samples each, 2 replica sets x
    32 temperatures geometric in [0.5, 2.0], one Metropolis sweep + one swap pass per
    step, 2^n_bins - 1 steps, all sizes in ONE persistent launch."""
    import torch

    from critmc_b200 import cubic
    from critmc_b200.glass import EdwardsAnderson, MultiSizeCampaign, SpinGlassCampaign, geometric_temperatures

    temps = geometric_temperatures(0.5, 2.0, 32)
    camps = []
    for L in (6, 8, 10, 12, 16):
        samples = [EdwardsAnderson(cubic(L), disorder="bimodal", seed=L * 100000 + i) for i in range(512)]
        camps.append(SpinGlassCampaign(samples, temps, seeds=[L * 200000 + i for i in range(512)], device=dev))
    mc = MultiSizeCampaign(camps)
    mc.run(2, 3)  # warm-up (first launch, shared-memory attribute)
    n_steps = (1 << n_bins) - 1
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    e0.record()
    mc.launch(n_bins, n_steps)
    e1.record()
    torch.cuda.synchronize(dev)
    s = e0.elapsed_time(e1) * 1e-3
    ups = mc.n_updates_per_step * n_steps / s / 1e9
    return {"workload": "EA +-J 3D, L 6..16 x 512 samples x 2 x 32 temperatures, one launch",
            "steps": n_steps, "seconds": s, "updates_per_ns": ups,
            "hbm_gbs_at_0.625B": ups * 0.625, "hbm_frac": ups * 0.625 / peak}


def on_bench(dev, steps: int = 40, peak: float = 6650.0) -> dict:
    """O(n) batched: XY and Heisenberg on L in {64, 128, 256}, 128 chains each (16
    temperatures in [0.7, 1.1] x 8 chains), each step 1 heat bath + 4 over-relaxation
    sweeps (5N attempted updates); ``steps`` steps per size timed (the full run is
    20,000)."""
    import torch

    from critmc_b200 import ON, hypercubic
    from critmc_b200.on_models import ONEnsemble

    temps = np.linspace(0.7, 1.1, 16)
    sched = np.array([[2, 1], [5, 4]])
    out = {}
    for n, name, bpu in ((2, "xy", 16), (3, "heisenberg", 24)):
        for L in (64, 128, 256):
            ens = ONEnsemble(ON(hypercubic((L, L)), n), temps, 8, seed=L, device=dev)
            ens.run(2, sched)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize(dev)
            e0.record()
            ens.run(steps, sched)
            e1.record()
            torch.cuda.synchronize(dev)
            s = e0.elapsed_time(e1) * 1e-3
            ups = ens.n_chains * ens.n_sites * 5 * steps / s / 1e9
            out[f"{name}_L{L}"] = {"updates_per_ns": ups, "hbm_frac": ups * bpu / peak}
            del ens
    return out


def cluster_bench(dev, updates: int = 20) -> dict:
    """Cluster updates, ``updates`` timed per case after two warm-up updates:
    Swendsen-Wang and Wolff on one 2D Ising chain of 1024 x 1024 (bit layout) at
    beta_c, q = 3 Potts 512 x 512 at 1.0 and XY 512 x 512 at beta 1.1; rate in
    sites per ns (one cluster update visits every site)."""
    import torch

    from critmc_b200 import ON, Ising, Potts, _lib, square
    from critmc_b200.device import empty_bytes, ptr, stream_handle

    out = {}
    cases = (("ising_L1024", Ising(square(1024)), 0.4406868), ("potts3_L512", Potts(square(512), 3), 1.0),
             ("xy_L512", ON(square(512), 2), 1.1))
    for name, model, beta in cases:
        rng = np.random.default_rng(1)
        s0 = model.initial_state("random", rng)
        ch = model.to_device(s0, rng, dev)
        shape = tuple(model.lattice.shape)
        dims = shape + (1,) * (3 - len(shape))
        scratch = empty_bytes(_lib.lib().critmc_cluster_scratch_bytes(1, model.n_sites), dev)
        stats = torch.zeros((1, 3), dtype=torch.int64, device=dev)
        for algo, aname in ((4, "sw"), (3, "wolff")):
            def one(sweep):
                if isinstance(model, ON):
                    _lib.call("critmc_on_cluster_update", ptr(ch.spins), 2, *dims, 2, 1, ch.key.ctypes.data, beta,
                              algo, sweep, ptr(stats), ptr(scratch), stream_handle(dev))
                else:
                    bits = isinstance(model, Ising)
                    q = 0 if bits else model.q
                    run = torch.zeros((1, 2), dtype=torch.int64, device=dev)
                    cnt = None if bits else torch.zeros(q, dtype=torch.int64, device=dev)
                    _lib.call("critmc_cluster_update", int(bits), ptr(ch.words if bits else ch.spins), 2, *dims, q,
                              1, ch.key.ctypes.data, beta, algo, sweep, ptr(run), ptr(cnt), ptr(stats),
                              ptr(scratch), stream_handle(dev))
            one(0)
            one(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize(dev)
            e0.record()
            for k in range(updates):
                one(2 + k)
            e1.record()
            torch.cuda.synchronize(dev)
            ms = e0.elapsed_time(e1) / updates
            out[f"{name}_{aname}"] = {"ms_per_update": ms, "sites_per_ns": model.n_sites / (ms * 1e6)}
    return out


def fh_bench(dev) -> dict:
    """Wang-Landau moves on the q = 10 Potts 8 x 8 torus, energy window [-1.95, -0.6]
    per site (critmc's flat-histogram double-peak case): 4736 walkers (32 per SM)
    and 18944 walkers (128 per SM, four shared-memory blocks) x 200,000 moves in
    one launch, and one walker x 1,000,000 moves, each with
    constant ln f and in 1/t mode; the C oracle runs one walker on one host core
    (2,000,000 moves) for comparison."""
    import torch

    import oracle
    from critmc_b200 import Potts, square
    from critmc_b200.flathist import WangLandau

    model = Potts(square(8), 10)
    out = {}
    for nw, moves in ((4736, 200_000), (18944, 200_000), (1, 1_000_000)):
        for one_t in (0, 1):
            wl = WangLandau(model, e_window=(-1.95, -0.6), seed=5, n_walkers=nw, device=dev)
            W = wl.walkers
            lng = torch.zeros((nw, wl.levels.size), dtype=torch.float64, device=dev)
            lnf = torch.full((nw,), 1e-3, dtype=torch.float64, device=dev)
            mode = torch.full((nw,), one_t, dtype=torch.int32, device=dev)
            args = dict(ln_f=lnf, n_levels=lnf * 80, one_over_t=mode)
            W.run(0, lng, 1000, t_base=W.trials.clone(), **args)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            base = W.trials.clone()
            torch.cuda.synchronize(dev)
            e0.record()
            W.run(0, lng, moves, t_base=base, **args)
            e1.record()
            torch.cuda.synchronize(dev)
            s = e0.elapsed_time(e1) * 1e-3
            out[f"walkers{nw}_{'one_over_t' if one_t else 'const'}_moves_per_ns"] = nw * moves / s / 1e9
    wl = WangLandau(model, e_window=(-1.95, -0.6), seed=6, device=dev)
    W = wl.walkers
    st = W.spins[0].cpu().numpy().copy()
    order = np.bincount(st.astype(np.int64), minlength=10).astype(np.int64)
    lng_h = np.zeros(wl.levels.size)
    hist_h = np.zeros(wl.levels.size, dtype=np.int64)
    key = W.keys[0].cpu().numpy().view(np.uint32)
    t0 = time.perf_counter()
    oracle.fh_run(0, st, (8, 8), 10, key, int(W.idx[0]), order, lng_h, hist_h, wl.window, 0, 1e-3, 0.0, False, 0,
                  2_000_000)
    cpu = 2_000_000 / (time.perf_counter() - t0) / 1e9
    out["cpu_oracle_one_walker_one_core_moves_per_ns"] = cpu
    out["batch_over_cpu_core"] = out["walkers18944_const_moves_per_ns"] / cpu
    return out


def small_case(dev, case: str) -> dict:
    """A small, short case of one secondary kernel: one warm-up launch, then one timed launch.

    ea-small: the EA campaign kernel on L in {6, 8, 10, 12, 16} x 64 samples x 2 x 32
    temperatures, 31 steps.  on-small: the O(n) block kernel on 128 XY chains of
    128 x 128 (16 temperatures x 8), 2 steps of 1 heat bath + 4 over-relaxation.
    fh-single / fh-batch: Wang-Landau moves (ln f = 1e-3) of one walker (500,000
    moves) or of 18944 walkers (128 per SM, 200,000 moves each) on the q = 10 Potts
    8 x 8 torus, energy window [-1.95, -0.6] per site.  cluster-sw: Swendsen-Wang
    updates of one 2D Ising chain of 1024 x 1024 (bit layout) at beta_c, two
    warm-up updates and one timed.  team-xy128: one XY 128 x 128 chain as a work
    item of an 8-block thread-block cluster, 400 Metropolis sweeps with a
    measurement after each (the served form of a large XY request).
    """
    import torch

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if case == "cluster-sw":
        from critmc_b200 import Ising, _lib, square
        from critmc_b200.device import empty_bytes, ptr, stream_handle

        model = Ising(square(1024))
        rng = np.random.default_rng(1)
        s0 = model.initial_state("random", rng)
        ch = model.to_device(s0, rng, dev)
        scratch = empty_bytes(_lib.lib().critmc_cluster_scratch_bytes(1, model.n_sites), dev)
        stats = torch.zeros((1, 3), dtype=torch.int64, device=dev)
        run = torch.zeros((1, 2), dtype=torch.int64, device=dev)

        def sw(sweep):
            _lib.call("critmc_cluster_update", 1, ptr(ch.words), 2, 1024, 1024, 1, 0, 1, ch.key.ctypes.data,
                      0.4406868, 4, sweep, ptr(run), None, ptr(stats), ptr(scratch), stream_handle(dev))

        sw(0)
        sw(1)
        torch.cuda.synchronize(dev)
        e0.record()
        sw(2)
        e1.record()
        units = model.n_sites
    elif case in ("fh-single", "fh-batch"):
        from critmc_b200 import Potts, square
        from critmc_b200.flathist import WangLandau

        nw, moves = (1, 500_000) if case == "fh-single" else (18944, 200_000)
        wl = WangLandau(Potts(square(8), 10), e_window=(-1.95, -0.6), seed=5, n_walkers=nw, device=dev)
        W = wl.walkers
        lng = torch.zeros((nw, wl.levels.size), dtype=torch.float64, device=dev)
        lnf = torch.full((nw,), 1e-3, dtype=torch.float64, device=dev)
        off = torch.zeros(nw, dtype=torch.int32, device=dev)
        W.run(0, lng, 1000, ln_f=lnf, n_levels=lnf, one_over_t=off, t_base=W.trials.clone())
        torch.cuda.synchronize(dev)
        e0.record()
        W.run(0, lng, moves, ln_f=lnf, n_levels=lnf, one_over_t=off, t_base=W.trials.clone())
        e1.record()
        units = nw * moves
    elif case == "team-xy128":
        from critmc_b200 import ON, square
        from critmc_b200.items import ItemRun, run_items

        model = ON(square(128), 2)
        s0 = model.initial_state("random", np.random.default_rng(1))
        ch = model.to_device(s0, np.random.default_rng(2), dev)
        run = model.begin(s0)
        sched = np.array([[0, 1]])
        warm = ItemRun(model, ch, run, 1.1, sched, 20, team=8)
        run_items([warm], dev)
        warm.finish()
        it = ItemRun(model, ch, run, 1.1, sched, 400, team=8)
        torch.cuda.synchronize(dev)
        e0.record()
        run_items([it], dev)
        e1.record()
        it.finish()
        units = model.lattice.n_sites * 400
    elif case == "ea-small":
        from critmc_b200 import cubic
        from critmc_b200.glass import EdwardsAnderson, MultiSizeCampaign, SpinGlassCampaign, geometric_temperatures

        temps = geometric_temperatures(0.5, 2.0, 32)
        camps = [SpinGlassCampaign([EdwardsAnderson(cubic(L), disorder="bimodal", seed=L * 1000 + i)
                                    for i in range(64)], temps, seeds=[L * 2000 + i for i in range(64)],
                                   device=dev) for L in (6, 8, 10, 12, 16)]
        mc = MultiSizeCampaign(camps)
        mc.launch(5, 31)
        torch.cuda.synchronize(dev)
        e0.record()
        mc.launch(5, 31)
        e1.record()
        units = mc.n_updates_per_step * 31
    else:
        from critmc_b200 import ON, hypercubic
        from critmc_b200.on_models import ONEnsemble

        ens = ONEnsemble(ON(hypercubic((128, 128)), 2), np.linspace(0.7, 1.1, 16), 8, seed=3, device=dev)
        sched = np.array([[2, 1], [5, 4]])
        ens.run(2, sched)
        torch.cuda.synchronize(dev)
        e0.record()
        ens.run(2, sched)
        e1.record()
        units = ens.n_chains * ens.n_sites * 5 * 2
    torch.cuda.synchronize(dev)
    s = e0.elapsed_time(e1) * 1e-3
    return {"case": case, "seconds": s, "updates_per_ns": units / s / 1e9}


def _critmc_port_state(L_x: int, L_y: int, t: int):
    """Spins, neighbour table and Generator state of host chain t (critmc's layouts)."""
    from critmc_b200 import square

    import oracle

    lat = square(L_x, L_y)
    s = (2 * np.random.default_rng(100 + t).integers(0, 2, lat.n_sites) - 1).astype(np.int8)
    words = oracle.pcg_words(np.random.PCG64DXSM(200 + t).state)
    return s, np.ascontiguousarray(lat.nbr, dtype=np.int64), words


def cpu_sample(threads: int, sweeps: int = 1, L: int = L_HEAD) -> dict:
    """critmc's own CPU Ising kernel (typewriter Metropolis, float64 table, PCG64DXSM),
    restated in C and bit-identical to critmc (tests/test_critmc_port_cpu.py), on
    `threads` host threads, one L x L chain per thread."""
    import oracle

    oracle.lib()
    s0, nbr, _ = _critmc_port_state(L, L, 0)
    states = [(2 * np.random.default_rng(100 + t).integers(0, 2, L * L) - 1).astype(np.int8) for t in range(threads)]
    words = [oracle.pcg_words(np.random.PCG64DXSM(200 + t).state) for t in range(threads)]
    del s0

    def one(t: int) -> float:
        t0 = time.perf_counter()
        oracle.critmc_ising_run(states[t], nbr, words[t], BETAS[t % 3], 0.0, [[0, 1]], sweeps,
                                running=np.zeros(2, np.int64))
        return time.perf_counter() - t0

    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(threads) as ex:
        list(ex.map(one, range(threads)))
    wall = time.perf_counter() - t0
    upd = threads * sweeps * L * L
    return {"value": upd / wall / 1e9, "unit": METRIC, "cores": threads, "kind": "port",
            "sample": f"{threads} chains of {L}x{L}, {sweeps} typewriter Metropolis sweep(s) each with critmc's "
                      f"kernel restated in C (bit-identical to critmc's numba run, same PCG64DXSM stream), one "
                      f"host thread per chain ({wall:.1f} s wall)"}


def run_reference(args) -> None:
    """CPU arm: critmc's own CPU Ising kernel (typewriter Metropolis with its
    float64 tables and PCG64DXSM stream), restated in C and bit-identical to
    critmc's numba ``run`` (tests/test_critmc_port_cpu.py), on every host thread.

    One step advances, on each host thread, its own torus of L = 4096 columns by
    one sweep: the whole 4096 x 4096 lattice when `--steps K` allows, else the
    tallest power-of-two strip of it (at least 64 rows) that keeps the K timed
    steps near 40 s (a full sweep takes about 0.2 s on one core); the rate is
    updates per ns of wall time over the K steps."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle

    oracle.lib()
    threads = os.cpu_count() or 1
    rows = L_HEAD
    while rows > 64 and args.steps * rows * L_HEAD / 0.08e9 > 40.0:
        rows //= 2
    shape = (L_HEAD, rows)
    n = shape[0] * shape[1]
    _, nbr, _ = _critmc_port_state(shape[0], shape[1], 0)  # one neighbour table, shared
    spins = [(2 * np.random.default_rng(100 + t).integers(0, 2, n) - 1).astype(np.int8) for t in range(threads)]
    words = [oracle.pcg_words(np.random.PCG64DXSM(200 + t).state) for t in range(threads)]
    runs = [np.zeros(2, np.int64) for _ in range(threads)]

    def step(t: int) -> None:
        oracle.critmc_ising_run(spins[t], nbr, words[t], BETAS[t % 3], 0.0, [[0, 1]], 1, running=runs[t])

    with cf.ThreadPoolExecutor(threads) as ex:
        for _ in range(args.warmup):
            list(ex.map(step, range(threads)))
        t0 = time.perf_counter()
        for _ in range(args.steps):
            list(ex.map(step, range(threads)))
        wall = time.perf_counter() - t0
    value = threads * n * args.steps / wall / 1e9
    what = "4096x4096 lattice" if rows == L_HEAD else f"{shape[0]}x{shape[1]} strip of the 4096x4096 lattice"
    sample = (f"{threads} host threads, each advancing its own {what} by one typewriter Metropolis sweep per "
              f"step with critmc's kernel restated in C (bit-identical to critmc)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": wall / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int8", "data": "synthetic",
        "config": {"workload": f"2D Ising L={L_HEAD} Metropolis ({what} per thread)",
                   "parallelism": f"{threads} host threads"},
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def serve_bench(dev, n_requests: int, rate: float, seed: int = 0, rank: int = 0, world: int = 1,
                max_grid_lanes: int = 8, grid_after_s: float | None = 1.0,
                team_after_s: float | None = 1.0, max_team: int = 8) -> dict | None:
    """Continuous-batching server on a seeded Poisson stream of mixed requests.

    Workload: ``n_requests`` requests at ``rate``/s, each uniform over 2D Ising
    L in {16..1024} (beta ~ U[0.38, 0.50]), q=10 Potts L in {16..128}
    (beta ~ U[1.35, 1.50]) and XY L in {32, 64, 128} (T ~ U[0.8, 1.0]), sweeps
    log-uniform in [1e3, 1e5].  Latency = arrival -> result on the host.
    With several ranks each serves its shard of the same stream (replicas);
    rank 0 returns the whole job's numbers, the others None.
    """
    from critmc_b200 import replicas
    from critmc_b200.serve import Request, Server, mixed_workload

    all_reqs = mixed_workload(n_requests, rate, seed)
    reqs = replicas.shard(all_reqs, rank, world)
    lat, upd = [], [0]

    def on_result(res):
        lat.append(res.latency)
        upd[0] += res.updates

    # series reduced to sums (stats_lag=0: no host-side error-bar sums inside the timed run)
    srv = Server(dev, keep_series=False, on_result=lambda r: None, costs="auto", max_grid_lanes=max_grid_lanes,
                 stats_lag=0, grid_after_s=grid_after_s, team_after_s=team_after_s, max_team=max_team)
    # warm-up: one short request per (model, size) of the mix builds the
    # lattice cache, the library streams and the kernels' first launches
    shapes = sorted({(r.model, r.L) for r in reqs})
    srv.run([Request(m, L, 0.44 if m == "ising" else 1.4 if m == "potts" else 1.1, 20, seed=i)
             for i, (m, L) in enumerate(shapes)])
    srv.on_result = on_result
    srv.ticks, srv.gpu_seconds, srv.updates_done, srv.max_queued, srv.peak_in_use = 0, 0.0, 0, 0, 0
    replicas.barrier(dev)
    srv.t0 = time.perf_counter()
    srv.run(reqs)
    st = srv.stats()
    parts = replicas.gather_to_root({"lat": lat, "upd": upd[0], "wall": srv.now(), "gpu": st["gpu_seconds"],
                                     "ticks": st["ticks"], "hbm": st["peak_hbm_bytes"], "queued": st["max_queued"]})
    if parts is None:
        return None
    wall = max(p["wall"] for p in parts)
    lat = [x for p in parts for x in p["lat"]]
    upd = [sum(p["upd"] for p in parts)]
    st = {"gpu_seconds": sum(p["gpu"] for p in parts), "ticks": sum(p["ticks"] for p in parts),
          "peak_hbm_bytes": max(p["hbm"] for p in parts), "max_queued": max(p["queued"] for p in parts)}
    lat_a = np.array(lat)
    return {"requests": len(lat), "rate_per_s": rate, "wall_s": wall, "gpus": world,
            "p50_latency_s": float(np.percentile(lat_a, 50)), "p99_latency_s": float(np.percentile(lat_a, 99)),
            "mean_latency_s": float(lat_a.mean()), "max_latency_s": float(lat_a.max()),
            "updates_per_ns": upd[0] / wall / 1e9, "gpu_busy_frac": st["gpu_seconds"] / wall,
            "ticks": st["ticks"], "peak_hbm_bytes": st["peak_hbm_bytes"], "max_queued": st["max_queued"],
            "team_after_s": team_after_s, "max_team": max_team if team_after_s is not None else None,
            "grid_after_s": grid_after_s if team_after_s is None else None,
            "workload": "Poisson arrivals; Ising L 16..1024 / Potts q=10 L 16..128 / XY L 32..128, "
                        "sweeps log-uniform 1e3..1e5, checkerboard Metropolis (critmc's default update)"}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--serve-requests", type=int, default=10000,
                    help="requests of the serving run (0 skips it; 1 GPU only)")
    ap.add_argument("--serve-rate", type=float, default=200.0)
    ap.add_argument("--serve-only", action="store_true", help="print only the serving run")
    ap.add_argument("--serve-grid-lanes", type=int, default=8, help="requests on multi-block lanes at once")
    ap.add_argument("--serve-grid-after", type=float, default=1.0,
                    help="item-lane seconds (cost model) above which a request takes a multi-block lane "
                         "(negative: every large lattice, first come first served)")
    ap.add_argument("--serve-max-team", type=int, default=8, choices=[2, 4, 8, 16],
                    help="largest thread-block cluster per request")
    ap.add_argument("--serve-team-after", type=float, default=1.0,
                    help="one-block seconds (cost model) above which a request runs as a thread-block-cluster "
                         "team (negative: no teams, multi-block lanes as --serve-grid-after says)")
    ap.add_argument("--case", choices=["ea-small", "on-small", "fh-single", "fh-batch", "cluster-sw", "team-xy128"],
                    help="run one small case of a secondary kernel (for profiling) and exit")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    grid_after = None if args.serve_grid_after < 0 else args.serve_grid_after
    team_after = None if args.serve_team_after < 0 else args.serve_team_after
    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    import torch.distributed as dist

    from critmc_b200.ensemble import IsingEnsemble

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    def barrier():
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def timed(fn, steps) -> float:
        s = torch.cuda.current_stream(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        barrier()
        e0.record(s)
        for _ in range(steps):
            fn()
        e1.record(s)
        barrier()
        return max_over_ranks(e0.elapsed_time(e1))

    if args.case:
        print(json.dumps(small_case(dev, args.case)), flush=True)
        return

    if args.serve_only:
        print(json.dumps({"serving": serve_bench(dev, args.serve_requests, args.serve_rate,
                                                 max_grid_lanes=args.serve_grid_lanes,
                                                 grid_after_s=grid_after, team_after_s=team_after,
                                                 max_team=args.serve_max_team)}), flush=True)
        return

    # launch shape (rows per thread, inline planes) from the autotuner; results do not depend on it
    ens = IsingEnsemble(L_HEAD, BETAS, CHAINS_PER_BETA, seed=1000 + rank, device=dev, tune=True)
    tuning = ens.tuning
    tuning_mode = (ens.mode & 0xFF) or 3  # 0 means the library's default, graph replay
    n_upd = ens.n_chains * ens.n_sites  # per step and rank
    for _ in range(args.warmup):
        ens.run(1, "metropolis", host=False)
    with Clocks(dev) as clk:
        ms = timed(lambda: ens.run(1, "metropolis", host=False), args.steps)
    value = world * n_upd * args.steps / (ms * 1e6)

    # end to end through the public API: host outputs (pinned) every step; the
    # pinned output buffers are made by untimed warm-up calls, as a caller that
    # advances its chains step after step would reuse them
    out = None
    for _ in range(2):
        out = ens.run(1, "metropolis", host=True, out=out)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        out = ens.run(1, "metropolis", host=True, out=out)
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    d2h = sum(t.numel() * t.element_size() for t in (out.Eb, out.M, out.aux))
    h2d = ens.keys.nbytes + ens.tables.nbytes + 16  # host inputs of a call: keys, tables, schedule
    e2e = {"value": world * n_upd * args.steps / (e2e_s * 1e9), "unit": METRIC,
           "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
           "note": "ensemble.run(1) with host (pinned) outputs, host wall clock; the spin "
                   "configurations stay resident on the GPU between steps"}

    peak, peak_kind = peaks()
    launches_per_step = 2  # half-sweep kernels (one launch covers <= 256 chains)
    avg_launch_ms = ms / (args.steps * launches_per_step)
    algo_bytes = ens.n_chains * (ens.n_sites / 2) * BYTES_PER_UPDATE
    achieved = algo_bytes / (avg_launch_ms * 1e-3) / 1e9
    prof = profile_traffic()
    traffic = prof["dram_bytes_per_chain_launch"] * ens.n_chains if prof else None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                "algorithmic_bytes_per_launch": algo_bytes,
                "kernel": "msc_halfsweep_kernel (Metropolis, zero field)"}

    extras = {}
    if rank == 0 and not args.no_extras:
        hb_steps = max(2, args.steps // 2)  # one heat-bath sweep per step
        ms_hb = timed(lambda: ens.run(1, "heatbath", host=False), hb_steps)
        extras["heatbath_L4096"] = n_upd * hb_steps / (ms_hb * 1e6)
        del ens
        torch.cuda.empty_cache()
        plain = IsingEnsemble(L_HEAD, BETAS[1:2], 1, seed=7, device=dev, mode=1)
        for _ in range(2):
            plain.run(1, host=False)
        ms_p = timed(lambda: plain.run(4, host=False), 3)
        extras["plain_one_chain_L4096"] = plain.n_sites * 12 / (ms_p * 1e6)
        del plain
        small = IsingEnsemble(1024, BETAS, CHAINS_PER_BETA, seed=8, device=dev)
        for _ in range(2):
            small.run(8, host=False)
        ms_s = timed(lambda: small.run(8, host=False), 3)
        extras["batched_L1024"] = small.n_chains * small.n_sites * 24 / (ms_s * 1e6)
        del small
        plain1k = IsingEnsemble(1024, BETAS[1:2], 1, seed=9, device=dev, mode=1)
        plain1k.run(4, host=False)
        ms_p1 = timed(lambda: plain1k.run(50, host=False), 1)
        extras["plain_one_chain_L1024"] = plain1k.n_sites * 50 / (ms_p1 * 1e6)
        extras["batched_over_plain"] = {
            "L4096": value / world / extras["plain_one_chain_L4096"],
            "L1024": extras["batched_L1024"] / extras["plain_one_chain_L1024"]}

    serving = None
    if args.serve_requests > 0:  # every rank serves its shard; rank 0 gets the job's numbers
        serving = serve_bench(dev, args.serve_requests, args.serve_rate, rank=rank, world=world,
                              max_grid_lanes=args.serve_grid_lanes, grid_after_s=grid_after,
                              team_after_s=team_after, max_team=args.serve_max_team)
    if rank == 0 and world == 1 and not args.no_extras:
        extras["ea_campaign"] = ea_bench(dev, peak=peaks()[0])
        extras["on_batched"] = on_bench(dev, peak=peaks()[0])
        extras["flat_histogram"] = fh_bench(dev)
        extras["cluster_updates"] = cluster_bench(dev)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_sample(min(32, os.cpu_count() or 1), sweeps=30)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic",
            "config": {"workload": f"2D Ising MSC L={L_HEAD}, betas {list(BETAS)} x "
                                   f"{CHAINS_PER_BETA} chains, checkerboard Metropolis, 1 sweep/step",
                       "chains_per_gpu": len(BETAS) * CHAINS_PER_BETA, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (384 MiB of spins per GPU)"},
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu,
            # per step: the half-sweep launches, the finalize scan, and with graph mode a cursor reset
            "gpu_launches": args.steps * (launches_per_step + 1 + (1 if tuning_mode != 1 else 0)),
            "tuning": tuning,
            "clocks": clk.summary(), "extras": extras, "serving": serving,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
