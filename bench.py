"""Benchmark of the :gradepro estimator on B200 (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
        [--workload c2|c1|c3|shape --dims 96x96x96|batched|batched-small|served]

A "step" is one complete :gradepro estimation (binning, forward transforms, every
bandwidth step, convergence, outputs) of one sample set.  The default workload is the
2-D configuration: 1,000,000 samples of a 3-component Gaussian mixture, grid 512 x 512,
200 bandwidth steps (201 bandwidths), 64 bootstrap resamples -- synthetic, seeded.

value: grid-point.bandwidth-steps per second over all ranks with samples resident in HBM;
e2e  : the same through the public API (initialize_estimation / estimate_density /
       get_density) with page-locked host samples copied in and the density copied out
       every step.
Multi-GPU: estimations are independent, so each rank runs its own (weak scaling, no
collective on the data path); timing is the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "parallelkde.jl_b200"))
sys.path.insert(0, REPO)

import numpy as np  # noqa: E402

METRIC = "KDE estimations/s + grid-pt·steps/s (%HBM peak) vs plain GPU form; p50/p99 ms"
UNIT = "grid-pt·steps/s"
HBM_FALLBACK_GBS = 6650.0


def workload(name, dims=None, samples=200_000):
    from pkde_b200 import workloads as W
    if name == "shape":  # one estimation of a batched-mix shape class (profiling single shapes)
        d = tuple(int(v) for v in dims.lower().split("x"))
        x = W.random_mixture(len(d), samples, np.random.default_rng(5))
        return x, dict(dims=d), dict(n_bootstraps=32, n_steps=100)
    if name == "c1":
        x, spec = W.gaussian_1d()
        return x, dict(dims=spec["dims"], grid_padding=spec["grid_padding"]), dict(n_bootstraps=100, n_steps=None)
    if name == "c3":
        x, spec = W.banana_t_3d()
        return x, dict(dims=spec["dims"]), dict(n_bootstraps=32, n_steps=150)
    x, spec = W.gmm_2d()
    return x, dict(dims=spec["dims"]), dict(n_bootstraps=64, n_steps=200)


def measured_traffic(workload):
    """DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one full-workload
    engine launch, from the committed ncu summary of that kernel (profiles/); None if
    there is no capture for this workload."""
    import re
    p = os.path.join(REPO, "profiles", f"engine_kernel_{workload}_ncu.md")
    if not os.path.exists(p):
        return None
    m = re.search(rf"dram_bytes_per_launch_full_{workload}:\s*([0-9.eE+]+)", open(p).read())
    return float(m.group(1)) if m else None


def peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return HBM_FALLBACK_GBS, "fallback"


class Clocks:
    """SM clock and clock-event reasons sampled every 100 ms during the timed region: NVML
    in a thread of this process (only the clock and the reason mask are read), else an
    `nvidia-smi` sampler.  (Measured on the 2-D workload: with `nvidia-smi -lms 100`
    running, the device waited for the host's launches and synchronisations ~8 ms per
    estimation -- p50 65.9 ms against 57.5 ms -- the NVML thread costs nothing visible.)"""

    NAMES = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20, "sw_power_cap": 0x4}

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.thread = None
        self.samples = []
        self.path = None

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:  # the CUDA device's own GPU, whatever CUDA_VISIBLE_DEVICES maps
            import torch
            pr = torch.cuda.get_device_properties(self.index)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def start(self):
        import threading
        try:
            nv, h = self._nvml_handle()
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            self.stop_flag = threading.Event()

            def run():
                while not self.stop_flag.is_set():
                    try:
                        self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)), int(reasons(h))))
                    except Exception:
                        pass
                    self.stop_flag.wait(0.1)

            self.thread = threading.Thread(target=run, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.thread = None
        import tempfile
        fd, self.path = tempfile.mkstemp(prefix="pkde_clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.thread is not None:
            time.sleep(0.15)
            self.stop_flag.set()
            self.thread.join(timeout=5)
            if not self.samples:
                return None
            reasons = sorted(nm for nm, bit in self.NAMES.items() if any(r & bit for _, r in self.samples))
            return {"sm_mhz": statistics.median(c for c, _ in self.samples), "sm_max_mhz": self.max_mhz,
                    "reasons": reasons, "samples": len(self.samples), "sampler": "nvml"}
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx = max(mx, float(f[1]))
            except ValueError:
                continue
            for nm, v in zip(names, f[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        try:
            os.unlink(self.path)
        except OSError:
            pass
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm),
                "sampler": "nvidia-smi"}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "gloo" if args.impl == "reference" else "nccl"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


# ----------------------------------------------------------------------- reference arm
class ReferenceSampler:
    """The reference's CPU path for this workload (the FP64 oracle port: OpenMP binning,
    scipy.fft, NumPy; ParallelKDE.jl itself needs Julia, which is absent) on bounded
    samples.  setup() does the once-per-estimation work (binning of every resample and
    of the full sample, forward FFTs, ladder); sample(k) runs k whole bandwidth steps of
    the reference's loop body (GradeProEstimator.jl:992-1043: propagate, inverse FFTs of
    all resamples, scaled VMR, means, convergence update), continuing along the ladder.
    The unit is grid-point.bandwidth-steps, so a sample's throughput needs no
    extrapolation."""

    def __init__(self, x, gspec, kw, threads):
        self.x, self.gspec, self.kw, self.threads = x, gspec, kw, threads

    def setup(self):
        from oracle import gradepro as og
        from oracle.rng import bootstrap_indices
        self.og = og
        x, kw, cores = self.x, self.kw, self.threads
        self.grid = og.find_grid(x, grid_dims=self.gspec["dims"], grid_padding=self.gspec.get("grid_padding"))
        n = x.shape[1]
        self.n = n
        idx = bootstrap_indices(0, n, kw["n_bootstraps"])
        t0 = time.perf_counter()
        Mb, Vb = og.dirac(x, self.grid, idx, nthreads=cores)
        Mf, _ = og.dirac(x, self.grid, np.arange(1, n + 1, dtype=np.int32)[None], include_var=False, nthreads=cores)
        self.Mh = og.fourier_statistics(Mb.astype(complex), cores)
        self.Vh = og.fourier_statistics(Vb.astype(complex), cores)
        self.Fh = og.fourier_statistics(Mf.astype(complex), cores)[0]
        self.times, sl, so, eps = og.ladder(x, self.grid, kw["n_steps"])
        self.tinit = og.initial_bandwidth(self.grid)
        self.state = og.DensityState(eps, sl, so, self.grid.shape_c)
        self.density = np.full(self.grid.shape_c, np.nan)
        self.s = 0
        self.setup_s = time.perf_counter() - t0
        return self.setup_s

    def sample(self, k=1):
        og, cores, st = self.og, self.threads, self.state
        t0sq = self.tinit ** 2
        with np.errstate(all="ignore"):
            for _ in range(k):
                s = self.s % len(self.times)
                t = self.times[s]
                Mt, Vt = og.propagate_statistics(self.Mh, self.Vh, self.grid, t, self.tinit)
                f = og.scaled_vmr(og.ifourier_statistics(Mt, True, cores), og.ifourier_statistics(Vt, True, cores), t,
                                  self.tinit, self.n)
                means = og.full_means(og.ifourier_statistics(og.propagate_means(self.Fh, self.grid, t), False, cores))
                dlogt = og.calculate_dlogt(t0sq, t) if s == 0 else og.calculate_dlogt(t0sq, t, self.times[s - 1])
                og.identify_convergence(self.density, means, f, st.f_prev1, st.f_prev2, dlogt, st.eps, st.steps_low,
                                        st.steps_over, st.minima, st.counters_low, st.counters_over, st.low_flags)
                st.f_prev2, st.f_prev1 = st.f_prev1, f
                self.s += 1
        return self.grid.size * k


def cpu_baseline(x, gspec, kw, budget_s=15.0, serial=True):
    """cpu_baseline of our arm's line: the oracle port threaded over every host core on
    bandwidth steps of the workload until ~budget_s, and (serial=True) one bandwidth
    step on one core (the reference's default method is :serial, Devices.jl:79-83)."""
    cores = os.cpu_count() or 1
    ref = ReferenceSampler(x, gspec, kw, cores)
    setup_s = ref.setup()
    S = len(ref.times)
    units, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < budget_s and ref.s < S:
        units += ref.sample(1)
    dt = time.perf_counter() - t0
    out = dict(value=units / dt, unit=UNIT, cores=cores, kind="port",
               sample=(f"oracle FP64 port on {cores} threads: {units // ref.grid.size} bandwidth steps of the workload "
                       f"(all {kw['n_bootstraps']} resamples, convergence update included) in {dt:.1f} s; "
                       f"binning + forward FFTs once per estimation took {setup_s:.1f} s (not in the value)"))
    if serial:
        one = ReferenceSampler(x, gspec, kw, 1)
        one.setup()
        t1 = time.perf_counter()
        u = one.sample(1)
        ts = time.perf_counter() - t1
        out["serial"] = dict(value=u / ts, unit=UNIT, cores=1, kind="port",
                             sample=f"one bandwidth step on 1 thread ({ts:.1f} s)")
    return out


def run_reference(args, x, gspec, kw, config, rank, dist):
    """--impl reference: rank 0 times the reference's CPU path; each step is one bounded
    sample (--ref-bandwidth-steps whole bandwidth steps of the workload's estimation,
    every host thread), so steps, ms_per_step and value are all measured."""
    if rank == 0:
        cores = os.cpu_count() or 1
        ref = ReferenceSampler(x, gspec, kw, cores)
        setup_s = ref.setup()
        k = max(1, args.ref_bandwidth_steps)
        for _ in range(args.warmup):
            ref.sample(k)
        units, t0 = 0, time.perf_counter()
        for _ in range(args.steps):
            units += ref.sample(k)
        dt = time.perf_counter() - t0
        value = units / dt
        serial = None
        if not args.no_serial:
            one = ReferenceSampler(x, gspec, kw, 1)
            one.setup()
            t1 = time.perf_counter()
            u = one.sample(1)
            serial = dict(value=u / (time.perf_counter() - t1), unit=UNIT, cores=1, kind="port",
                          sample="one bandwidth step on 1 thread (the reference's default :serial method)")
        S = len(ref.times)
        sample = (f"oracle FP64 port (the reference's CPU path restated; Julia is absent) on {cores} threads; each step "
                  f"= {k} whole bandwidth step(s) of the workload's estimation: propagate, inverse FFTs of all "
                  f"{kw['n_bootstraps']} resamples, scaled VMR, means, convergence update; binning + forward FFTs "
                  f"once ({setup_s:.1f} s per estimation, outside the timed steps)")
        line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * dt / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": config,
                "estimations_per_s_derived": 1.0 / (setup_s + S * (dt / (args.steps * k))),
                "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        if serial:
            line["cpu_baseline"]["serial"] = serial
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


# ---------------------------------------------------------------------------- our arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2",
                    choices=["c1", "c2", "c3", "shape", "batched", "batched-small", "served"])
    ap.add_argument("--dims", default="96x96x96",
                    help="--workload shape: grid dims of one estimation like the batched mix's (B=32, 101 "
                         "bandwidths, a random 1-4 component Gaussian mixture of --samples samples)")
    ap.add_argument("--samples", type=int, default=200_000, help="--workload shape: samples")
    ap.add_argument("--rate", type=float, default=50.0, help="requests/s (--workload served)")
    ap.add_argument("--requests", type=int, default=64, help="requests (--workload served)")
    ap.add_argument("--lanes", type=int, default=2, help="serving lanes (--workload served)")
    ap.add_argument("--batch", type=int, default=256, help="estimations per batch (--workload batched)")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-parity", action="store_true")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched-mix record that the default (c2) run appends")
    ap.add_argument("--batched-steps", type=int, default=2, help="timed batch calls of the batched-mix record")
    ap.add_argument("--ref-bandwidth-steps", type=int, default=1,
                    help="bandwidth steps per timed step of --impl reference")
    ap.add_argument("--no-serial", action="store_true", help="--impl reference: skip the 1-thread sample")
    ap.add_argument("--bandwidth-steps", type=int, default=None,
                    help="override the workload's bandwidth steps (small profiling runs only)")
    ap.add_argument("--bootstraps", type=int, default=None,
                    help="override the workload's bootstrap count (small profiling runs only)")
    args = ap.parse_args()
    world, rank, local, dist = dist_setup(args)
    if args.workload in ("batched", "batched-small", "served") and args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference arm covers the single-estimation "
                              "workloads c1/c2/c3 (the reference estimates one sample set per call)"}), flush=True)
        if dist:
            dist.destroy_process_group()
        return
    if args.workload in ("batched", "batched-small"):
        return run_batched(args, world, rank, local, dist)
    if args.workload == "served":
        return run_served(args, world, rank, local, dist)
    x, gspec, kw = workload(args.workload, args.dims, args.samples)
    if args.bandwidth_steps:
        kw["n_steps"] = args.bandwidth_steps
    if args.bootstraps:
        kw["n_bootstraps"] = args.bootstraps
    small = bool(args.bandwidth_steps or args.bootstraps)  # a profiling case, not the workload
    wl_name = {"c1": "1-D N(0,1) n=1e4, 1024 pts, B=100, 251 bandwidths",
               "c2": "2-D 3-GMM n=1e6, 512x512, B=64, 201 bandwidths",
               "c3": "3-D banana+t3 n=4e6, 128^3, B=32, 151 bandwidths",
               "shape": (f"{len(gspec['dims'])}-D random Gaussian mixture n={x.shape[1]}, "
                         f"{'x'.join(map(str, gspec['dims']))}, B=32, 101 bandwidths")}[args.workload]
    if small:
        wl_name = (f"profiling case of {args.workload} ({wl_name.split(',')[0]}): B={kw['n_bootstraps']}, "
                   f"{(kw['n_steps'] or 250) + 1} bandwidths")
    # the workload only (identical in both arms); measured figures sit outside `config`
    S_cfg = (kw["n_steps"] or 250) + 1
    config = {"workload": wl_name, "grid_points": int(np.prod(gspec["dims"])), "bandwidths": S_cfg,
              "bootstraps": kw["n_bootstraps"], "samples": int(x.shape[1]),
              "l2": "inputs (spectra 16(B+1)G bytes) larger than the 126 MB L2",
              "parallelism": f"independent estimations per rank x{world}"}

    if args.impl == "reference":
        return run_reference(args, x, gspec, kw, config, rank, dist)

    import torch
    import pkde_b200 as pk
    from pkde_b200 import _lib, multi, raw
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pk.load()
    pk.context(local)
    grid = pk.find_grid(x, grid_dims=gspec["dims"], grid_padding=gspec.get("grid_padding"))
    G = int(np.prod(grid.dims))
    n, N = x.shape[1], x.shape[0]
    S = (kw["n_steps"] or 250) + 1
    samples = torch.from_numpy(np.ascontiguousarray(x.T)).to(dev)
    dens = torch.empty(G, dtype=torch.float64, device=dev)
    sel = torch.empty(G, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream

    def one(seed):
        raw.gradepro_device(grid, samples, n, dens, sel, seed=seed, stream=sp, device_id=local,
                            n_bootstraps=kw["n_bootstraps"], n_steps=kw["n_steps"])

    # the clock sampler starts before the warm-up, so that its start-up (NVML initialisation
    # in a separate process) is over before the timed region; it samples through it
    clocks = Clocks(local)
    clocks.start()
    for w in range(args.warmup):
        one(1000 + w)
    # timed region: K estimations, samples resident in HBM; events around the step-engine
    # launches only (the per-phase breakdown comes from one profiled estimation afterwards)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    _lib.get_stats(local, reset=True)
    _lib.set_profiling(_lib.PKDE_PROFILE_STEPS, local)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    lat = []
    torch.cuda.synchronize()
    ev0.record(stream)
    for k in range(args.steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        one(multi.estimation_seed(rank, k))
        b.record(stream)
        lat.append((a, b))
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    _lib.set_profiling(_lib.PKDE_PROFILE_OFF, local)
    stats = _lib.get_stats(local, reset=True)
    elapsed_ms = ev0.elapsed_time(ev1)
    lat_ms = sorted(a.elapsed_time(b) for a, b in lat)
    t_max = multi.max_over_ranks(elapsed_ms, dist, dev)
    units = G * S * args.steps * world
    value = units / (t_max / 1000.0)

    # e2e through the public API with page-locked host samples
    e2e_value = None
    if not args.no_e2e:
        est = pk.initialize_estimation(x, grid=grid)
        est.kde.pin()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        e0 = time.perf_counter()
        ev2, ev3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev2.record(stream)
        e2e_walls = []
        for k in range(args.steps):
            tk = time.perf_counter()
            pk.estimate_density(est, "gradepro", n_bootstraps=kw["n_bootstraps"], n_steps=kw["n_steps"],
                                seed=multi.estimation_seed(rank, k), device_id=local)
            pk.get_density(est)
            e2e_walls.append((time.perf_counter() - tk) * 1000.0)
        ev3.record(stream)
        torch.cuda.synchronize()
        e2e_ms = max(ev2.elapsed_time(ev3), (time.perf_counter() - e0) * 1000.0)
        e2e_ms = multi.max_over_ranks(e2e_ms, dist, dev)
        e2e_value = units / (e2e_ms / 1000.0)

    # parity of the estimation timed first (estimation_seed(0, 0): bootstrap seed 0, the
    # fixture's) against the FP64 oracle's committed result; recomputed here, outside the
    # timed region (the estimation is deterministic)
    parity = None
    if not args.no_parity and not small and rank == 0:
        sys.path.insert(0, os.path.join(REPO, "tests", "golden"))
        import config_parity as cp
        z = cp.load(args.workload)
        if z is not None:
            one(multi.estimation_seed(0, 0))
            torch.cuda.synchronize()
            parity = cp.parity(dens.cpu().numpy(), sel.cpu().numpy(), z)
            parity["fixture"] = os.path.basename(cp.fixture_path(args.workload))

    # per-phase breakdown: one more estimation with every launch timed (not in any timed region)
    _lib.get_stats(local, reset=True)
    _lib.set_profiling(_lib.PKDE_PROFILE_ALL, local)
    one(4242)
    torch.cuda.synchronize()
    _lib.set_profiling(_lib.PKDE_PROFILE_OFF, local)
    pstats = _lib.get_stats(local, reset=True)

    # roofline of the per-bandwidth-step pipeline: FP64 spectra (2 bootstraps' means or
    # second moments per complex array, plus the full-sample means) read once per step:
    # 16 (B + 1) bytes per grid point per step.
    B = kw["n_bootstraps"]
    peak, peak_kind = peaks()
    step_phases = ["step_fft", "step_vmr", "step_means"]
    step_ms = sum(stats["phase_ms"][p] for p in step_phases) / args.steps
    step_launches = sum(stats["phase_launches"][p] for p in step_phases) / args.steps
    alg_bytes = 16.0 * (B + 1) * G * S
    achieved = alg_bytes / (step_ms / 1000.0) / 1e9 if step_ms > 0 else None
    dominant = max(pstats["phase_ms"], key=lambda p: pstats["phase_ms"][p])
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic", "config": config,
        "estimations_per_s": args.steps * world / (t_max / 1000.0),
        "p50_ms": lat_ms[len(lat_ms) // 2], "p99_ms": lat_ms[min(len(lat_ms) - 1, int(0.99 * len(lat_ms)))],
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(n * N * 8),
                "d2h_bytes_per_step": int(G * 12),
                "wall_ms_per_step": [round(v, 2) for v in e2e_walls] if e2e_value else None},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None,
                     "traffic": measured_traffic(args.workload) if not small else None,
                     "algorithmic_bytes": alg_bytes,
                     "kernel": "engine_kernel (persistent step engine: all bandwidth steps, one launch)",
                     "peak_source": peak_kind, "step_ms_per_estimation": step_ms,
                     "launches_per_estimation": step_launches},
        "phase_ms_per_estimation": dict(pstats["phase_ms"]),
        "dominant_phase": dominant,
        "gpu_launches": stats["launches"],
        "clocks": clk,
    }
    if parity is not None:
        line["parity"] = parity
    if not args.no_batched and args.workload == "c2" and not small:
        # the metric's "vs plain GPU form" part: the batched mix of 256 estimations, the same
        # set on the plain form (one estimation per call, per-bandwidth-step launches)
        args.steps, args.warmup = args.batched_steps, 1
        line["batched"] = run_batched(args, world, rank, local, dist, record=True)
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        line["cpu_baseline"] = cpu_baseline(x, gspec, kw, budget_s=args.cpu_budget)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def batched_jobs(count, seed, device, torch, small=False):
    """The batched workload: `count` independent estimations, dims uniform in {1,2,3},
    samples log-uniform in [1e3, 1e6] from random 1-4 component Gaussian mixtures, grids
    256-4096 (1-D), 128^2-512^2 (2-D), 32^3-96^3 (3-D), 100 bandwidth steps, 32
    bootstraps.  Samples and outputs are device-resident torch tensors; the host copies
    are kept for the end-to-end leg."""
    import pkde_b200 as pk
    from pkde_b200 import workloads as W
    jobs = []
    mix = W.batched_small_mix(count=count, seed=seed) if small else W.batched_mix(count=count, seed=seed)
    for e, m in enumerate(mix):
        grid = pk.find_grid(m["data"], grid_dims=m["dims"])
        G = int(np.prod(grid.dims))
        host = np.ascontiguousarray(m["data"].T)
        jobs.append(dict(grid=grid, host=host, data=torch.from_numpy(host).to(device),
                         density=torch.empty(G, dtype=torch.float64, device=device),
                         selected=torch.empty(G, dtype=torch.int32, device=device), seed=e,
                         n_bootstraps=m["n_bootstraps"], n_steps=m["n_steps"]))
    return jobs


def run_batched(args, world, rank, local, dist, record=False):
    """--workload batched: one step = one pkde_gradepro_estimate_batch call over the whole
    set.  Also timed once each, on the same set: the plain form (one estimation per call,
    per-bandwidth-step kernel launches: the structure of the reference's CUDA path) and
    the step engine one estimation per call.  record=True (the default c2 run): the
    configs' batched mix, returned as a dict for the main line instead of printed."""
    import torch
    import pkde_b200 as pk
    from pkde_b200 import _lib, multi, raw
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pk.load()
    pk.context(local)
    small = args.workload == "batched-small" and not record
    jobs = batched_jobs(args.batch, 3 + rank, dev, torch, small=small)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    units = sum(int(np.prod(j["grid"].dims)) * (j["n_steps"] + 1) for j in jobs)
    alg_bytes = sum(16.0 * (j["n_bootstraps"] + 1) * int(np.prod(j["grid"].dims)) * (j["n_steps"] + 1) for j in jobs)

    def batch():
        raw.gradepro_batch(jobs, device=True, stream=sp, device_id=local)

    clocks = Clocks(local)  # started before the warm-up (its start-up stays out of the timed region)
    clocks.start()
    for _ in range(args.warmup):
        batch()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    _lib.get_stats(local, reset=True)
    _lib.set_profiling(_lib.PKDE_PROFILE_STEPS, local)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    lat = []
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(args.steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        batch()
        b.record(stream)
        lat.append((a, b))
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    _lib.set_profiling(_lib.PKDE_PROFILE_OFF, local)
    stats = _lib.get_stats(local, reset=True)
    # per-phase breakdown from one more batch with every launch timed (untimed)
    _lib.set_profiling(_lib.PKDE_PROFILE_ALL, local)
    batch()
    torch.cuda.synchronize()
    _lib.set_profiling(_lib.PKDE_PROFILE_OFF, local)
    pstats = _lib.get_stats(local, reset=True)
    t_max = multi.max_over_ranks(ev0.elapsed_time(ev1), dist, dev)
    lat_ms = sorted(a.elapsed_time(b) for a, b in lat)
    value = units * args.steps * world / (t_max / 1000.0)
    est_per_s = len(jobs) * args.steps * world / (t_max / 1000.0)
    eng_ms = stats["phase_ms"]["step_vmr"] / args.steps
    achieved = alg_bytes / (eng_ms / 1000.0) / 1e9 if eng_ms > 0 else None
    peak, peak_kind = peaks()

    # comparators, one pass each over the same set (not part of the timed region)
    def one_at_a_time():
        for j in jobs:
            raw.gradepro_device(j["grid"], j["data"], j["data"].shape[0], j["density"], j["selected"],
                                seed=j["seed"], stream=sp, device_id=local, n_bootstraps=j["n_bootstraps"],
                                n_steps=j["n_steps"])

    def timed(fn):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b)

    engine_single_ms = timed(one_at_a_time)
    _lib.set_step_path(_lib.PKDE_STEPS_PER_STEP_LAUNCH, local)
    try:
        plain_ms = timed(one_at_a_time)
    finally:
        _lib.set_step_path(_lib.PKDE_STEPS_AUTO, local)
    plain_ms = multi.max_over_ranks(plain_ms, dist, dev)
    engine_single_ms = multi.max_over_ranks(engine_single_ms, dist, dev)

    # e2e: the same batch call with host samples in page-locked memory and host outputs
    e2e_value = None
    if not args.no_e2e and not record:
        pinned = []
        for j in jobs:
            t = torch.empty(j["host"].shape, dtype=torch.float64, pin_memory=True)
            t.numpy()[...] = j["host"]
            G = int(np.prod(j["grid"].dims))
            dens = torch.empty(G, dtype=torch.float64, pin_memory=True)
            sel = torch.empty(G, dtype=torch.int32, pin_memory=True)
            pinned.append(dict(grid=j["grid"], data=t.numpy(), density=dens.numpy(), selected=sel.numpy(),
                               seed=j["seed"], n_bootstraps=j["n_bootstraps"], n_steps=j["n_steps"], _keep=(t, dens, sel)))
        raw.gradepro_batch(pinned, device_id=local)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        e0 = time.perf_counter()
        for _ in range(args.steps):
            raw.gradepro_batch(pinned, device_id=local)
        e2e_ms = multi.max_over_ranks((time.perf_counter() - e0) * 1000.0, dist, dev)
        e2e_value = units * args.steps * world / (e2e_ms / 1000.0)
    h2d = sum(j["host"].nbytes for j in jobs)
    d2h = sum(int(np.prod(j["grid"].dims)) * 12 for j in jobs)
    kinds = {}
    for j in jobs:
        d = j["grid"].dims
        k = f"{len(d)}-D " + ("pow2" if all((v & (v - 1)) == 0 for v in d) else "other")
        kinds[k] = kinds.get(k, 0) + 1
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": (f"batched-small: {len(jobs)} estimations per step, dims 1-2, n log-uniform 1e3-1e4, "
                                "grids 256-1024 / 64^2-128^2, 101 bandwidths, B=32") if small else
                               (f"batched: {len(jobs)} estimations per step, dims 1-3, n log-uniform 1e3-1e6, "
                                "grids 256-4096 / 128^2-512^2 / 32^3-96^3, 101 bandwidths, B=32"),
                   "shapes": kinds, "estimations_per_s": est_per_s,
                   "plain_form_estimations_per_s": len(jobs) * world / (plain_ms / 1000.0),
                   "engine_one_at_a_time_estimations_per_s": len(jobs) * world / (engine_single_ms / 1000.0),
                   "batched_over_plain": (plain_ms / 1000.0) / (t_max / 1000.0 / args.steps),
                   "p50_ms": lat_ms[len(lat_ms) // 2], "p99_ms": lat_ms[min(len(lat_ms) - 1, int(0.99 * len(lat_ms)))],
                   "l2": "inputs (spectra of all estimations, GBs) larger than the 126 MB L2",
                   "parallelism": f"independent batches per rank x{world}"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": None,
                     "kernel": "engine_kernel (all N-D estimations of the batch in one launch)",
                     "peak_source": peak_kind},
        "phase_ms_per_step": dict(pstats["phase_ms"]),
        "gpu_launches": stats["launches"],
        "clocks": clk,
    }
    if record:
        cfg = line["config"]
        return {"workload": cfg["workload"], "shapes": cfg["shapes"], "estimations_per_step": len(jobs),
                "steps": args.steps, "ms_per_step": line["ms_per_step"], "estimations_per_s": est_per_s,
                "plain_form_estimations_per_s": cfg["plain_form_estimations_per_s"],
                "engine_one_at_a_time_estimations_per_s": cfg["engine_one_at_a_time_estimations_per_s"],
                "batched_over_plain": cfg["batched_over_plain"], "value": value, "unit": UNIT,
                "p50_ms_per_batch": cfg["p50_ms"], "p99_ms_per_batch": cfg["p99_ms"],
                "roofline": line["roofline"], "gpu_launches": line["gpu_launches"], "clocks": clk}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def run_served(args, world, rank, local, dist):
    """--workload served: a Poisson stream of `--requests` estimations at `--rate`
    requests/s into the serving loop (pkde_submit / pkde_wait, continuous batching over
    `--lanes` lanes).  Latency per request (submit -> results in host memory) comes
    from the library's timestamps; throughput = requests (and grid-point.steps) over the
    makespan.  Host wall clock: a served stream has no single device region to time."""
    import torch
    import pkde_b200 as pk
    from pkde_b200 import multi
    from pkde_b200 import workloads as W
    from pkde_b200.serve import Server
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pk.load()
    pk.context(local)
    mix = W.served_mix(count=args.requests, seed=4 + rank)
    reqs = [(pk.find_grid(m["data"], grid_dims=m["dims"]), m) for m in mix]
    srv = Server(device_id=local, lanes=args.lanes)

    def submit(g, m, seed):
        return srv.submit(g, m["data"], n_bootstraps=m["n_bootstraps"], n_steps=m["n_steps"], seed=seed)

    for k in range(args.warmup):  # warm-up requests, one at a time
        g, m = reqs[k % len(reqs)]
        srv.wait(submit(g, m, 10_000 + k))
    gaps = np.random.default_rng(7 + rank).exponential(1.0 / args.rate, len(reqs))
    if dist:
        dist.barrier()
    clocks = Clocks(local)
    clocks.start()
    tickets = []
    start = time.perf_counter()
    due = start
    for i, ((g, m), gap) in enumerate(zip(reqs, gaps)):
        due += gap
        delay = due - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        tickets.append(submit(g, m, i))
    results = [srv.wait(t) for t in tickets]
    makespan = time.perf_counter() - start
    clk = clocks.stop()
    bad = [r["message"] for r in results if r["status"] != 0]
    if bad:
        raise RuntimeError(f"served requests failed: {bad[:3]}")
    makespan = multi.max_over_ranks(makespan, dist, dev)
    units = sum(int(np.prod(g.dims)) * (m["n_steps"] + 1) for g, m in reqs)
    lat = sorted(r["total_ms"] for r in results)
    que = sorted(r["queue_ms"] for r in results)
    pct = lambda v, q: v[min(len(v) - 1, int(q * len(v)))]
    h2d = sum(m["data"].nbytes for _, m in reqs)
    d2h = sum(int(np.prod(g.dims)) * 12 for g, _ in reqs)
    kinds = {}
    for g, _ in reqs:
        kinds[f"{len(g.dims)}-D"] = kinds.get(f"{len(g.dims)}-D", 0) + 1
    line = {
        "metric": METRIC, "value": units * world / makespan, "unit": UNIT, "n_gpus": world,
        "steps": len(reqs), "warmup": args.warmup, "ms_per_step": 1000.0 * makespan / len(reqs),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"served: Poisson {args.rate:g} req/s, {len(reqs)} requests, dims 1-4, n log-uniform "
                               "1e3-4e6, grids to 512^2 / 128^3 / 48^4, 101 bandwidths, B=32",
                   "shapes": kinds, "lanes": args.lanes, "estimations_per_s": len(reqs) * world / makespan,
                   "p50_ms": pct(lat, 0.5), "p99_ms": pct(lat, 0.99), "queue_p50_ms": pct(que, 0.5),
                   "queue_p99_ms": pct(que, 0.99), "mean_wave": float(np.mean([r["batch_size"] for r in results])),
                   "timing": "host wall clock (submit -> results in host memory)",
                   "parallelism": f"independent request streams per rank x{world}"},
        "e2e": {"value": units * world / makespan, "unit": UNIT, "h2d_bytes_per_step": int(h2d // len(reqs)),
                "d2h_bytes_per_step": int(d2h // len(reqs))},
        "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
