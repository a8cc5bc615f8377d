#!/usr/bin/env python
"""Benchmark of the NISE propagation engine on one node.

Workload (default): batched linear absorption, Propagation Sparse (exact
propagator, Threshold 0), N = 1024 sites on an 8x8x16 lattice (8 A spacing,
static point-dipole couplings cut at 2 cm^-1), OU site energies (15000 cm^-1,
sigma 300, tau 50 fs), 100000 frames x 1 fs, RunTimes 256, Samplerate 50:
1995 start points x 3 polarisations = 1.57e9 site-steps per step.  Seeded
synthetic trajectory (no dataset exists for this benchmark).

A step is one whole job: every start point and polarisation propagated
through its 256 frames, the response reduced and the 1D spectrum computed.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (under torch.distributed.run) every rank runs an independent
replica of the job on its own GPU (replicas only: the path has no exchange
step); value = site-steps of all ranks / max device time over ranks.

--impl reference times the reference's own CPU propagator
(propagate_vector, compiled from the reference sources into
oracle/_ref/ref_bench) on the same workload's Hamiltonian: one vector step
per host thread, all threads concurrently; rank 0 only.
"""
import argparse
import ctypes
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "site-steps/s & time-to-spectrum: batched vs plain on 1 B200, <=1e-5 vs CPU"
UNIT = "site-steps/s"
WORKLOAD = "batched linear absorption, Propagation Sparse (exact exp(-iH dt), Threshold 0), N=1024 lattice"


def max_over_ranks(x, world, device):
    """Largest value of x over all ranks (the job time of replicas is the slowest rank's)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(units_per_rank, max_ms, world):
    """Whole-job throughput of `world` independent replicas: all ranks' units over the max time."""
    return world * units_per_rank / (max_ms / 1e3)


def parse():
    a = argparse.ArgumentParser()
    a.add_argument("--gpus", type=int, default=1)
    a.add_argument("--steps", type=int, default=10)
    a.add_argument("--warmup", type=int, default=3)
    a.add_argument("--impl", choices=["ours", "reference"], default="ours")
    a.add_argument("--frames", type=int, default=100000, help="trajectory length (default: the full workload)")
    a.add_argument("--no-cpu-baseline", action="store_true", help="skip the CPU baseline (profiling runs)")
    a.add_argument("--no-secondary", action="store_true", help="c1: skip the 2DIR secondary block")
    a.add_argument("--config", choices=["c0", "c1", "c2", "c3", "c4"], default="c1",
                   help="c1: the headline (batched absorption, N=1024); c0: plain absorption, N=16 chain; c2: 2DIR, "
                        "N=64 cluster; c3: adjoint, N=256 chain; c4: 64-trajectory mixed-size batch (secondary "
                        "workloads)")
    a.add_argument("--t2", type=int, default=0, help="c2 only: waiting-time steps (RunTimes 64 t2 64)")
    a.add_argument("--end", type=int, default=0, help="c2 only: EndPoint (0 = all start points)")
    a.add_argument("--c4-true-diag", action="store_true",
                   help="c4 only: the 32 Diagonal jobs with every frame diagonalised (kernel_config 2), one "
                        "context at a time, on the first --c4-frames frames, extrapolated to 5000")
    a.add_argument("--c4-frames", type=int, default=500, help="c4 --c4-true-diag: frames per job sampled")
    a.add_argument("--c4-job", type=int, default=-1,
                   help="c4 only: time job I (0..63) of the batch alone, default kernel configuration")
    return a.parse_args()


def config_dict(frames, extra=None):
    d = {"workload": WORKLOAD, "sites": 1024, "frames": frames, "timestep_fs": 1.0, "tmax1": 256,
         "samplerate": 50, "polarisations": 3, "propagation": "Sparse", "threshold": 0,
         "hamiltonian": "Coupling (static point-dipole couplings, |J| >= 2 cm^-1)",
         "l2": "inputs larger than L2 (410 MB trajectory streamed per step)", "parallelism": "replicas"}
    if extra:
        d.update(extra)
    return d


def workload(frames):
    from nise_2017_b200 import synth
    s = synth.c1_spec(frames=frames)
    kw = synth.c1_keywords(Length=frames)
    return s, kw


def site_steps(kw_len, n=1024, tmax=256, sample=50):
    nsamp = (kw_len - tmax - 1) // sample + 1
    return nsamp, 3 * nsamp * n * tmax


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.QUERY,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": len(self.rows)}
        try:
            sm = [float(r[1]) for r in self.rows]
            out["sm_mhz"] = statistics.median(sm) if sm else None
            out["sm_max_mhz"] = float(self.rows[0][2]) if self.rows else None
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            reasons = set()
            for r in self.rows:
                for i, nm in enumerate(names):
                    if r[5 + i].lower() == "active":
                        reasons.add(nm)
            out["reasons"] = sorted(reasons)
        except (ValueError, IndexError):
            pass
        return out


def read_traffic():
    """DRAM bytes per launch (dram__bytes_read.sum + write) from the committed ncu summary."""
    out = {}
    try:
        with open(os.path.join(ROOT, "profiles", "dram_traffic.txt")) as f:
            for line in f:
                parts = line.split()
                if len(parts) == 2:
                    out[parts[0]] = float(parts[1])
    except (OSError, ValueError):
        pass
    return out


def cpu_baseline(frames_dir, threads, steps=1):
    """The reference's propagate_vector (oracle/_ref/ref_bench) on this workload's Hamiltonian."""
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_bench")
    if not os.path.exists(exe):
        return None, "oracle/_ref/ref_bench not built"
    env = dict(os.environ, OPENBLAS_NUM_THREADS="1", OMP_NUM_THREADS=str(threads))
    cmd = [exe, os.path.join(frames_dir, "Energy.bin"), os.path.join(frames_dir, "Coupling.bin"), "1024", "0", "2",
           "1", "5", "0", "13500", "16500", str(threads), str(steps)]
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, env=env)
    if r.returncode != 0:
        return None, r.stdout[-300:]
    d = json.loads(r.stdout.strip().splitlines()[-1])
    return d, None


def write_small_trajectory(directory, frames=4):
    from nise_2017_b200 import synth
    s = synth.c1_spec(frames=frames)
    synth.write(s, directory)


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ---------------------------------------------------------------- our arm
def run_ours(args):
    import torch
    import torch.distributed as dist
    import nise_2017_b200 as nise
    from nise_2017_b200 import synth

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    spec, kw = workload(args.frames)
    nsamp, per_step = site_steps(args.frames)
    n = spec.n_sites
    e_bytes = spec.frames * (4 + 4 * n)
    d_bytes = 4 + 12 * n
    c_bytes = 4 + 4 * n * (n + 1) // 2
    E = torch.empty(e_bytes, dtype=torch.uint8, pin_memory=True)
    D = torch.empty(d_bytes, dtype=torch.uint8, pin_memory=True)
    C = torch.empty(c_bytes, dtype=torch.uint8, pin_memory=True)
    rc = synth.lib().nise_synth_fill(ctypes.byref(spec), E.data_ptr(), D.data_ptr(), C.data_ptr(), None, None)
    assert rc == 0
    stream = torch.cuda.current_stream()

    def ctx_for(mode, **extra):
        p = nise.params_from_keywords(dict(kw, **extra), device=local, launch_mode=mode)
        c = nise.Context(p)
        c.set_stream(stream.cuda_stream)
        return c

    def trajectory(c):
        lib = nise.lib()
        rc = lib.nise_set_trajectory(c._h, E.data_ptr(), e_bytes, D.data_ptr(), d_bytes, C.data_ptr(), c_bytes,
                                     None, 0, None, 0)
        c._check(rc)

    def one_step(c):
        re, im, ns = c.absorption()
        tot, main, launches = c.timing()
        fl, hb = c.work()
        w, sr, si = c.absorption_fft(re, im, ns)
        return main, launches + 2, fl, hb, (re, im, ns, len(w))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    c = ctx_for(nise.BATCHED)
    trajectory(c)
    for _ in range(max(args.warmup, 3)):
        one_step(c)
    clocks = ClockSampler(local)
    barrier()
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    mains, launches, flops = [], 0, 0.0
    ev0.record(stream)
    for _ in range(args.steps):
        m, l, fl, hb, last = one_step(c)
        mains.append(m)
        launches += l
        flops = fl
        hbm = hb
    ev1.record(stream)
    barrier()
    clk = clocks.stop()
    ms = max_over_ranks(ev0.elapsed_time(ev1), world, "cuda")
    value = replica_throughput(per_step * args.steps, ms, world)

    # end to end through the C ABI from pinned host buffers, copies inside the timed region
    barrier()
    for _ in range(2):
        trajectory(c)
        one_step(c)
    barrier()
    ev0.record(stream)
    for _ in range(args.steps):
        trajectory(c)
        one_step(c)
    ev1.record(stream)
    barrier()
    e2e_ms = max_over_ranks(ev0.elapsed_time(ev1), world, "cuda")
    e2e_value = replica_throughput(per_step * args.steps, e2e_ms, world)
    fft = max(c.params.fft, c.params.tmax1)
    h2d = e_bytes + d_bytes + c_bytes
    d2h = c.params.tmax1 * 16 + fft * 16  # response sums and device spectrum

    # plain: one start point (3 polarisations) per launch, over the first
    # PLAIN_SAMPLES start points of the same job (throughput per launch does
    # not depend on how many launches follow)
    plain_samples = min(100, nsamp)
    cp = ctx_for(nise.PLAIN, EndPoint=plain_samples)
    trajectory(cp)
    one_step(cp)
    barrier()
    ev0.record(stream)
    one_step(cp)
    ev1.record(stream)
    barrier()
    plain_ms = max_over_ranks(ev0.elapsed_time(ev1), world, "cuda")
    plain_value = replica_throughput(3 * plain_samples * n * 256, plain_ms, world)
    cp.close()

    main_ms = statistics.mean(mains)
    achieved = flops / (main_ms / 1e3) / 1e12
    peak = nise.fp32_peak(local)
    traffic = read_traffic().get("k_abs_taylor_rv_fp32_per_launch")
    # shared-memory side of the same kernels: every Chebyshev term gathers each
    # coupling's neighbour state (8 bytes per vector); their rate against the
    # SM shared-memory bandwidth, 128 bytes per clock per SM at the sampled clock
    cf = np.frombuffer(C.numpy().tobytes(), dtype=np.float32)[1:]
    iu = np.triu_indices(n)
    nnz = 2 * int(np.count_nonzero((np.abs(cf) >= float(kw["Couplingcut"])) & (iu[0] != iu[1])))
    orders_cross = flops / (4.0 * nnz + 10.0 * n)
    smem_bytes = orders_cross * nnz * 8.0
    nsm = torch.cuda.get_device_properties(local).multi_processor_count
    smem_peak = nsm * 128.0 * (clk.get("sm_mhz") or 1965.0) * 1e6 / 1e9
    # the HBM side of the same kernel, against the measured copy bandwidth
    try:
        with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")) as f:
            hbm_peak, hbm_src = float(json.load(f)["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (measured)"
    except (OSError, ValueError, KeyError):
        hbm_peak, hbm_src = 6650.0, "fallback 6.65 TB/s"
    hbm_achieved = hbm / (main_ms / 1e3) / 1e9
    out = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            with tempfile.TemporaryDirectory() as td:
                write_small_trajectory(td)
                threads = min(host_threads(), 16)
                t0 = time.time()
                d, err = cpu_baseline(td, threads)
                if d:
                    cpu = {"value": d["site_steps"] / d["seconds"], "unit": UNIT, "cores": threads,
                           "kind": "reference",
                           "sample": "%d concurrent vector steps (one per thread) of the reference's propagate_vector "
                                     "(Sparse, Threshold 0: ssyev_ + dense U) at N=1024 on frame 0 of this workload, "
                                     "%.1f s wall" % (threads, d["seconds"])}
                else:
                    cpu = {"value": None, "unit": UNIT, "cores": threads, "kind": "reference", "sample": err}
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (propagation), f64 (response sums)",
            "data": "synthetic (seeded OU trajectory, point-dipole lattice couplings)",
            "config": config_dict(args.frames, {"start_points": nsamp}),
            "time_to_spectrum_s": e2e_ms / args.steps / 1e3,
            "plain": {"value": plain_value, "unit": UNIT, "ms": plain_ms, "start_points": plain_samples,
                      "mode": "one start point (3 polarisations) per launch"},
            "batched_over_plain": value / plain_value,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": e2e_ms / args.steps},
            "roofline": {"bound": "fp32",
                         "kernel": "k_abs_taylor_rv (row-owner Chebyshev series, whole waves) + k_abs_taylor3 "
                                   "(1-vector tail) + series prep",
                         "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak if peak else None, "traffic": traffic,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of k_abs_taylor_rv on "
                                           "the 40 000-frame case, scaled by start points (profiles/dram_traffic.txt)",
                         "peak_source": "measured in-process FP32 FMA throughput (nise_probe_fp32_peak)",
                         "algorithmic_flops_per_launch": flops, "algorithmic_hbm_bytes_per_launch": hbm,
                         "kernel_ms": main_ms,
                         "smem": {"achieved": smem_bytes / (main_ms / 1e3) / 1e9, "peak": smem_peak, "unit": "GB/s",
                                  "frac": smem_bytes / (main_ms / 1e3) / 1e9 / smem_peak,
                                  "algorithmic_bytes_per_launch": smem_bytes,
                                  "peak_source": "%d SMs x 128 B/clock at the median sampled SM clock" % nsm,
                                  "note": "the binding resource: the neighbour-state gathers of every series term"},
                         "hbm": {"achieved": hbm_achieved, "peak": hbm_peak, "unit": "GB/s",
                                 "frac": hbm_achieved / hbm_peak, "peak_source": hbm_src,
                                 "note": "each frame is read once and shared by every vector in flight: "
                                         "HBM is not the binding resource"}},
            "cpu_baseline": cpu,
            "clocks": clk,
            "gpu_launches": launches,
        }
    c.close()
    if rank == 0 and world == 1 and not args.no_secondary:
        # the 2DIR workload on its first 20 start points, with its own clock record
        sec = argparse.Namespace(**vars(args))
        sec.end, sec.t2, sec.steps, sec.warmup = 20, 0, 2, 1
        out["secondary"] = {"c2": run_c2(sec, emit=False)}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return out


# ---------------------------------------------------------------- C0 (secondary)
def run_c0(args):
    """Linear absorption, Propagation Coupling (Trotter), N = 16 chain (c0 statistics), 10000 x 2 fs
    frames, RunTimes 128, Samplerate 20 (494 start points), Couplingcut 0.1, Trotter 5.

    value = site-steps per second of the batched job (all start points in one launch); plain =
    the same job with one start point (3 polarisations) per launch."""
    import torch
    import nise_2017_b200 as nise
    from nise_2017_b200 import synth
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    kw = synth.c0_keywords()
    out = {}
    with tempfile.TemporaryDirectory() as td:
        files = synth.write(synth.c0_spec(), td)
        for mode in (nise.BATCHED, nise.PLAIN):
            with nise.Context(nise.params_from_keywords(kw, files, device=local, launch_mode=mode)) as c:
                c.load_files()
                for _ in range(max(args.warmup, 3)):
                    c.absorption()
                clk = ClockSampler(local)
                clk.start()
                times = []
                for _ in range(args.steps):
                    re, im, ns = c.absorption()
                    tot, main, launches = c.timing()
                    times.append(tot)
                out[mode] = (statistics.mean(times), launches, clk.stop(), ns)
    ms, launches, clocks, ns = out[nise.BATCHED]
    pms = out[nise.PLAIN][0]
    site_steps = 3 * ns * 128 * 16
    res = {"metric": "C0 linear absorption, Trotter scheme: site-steps/s, batched vs plain (secondary workload)",
           "value": site_steps / (ms / 1e3), "unit": "site-steps/s", "n_gpus": 1, "steps": args.steps,
           "warmup": max(args.warmup, 3), "ms_per_step": ms, "higher_is_better": True,
           "dtype": "f32 (propagation), f64 (response sums)",
           "config": {"workload": "plain linear absorption, Propagation Coupling, N=16 chain, 10000 x 2 fs, "
                                  "RunTimes 128, Samplerate 20, Couplingcut 0.1, Trotter 5", "start_points": ns},
           "plain": {"value": site_steps / (pms / 1e3), "unit": "site-steps/s", "ms": pms,
                     "mode": "one start point (3 polarisations) per launch", "launches": out[nise.PLAIN][1]},
           "batched_over_plain": pms / ms, "clocks": clocks, "gpu_launches": launches}
    print(json.dumps(res), flush=True)
    return res


# ---------------------------------------------------------------- 2DIR (secondary)
def run_c2(args, emit=True):
    """2DIR, N = 64 random cluster, Tmax1 = Tmax3 = 64, Samplerate 100, 20000 x 2 fs frames.

    value = reference-equivalent doubles site-steps per second: the reference
    propagates 21 * (tmax1 + 1) doubles vectors of N(N+1)/2 states through
    tmax3 steps per start point (calc_2DIR.c:448-505)."""
    import torch
    import nise_2017_b200 as nise
    from nise_2017_b200 import synth
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    s = synth.c2_spec()
    kw = synth.c2_keywords(RunTimes="64 %d 64" % args.t2)
    if args.end:
        kw["EndPoint"] = args.end
    with tempfile.TemporaryDirectory() as td:
        files = synth.write(s, td)
        p = nise.params_from_keywords(kw, files, device=local)
        with nise.Context(p) as c:
            c.load_files()
            for _ in range(max(args.warmup, 1)):
                c.twodir()
            times, mains = [], []
            clk = ClockSampler(local)
            clk.start()
            for _ in range(args.steps):
                R, n = c.twodir()
                tot, main, launches = c.timing()
                times.append(tot)
                mains.append(main)
            clocks = clk.stop()
            flops, _ = c.work()
        # plain: one start point per launch of every kernel, over the first 4 start points
        plain_samples = 4
        pp = nise.params_from_keywords(dict(kw, EndPoint=plain_samples), files, device=local,
                                       launch_mode=nise.PLAIN)
        with nise.Context(pp) as c:
            c.load_files()
            c.twodir()
            c.twodir()
            plain_ms, _, _ = c.timing()
    n2 = 64 * 65 // 2
    site_steps = n * 21 * 65 * 64 * n2
    plain_value = plain_samples * 21 * 65 * 64 * n2 / (plain_ms / 1e3)
    ms = statistics.mean(times)
    out = {"metric": "2DIR time-to-spectrum and doubles site-steps/s (secondary workload)",
           "value": site_steps / (ms / 1e3), "unit": "site-steps/s", "n_gpus": 1, "steps": args.steps,
           "warmup": max(args.warmup, 1), "ms_per_step": ms, "time_to_spectrum_s": ms / 1e3,
           "config": {"workload": "2DIR, Propagation Coupling, N=64 random cluster, RunTimes 64 %d 64, "
                                  "Samplerate 100, 20000 x 2 fs" % args.t2, "start_points": n},
           "doubles_fp32_tflops": flops / (statistics.mean(mains) / 1e3) / 1e12, "gpu_launches": launches,
           "plain": {"value": plain_value, "unit": "site-steps/s", "ms": plain_ms, "start_points": plain_samples,
                     "mode": "one start point per launch of every kernel"},
           "batched_over_plain": (site_steps / (ms / 1e3)) / plain_value, "clocks": clocks}
    if emit:
        print(json.dumps(out), flush=True)
    return out


def run_c3(args):
    """Adjoint of linear absorption (FP64 Trotter model): N = 256 chain with the c0
    statistics, 20000 x 2 fs frames, Tmax1 128, Samplerate 20.  The loss is the L2
    distance to a target spectrum made by the same model with per-site shifts drawn
    from N(0, 5 cm^-1) and a coupling scale of 1.1; gradients with respect to the 256
    shifts, the coupling scale and the lifetime, checkpoints every 32 steps.

    value = site-steps per second of one forward model run plus one backward run (the
    backward sweep recomputes the states from checkpoints); fd_check = the largest
    disagreement with central differences (h = 1e-3, one Richardson step) over sites 0,
    85, 170, 255, the scale and the lifetime, relative to the largest gradient component."""
    import numpy as np
    import torch
    import nise_2017_b200 as nise
    from nise_2017_b200 import synth
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    s = synth.c3_spec()
    kw = synth.c3_keywords()
    with tempfile.TemporaryDirectory() as td:
        files = synth.write(s, td)
        p = nise.params_from_keywords(kw, files, device=local, precision=nise.FP64)
        n, lt0 = p.singles, float(p.lifetime)
        nsamp = (p.length - p.tmax1 - 1) // p.sample + 1
        site_steps = 3 * nsamp * p.tmax1 * n
        rng = np.random.default_rng(20173)
        with nise.Context(p) as c:
            c.load_files()
            _, tr, ti = c.absorption_model(rng.normal(0, 5, n), 1.1, lt0)

            def loss(shift, scale, lt):
                _, sr, si = c.absorption_model(shift, scale, lt)
                return float(((sr - tr) ** 2).sum() + ((si - ti) ** 2).sum()), 2 * (sr - tr), 2 * (si - ti)

            shift = np.zeros(n)
            for _ in range(max(args.warmup, 3)):
                L, dre, dim = loss(shift, 1.0, lt0)
                c.backward_absorption(shift, 1.0, lt0, dre, dim)
            clk = ClockSampler(local)
            clk.start()
            times, fwd_ms, bwd_ms = [], [], []
            for _ in range(args.steps):
                t0 = time.perf_counter()
                L, dre, dim = loss(shift, 1.0, lt0)
                f_ms, _, _ = c.timing()
                g, gs, gl = c.backward_absorption(shift, 1.0, lt0, dre, dim)
                b_ms, _, launches = c.timing()
                times.append((time.perf_counter() - t0) * 1e3)
                fwd_ms.append(f_ms)
                bwd_ms.append(b_ms)
            clocks = clk.stop()

            def central(f, x, h=1e-3):
                d1 = (f(x + h) - f(x - h)) / (2 * h)
                d2 = (f(x + h / 2) - f(x - h / 2)) / h
                return (4 * d2 - d1) / 3

            fd, adj = [], []
            for a in (0, 85, 170, 255):
                e = np.zeros(n)
                e[a] = 1.0
                fd.append(central(lambda x: loss(shift + x * e, 1.0, lt0)[0], 0.0))
                adj.append(g[a])
            fd.append(central(lambda x: loss(shift, x, lt0)[0], 1.0))
            adj.append(gs)
            fd.append(central(lambda x: loss(shift, 1.0, x)[0], lt0))
            adj.append(gl)
            scale = max(np.abs(g).max(), abs(gs), abs(gl))
            fd_err = float(max(abs(x - y) for x, y in zip(adj, fd)) / scale)
    dev_ms = statistics.mean(fwd_ms) + statistics.mean(bwd_ms)
    out = {"metric": "adjoint of linear absorption: forward + backward site-steps/s (secondary workload)",
           "value": site_steps / (dev_ms / 1e3), "unit": "site-steps/s", "n_gpus": 1, "steps": args.steps,
           "warmup": max(args.warmup, 3), "ms_per_step": dev_ms, "higher_is_better": True, "dtype": "f64",
           "config": {"workload": "adjoint, N=256 chain (c0 statistics), 20000 x 2 fs, RunTimes 128 0 0, "
                                  "Samplerate 20, Trotter 5, checkpoints every 32 steps; loss vs a target with "
                                  "shifts ~ N(0, 5 cm^-1) and coupling scale 1.1", "start_points": nsamp},
           "forward_ms": statistics.mean(fwd_ms), "backward_ms": statistics.mean(bwd_ms),
           "time_to_gradient_s": statistics.mean(times) / 1e3, "gpu_launches": launches,
           "fd_check": {"max_rel_err": fd_err, "components": "sites 0, 85, 170, 255; scale; lifetime",
                        "h": 1e-3, "scheme": "central, one Richardson step"},
           "clocks": clocks}
    print(json.dumps(out), flush=True)
    return out


def c4_sites():
    """Site counts of the mixed-size batch: round(8 * 256^(i/63)), i = 0..63 (8 ... 2048)."""
    return [int(round(8 * 256 ** (i / 63.0))) for i in range(64)]


def run_c4(args):
    """64 absorption trajectories, N log-spaced 8..2048, lattice couplings and OU site noise (the
    C1 statistics), 5000 x 1 fs frames, Tmax1 128, Samplerate 25; even i Propagation Coupling,
    odd i Propagation Diagonal; all jobs in one CUDA graph (nise_batch_*), autotuned.

    value = aggregate site-steps per second of one graph launch (all 64 spectra).  The
    sequential comparison runs the same jobs one context at a time (nise_absorption)."""
    import torch
    import nise_2017_b200 as nise
    from nise_2017_b200 import synth
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    frames, tmax, sample = 5000, 128, 25
    sizes = c4_sites()
    if args.c4_job >= 0:
        return run_c4_job(args, args.c4_job, sizes[args.c4_job], frames, tmax, sample, local)
    if args.c4_true_diag:
        return run_c4_true_diag(args, sizes, frames, tmax, sample, local)
    nsamp = (frames - tmax - 1) // sample + 1
    site_steps = sum(3 * nsamp * tmax * n for n in sizes)
    ctxs = []
    with tempfile.TemporaryDirectory() as td:
        try:
            for i, n in enumerate(sizes):
                s = synth.c1_spec(n_sites=n, frames=frames, seed=40000 + i)
                files = synth.write(s, os.path.join(td, "t%02d" % i))
                kw = synth.c1_keywords(Singles=n, Length=frames, RunTimes="%d 0 0" % tmax, Samplerate=sample,
                                       Propagation="Coupling" if i % 2 == 0 else "Diagonal", FFT=1024)
                c = nise.Context(nise.params_from_keywords(kw, files, device=local))
                c.load_files()
                ctxs.append(c)
            # sequential comparison: every job on its own, one after another (device time)
            seq_ms, per_job = 0.0, []
            for c in ctxs:
                re, im, n = c.absorption()
                c.absorption_fft(re, im, n)
                re, im, n = c.absorption()
                tot, _, _ = c.timing()
                seq_ms += tot
                per_job.append(tot)
            with nise.Batch(ctxs, autotune=True) as b:
                for _ in range(max(args.warmup, 3)):
                    b.run()
                times = []
                clk = ClockSampler(local)
                clk.start()
                for _ in range(args.steps):
                    b.run()
                    ms, launches = b.timing()
                    times.append(ms)
                clocks = clk.stop()
        finally:
            for c in ctxs:
                c.close()
    ms = statistics.mean(times)
    out = {"metric": "C4 mixed-size batch: aggregate site-steps/s and time-to-spectrum (secondary workload)",
           "value": site_steps / (ms / 1e3), "unit": "site-steps/s", "n_gpus": 1, "steps": args.steps,
           "warmup": max(args.warmup, 3), "ms_per_step": ms, "higher_is_better": True,
           "time_to_spectrum_s": ms / 1e3,
           "config": {"workload": "64 trajectories, N = round(8*256^(i/63)) = 8..2048 (sum %d), lattice couplings, "
                                  "OU sites, 5000 x 1 fs, RunTimes 128 0 0, Samplerate 25, even i Coupling, "
                                  "odd i Diagonal, one CUDA graph, autotuned" % sum(sizes),
                      "site_steps": site_steps},
           "sequential": {"ms": seq_ms, "value": site_steps / (seq_ms / 1e3),
                          "mode": "the same jobs one context at a time (nise_absorption)",
                          "slowest_job_ms": max(per_job), "slowest_job_sites": sizes[per_job.index(max(per_job))]},
           "batched_over_sequential": seq_ms / ms, "clocks": clocks, "gpu_launches": launches}
    print(json.dumps(out), flush=True)
    return out


def run_c4_true_diag(args, sizes, frames, tmax, sample, local):
    """The Diagonal half of C4 (odd i, 9..2048 sites) with every frame diagonalised: the eigen
    route (kernel_config 2: per-frame FP64 eigendecomposition, U = V exp(-i e f) V^T, applied on
    the tensor cores above 120 sites with the propagators built chunk by chunk), one context at a
    time on the first F frames of each trajectory; device time per job, summed, and scaled by
    5000 / F (the route's cost is per frame).  Beside it the default route (the Chebyshev series
    for static couplings) on the same sample."""
    import nise_2017_b200 as nise
    from nise_2017_b200 import synth
    F = max(tmax + sample, min(args.c4_frames, frames))
    jobs = []
    with tempfile.TemporaryDirectory() as td:
        for i in range(1, 64, 2):
            n = sizes[i]
            s = synth.c1_spec(n_sites=n, frames=F, seed=40000 + i)
            files = synth.write(s, os.path.join(td, "t%02d" % i))
            kw = synth.c1_keywords(Singles=n, Length=F, RunTimes="%d 0 0" % tmax, Samplerate=sample,
                                   Propagation="Diagonal", FFT=1024)
            row = {"i": i, "sites": n}
            for label, cfg in (("eigen_ms", 2), ("series_ms", 0)):
                with nise.Context(nise.params_from_keywords(kw, files, device=local, kernel_config=cfg)) as c:
                    c.load_files()
                    c.absorption()
                    tot, _, _ = c.timing()
                row[label] = tot
            jobs.append(row)
            shutil.rmtree(os.path.join(td, "t%02d" % i), ignore_errors=True)
    eig = sum(j["eigen_ms"] for j in jobs)
    ser = sum(j["series_ms"] for j in jobs)
    out = {"metric": "C4 Diagonal half with true diagonalisation (eigen route) vs the series route",
           "unit": "ms", "frames_sampled": F, "frames_full": frames,
           "eigen_ms_sample": eig, "series_ms_sample": ser,
           "eigen_ms_extrapolated": eig * frames / F, "series_ms_extrapolated": ser * frames / F,
           "eigen_over_series": eig / ser if ser else None,
           "note": "one context at a time, device time of one absorption call each (the plan's allocations "
                   "outside); extrapolated linearly in frames",
           "jobs": jobs}
    print(json.dumps(out), flush=True)
    return out


def run_c4_job(args, i, n, frames, tmax, sample, local):
    """One job of the C4 batch alone (profiling case): the same trajectory and keywords,
    the default kernel configuration, device time per absorption call."""
    import nise_2017_b200 as nise
    from nise_2017_b200 import synth
    prop = "Coupling" if i % 2 == 0 else "Diagonal"
    times = []
    with tempfile.TemporaryDirectory() as td:
        s = synth.c1_spec(n_sites=n, frames=frames, seed=40000 + i)
        files = synth.write(s, td)
        kw = synth.c1_keywords(Singles=n, Length=frames, RunTimes="%d 0 0" % tmax, Samplerate=sample,
                               Propagation=prop, FFT=1024)
        with nise.Context(nise.params_from_keywords(kw, files, device=local)) as c:
            c.load_files()
            for k in range(max(args.warmup, 1) + args.steps):
                c.absorption()
                tot, main, launches = c.timing()
                if k >= max(args.warmup, 1):
                    times.append((tot, main))
    nsamp = (frames - tmax - 1) // sample + 1
    out = {"metric": "C4 job %d alone: site-steps/s" % i, "value": 3 * nsamp * tmax * n / (statistics.mean(
        t[0] for t in times) / 1e3), "unit": "site-steps/s", "sites": n, "propagation": prop,
        "ms_per_job": statistics.mean(t[0] for t in times), "main_kernel_ms": statistics.mean(t[1] for t in times),
        "steps": args.steps, "gpu_launches": launches}
    print(json.dumps(out), flush=True)
    return out


# ---------------------------------------------------------------- reference arm
def ref_exe(name):
    exe = os.path.join(ROOT, "oracle", "_ref", name)
    return exe if os.path.exists(exe) else None


def run_program(exe, inp, cwd, threads):
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OPENBLAS_NUM_THREADS="1")
    t0 = time.perf_counter()
    r = subprocess.run([exe, inp], cwd=cwd, env=env, stdout=subprocess.DEVNULL, stderr=subprocess.STDOUT)
    return time.perf_counter() - t0, r.returncode


def run_reference_c0(args):
    """The reference program (oracle/_ref/NISE_acc, absorption.c) on the whole C0 job: one process,
    and P processes over disjoint BeginPoint/EndPoint ranges (absorption is serial in the
    reference; its response sums are additive over start points)."""
    from nise_2017_b200 import synth
    exe = ref_exe("NISE_acc")
    if not exe:
        return {"impl": "reference", "unavailable": "oracle/_ref/NISE_acc was not built"}
    kw = synth.c0_keywords()
    nsamp = (10000 - 128 - 1) // 20 + 1
    site_steps = 3 * nsamp * 128 * 16
    procs = max(1, min(host_threads(), 8))
    with tempfile.TemporaryDirectory() as td:
        files = synth.write(synth.c0_spec(), td)
        inp = synth.write_input(os.path.join(td, "input"), kw, files)
        run_program(exe, inp, td, 1)  # untimed: pages in the binary
        one, rc = run_program(exe, inp, td, 1)
        if rc:
            return {"impl": "reference", "unavailable": "NISE_acc failed on the C0 input"}
        jobs, t0 = [], time.perf_counter()
        for k in range(procs):
            d = os.path.join(td, "p%d" % k)
            os.makedirs(d)
            b, e = k * nsamp // procs, (k + 1) * nsamp // procs
            ip = synth.write_input(os.path.join(d, "input"), dict(kw, BeginPoint=b, EndPoint=e), files)
            jobs.append(subprocess.Popen([exe, ip], cwd=d, env=dict(os.environ, OMP_NUM_THREADS="1"),
                                         stdout=subprocess.DEVNULL, stderr=subprocess.STDOUT))
        for j in jobs:
            j.wait()
        multi = time.perf_counter() - t0
    return {"impl": "reference", "config": "c0", "value": site_steps / multi, "unit": UNIT,
            "time_to_spectrum_s": multi, "one_process": {"value": site_steps / one, "seconds": one, "cores": 1},
            "cpu_baseline": {"value": site_steps / multi, "unit": UNIT, "cores": procs, "kind": "reference",
                             "sample": "the whole C0 job (%d start points) in %d processes over disjoint "
                                       "BeginPoint/EndPoint ranges" % (nsamp, procs)}}


def run_reference_c2(args):
    """The reference program (calc_2DIR.c, OpenMP over t1 in propagate.c:1541) on the first
    start points of the C2 job, extrapolated linearly to all 199."""
    from nise_2017_b200 import synth
    exe = ref_exe("NISE_acc")
    if not exe:
        return {"impl": "reference", "unavailable": "oracle/_ref/NISE_acc was not built"}
    threads = host_threads()
    sample_points = 2
    kw = synth.c2_keywords(EndPoint=sample_points)
    nsamp = (20000 - 64 - 0 - 64 - 1) // 100 + 1
    with tempfile.TemporaryDirectory() as td:
        files = synth.write(synth.c2_spec(), td)
        inp = synth.write_input(os.path.join(td, "input"), kw, files)
        secs, rc = run_program(exe, inp, td, threads)
        if rc:
            return {"impl": "reference", "unavailable": "NISE_acc failed on the C2 input"}
    n2 = 64 * 65 // 2
    per_point = secs / sample_points
    return {"impl": "reference", "config": "c2", "value": 21 * 65 * 64 * n2 / per_point, "unit": "site-steps/s",
            "time_to_spectrum_s": per_point * nsamp, "extrapolated": True,
            "cpu_baseline": {"value": 21 * 65 * 64 * n2 / per_point, "unit": "site-steps/s", "cores": threads,
                             "kind": "reference",
                             "sample": "%d of %d start points (%.1f s), extrapolated linearly" % (
                                 sample_points, nsamp, secs)}}


def run_reference_c4(args):
    """The reference's propagate_vector (oracle/_ref/ref_bench) per C4 job: the Coupling (Trotter)
    jobs timed on a few concurrent vector steps each; the Diagonal jobs (the reference runs them as
    Sparse, Threshold 0: ssyev_ plus N^3 per vector step) timed up to 300 sites and extrapolated
    with the measured N^3 law above.  Job time = vector steps x time per vector step."""
    from nise_2017_b200 import synth
    exe = ref_exe("ref_bench")
    if not exe:
        return {"impl": "reference", "unavailable": "oracle/_ref/ref_bench was not built"}
    threads = max(1, min(host_threads(), 16))
    frames, tmax, sample = 5000, 128, 25
    nsamp = (frames - tmax - 1) // sample + 1
    vec_steps = 3 * nsamp * (tmax - 1)
    per_step, measured = {}, {}
    with tempfile.TemporaryDirectory() as td:
        for i, n in enumerate(c4_sites()):
            diag = i % 2 == 1
            if diag and n > 300:
                continue
            d = os.path.join(td, "t%02d" % i)
            synth.write(synth.c1_spec(n_sites=n, frames=2, seed=40000 + i), d)
            reps = 1 if diag else 8
            env = dict(os.environ, OPENBLAS_NUM_THREADS="1", OMP_NUM_THREADS=str(threads))
            cmd = [exe, os.path.join(d, "Energy.bin"), os.path.join(d, "Coupling.bin"), str(n), "0" if diag else "1",
                   "2", "1", "5", "0", "13500", "16500", str(threads), str(reps)]
            r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, env=env)
            if r.returncode:
                return {"impl": "reference", "unavailable": "ref_bench failed on C4 job %d" % i}
            dd = json.loads(r.stdout.strip().splitlines()[-1])
            per_step[i] = dd["seconds"] / reps  # wall time of one round of `threads` concurrent vector steps
            measured[i] = True
    # Diagonal jobs above 300 sites: a * N^3 fitted on the measured Diagonal jobs above 100 sites
    pts = [(c4_sites()[i], t) for i, t in per_step.items() if i % 2 == 1 and c4_sites()[i] > 100]
    a = statistics.mean(t / n ** 3 for n, t in pts) if pts else None
    total, job_s = 0.0, []
    for i, n in enumerate(c4_sites()):
        t = per_step.get(i, a * n ** 3 if a else float("nan"))
        secs = vec_steps * t / threads  # `threads` vectors propagated concurrently
        job_s.append(secs)
        total += secs
    site_steps = sum(3 * nsamp * tmax * n for n in c4_sites())
    return {"impl": "reference", "config": "c4", "value": site_steps / total, "unit": "site-steps/s",
            "time_to_all_spectra_s": total, "slowest_job_s": max(job_s), "extrapolated": True,
            "cpu_baseline": {"value": site_steps / total, "unit": "site-steps/s", "cores": threads,
                             "kind": "reference",
                             "sample": "per job: %d concurrent vector steps (8 each for Coupling jobs, 1 for "
                                       "Diagonal jobs up to 300 sites; larger Diagonal jobs from the fitted N^3 "
                                       "law), scaled to the job's %d vector steps" % (threads, vec_steps)}}


def run_reference(args):
    if args.config in ("c0", "c2", "c4"):
        if int(os.environ.get("RANK", "0")) != 0:
            return None
        fn = {"c0": run_reference_c0, "c2": run_reference_c2, "c4": run_reference_c4}[args.config]
        out = fn(args)
        print(json.dumps(out), flush=True)
        return out
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return None
    threads = min(host_threads(), 64)
    steps = min(args.steps, 3)  # each timed step is ~30 s of reference CPU time per thread
    with tempfile.TemporaryDirectory() as td:
        write_small_trajectory(td)
        exe = os.path.join(ROOT, "oracle", "_ref", "ref_bench")
        if not os.path.exists(exe):
            out = {"impl": "reference", "unavailable": "oracle/_ref/ref_bench was not built (needs the reference "
                                                       "sources at build time)"}
            print(json.dumps(out), flush=True)
            return out
        for _ in range(args.warmup):  # untimed: pages in the binary and OpenBLAS
            subprocess.run([exe, os.path.join(td, "Energy.bin"), os.path.join(td, "Coupling.bin"), "1024", "1",
                            "2", "1", "5", "0", "13500", "16500", "1", "1"], stdout=subprocess.DEVNULL)
        secs, site = 0.0, 0
        for _ in range(steps):
            d, err = cpu_baseline(td, threads)
            if d is None:
                out = {"impl": "reference", "unavailable": "reference harness failed: %s" % err}
                print(json.dumps(out), flush=True)
                return out
            secs += d["seconds"]
            site += d["site_steps"]
    value = site / secs
    sample = ("%d concurrent vector steps per step (one per host thread) of the reference's propagate_vector "
              "(Sparse, Threshold 0) at N=1024" % threads)
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps,
        "steps_requested": args.steps, "warmup": args.warmup, "ms_per_step": secs / steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded OU trajectory, point-dipole lattice couplings)",
        "config": config_dict(args.frames),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)
    return out


if __name__ == "__main__":
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    elif a.config == "c0":
        run_c0(a)
    elif a.config == "c2":
        run_c2(a)
    elif a.config == "c3":
        run_c3(a)
    elif a.config == "c4":
        run_c4(a)
    else:
        run_ours(a)
