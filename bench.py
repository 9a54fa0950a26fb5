"""Benchmark of the plain checkerboard sweep: site updates/s and HBM roofline.

Workload (one "step" = one full checkerboard sweep: director trials and
chirality flips on both colours, run as the library's two fused passes):
  480^3 periodic lattice, eps=1, K=1, h=0, kT=0.3, directors uniform on the
  sphere and chiralities +-1 (Philox seed 11 + rank), d0 = 0.1 with the
  reference's adaptation, FP64 observables every 100 sweeps.  The float4
  lattice is 1.77 GB, far above the 126 MB L2, so no L2 flush is needed.

Arms:
  default            the CUDA library (one process per GPU, independent
                     replicas, no collective on the data path: weak scaling)
  --impl reference   the reference algorithm on the host cores (the C oracle
                     port, OpenMP), each step one sweep of a bounded slab of
                     the same lattice; rank 0 only.

Prints ONE JSON line (rank 0).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

L_EDGE = 480
KT, KK, FIELD, EPS, D0, SEED = 0.3, 1.0, 0.0, 1.0, 0.1, 11
NOUT = 100
E2E_SWEEPS = 10000  # the 480^3 workload's run length (observables every NOUT sweeps)
# FP64 measurements of the batched grid every BATCH_NOUT sweeps in both arms,
# as the reference's phase-diagram driver runs its 64^3 grid points
# (scripts/phase_diagram.py:30, sim.run(200000, 50)).
BATCH_NOUT = 50
BYTES_PER_SITE_PASS = 24  # 16 B read (every site once) + 8 B written (half the sites)
# DRAM read + write per site and launch of the fused pass kernels, measured
# with ncu (dram__bytes_read.sum + dram__bytes_write.sum, mean of passes A and
# B) on a 256^3 launch and scaled by sites to 480^3: 372.3 MB (A) and
# 372.2 MB (B) per launch of 16.78 M sites.
TRAFFIC_BYTES_PER_SITE_PASS = 22.19
METRIC = "site_updates_per_s"
UNIT = "site-updates/s"
WORKLOAD = (f"plain {L_EDGE}^3 periodic checkerboard sweep (director + chirality Metropolis), "
            f"eps=1 K=1 h=0 kT=0.3, FP64 observables every {NOUT} sweeps")


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    _count = 0

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        ClockSampler._count += 1  # one file per sampler: several may be summarised late
        self.path = os.path.join("/tmp", f"chll_clocks_{os.getpid()}_{ClockSampler._count}.csv")
        self._summary = None

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:  # noqa: BLE001 - no nvidia-smi
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:  # noqa: BLE001
                self.proc.kill()
        if getattr(self, "fh", None):
            self.fh.close()

    def summary(self):
        if self._summary is None:
            self._summary = self._read()
        return self._summary

    def _read(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU arm: the oracle port of the reference algorithm on the host cores
# ---------------------------------------------------------------------------
def cpu_sample(seconds: float, threads: int | None = None, nz: int = 8):
    """Times reference sweeps of a 480 x 480 x nz periodic slab of the workload
    on the host cores until `seconds` have elapsed (at least one sweep)."""
    from oracle import oracle as O

    if threads:
        O.set_threads(threads)
    cores = O.max_threads()
    cfg = O.make_cfg(L_EDGE, L_EDGE, nz, periodic=True, kT=KT, K=KK, g=FIELD, eps=EPS,
                     seed=SEED)
    nx, ny, nz_, s = O.init_random(cfg)
    n = L_EDGE * L_EDGE * nz
    sweeps, t0, step = 0, time.perf_counter(), 1
    while True:
        for p in range(4):
            O.run_pass(cfg, p, step, D0, nx, ny, nz_, s)
        step += 1
        sweeps += 1
        dt = time.perf_counter() - t0
        if dt >= seconds:
            break
    return {"value": n * sweeps / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{sweeps} sweep(s) of a {L_EDGE}x{L_EDGE}x{nz} periodic slab "
                      f"({n} sites) of the workload, {dt:.1f} s, FP64 reference arithmetic"}


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import oracle as O

    cores = O.max_threads()
    nz = 8
    cfg = O.make_cfg(L_EDGE, L_EDGE, nz, periodic=True, kT=KT, K=KK, g=FIELD, eps=EPS, seed=SEED)
    nx, ny, nz_, s = O.init_random(cfg)
    n = L_EDGE * L_EDGE * nz
    step = 1
    for _ in range(args.warmup):
        for p in range(4):
            O.run_pass(cfg, p, step, D0, nx, ny, nz_, s)
        step += 1
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        for p in range(4):
            O.run_pass(cfg, p, step, D0, nx, ny, nz_, s)
        times.append(time.perf_counter() - t0)
        step += 1
    tot = sum(times)
    value = n * args.steps / tot
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "lattice": [L_EDGE, L_EDGE, L_EDGE],
                   "sample": f"each step one sweep of a {L_EDGE}x{L_EDGE}x{nz} periodic slab"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{args.steps} sweeps of a {L_EDGE}x{L_EDGE}x{nz} periodic "
                                   f"slab ({n} sites); the reference's Fortran/OpenACC build "
                                   f"needs nvfortran, absent here, so its C restatement runs"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def gpu_arm(args):
    import numpy as np
    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    from chllmodel_b200 import chll
    from chllmodel_b200.lattice import FUSED_A, FUSED_A0, FUSED_B, FUSED_F, Lattice, coupling

    edge = args.edge
    n = edge ** 3
    cp = coupling(KT, KK, FIELD, EPS)
    stream = torch.cuda.Stream()
    lat = Lattice(edge, edge, edge, boundary="periodic")
    lat.set_stream(stream.cuda_stream)
    lat.init_random(SEED + rank)
    lat.set_control(D0, step=1)
    nmeas = (args.steps + args.warmup) // NOUT + 2
    lat.reserve_rows(nmeas)

    # One step = one sweep in the library's fused form (chll_lattice_sweep's
    # graph holds the same launches): pass A (A0 after a closed step) and
    # pass B per sweep, the closing colour-0 flip pass F before each FP64
    # measurement and after the last sweep.  Every A/B launch is bracketed by
    # CUDA events on its stream: their mean is the roofline's launch time.
    class Runner:
        """Issues sweeps as fused passes and FP64 measurements into row slots."""

        def __init__(self):
            self.slot = 0  # last row slot written

        def sweeps(self, count, first_step, events=None):
            pending, nl = False, 0
            for i in range(count):
                e = None
                if events is not None:
                    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
                    e[0].record(stream)
                lat.half_sweep(cp, FUSED_A if pending else FUSED_A0, seed=SEED, replica=rank)
                if e:
                    e[1].record(stream)
                lat.half_sweep(cp, FUSED_B, seed=SEED, replica=rank)
                if e:
                    e[2].record(stream)
                    events.append(e)
                nl += 2
                pending = True
                meas = (first_step + i) % NOUT == 0
                if meas or i == count - 1:
                    lat.half_sweep(cp, FUSED_F, seed=SEED, replica=rank)
                    nl += 1
                    pending = False
                if meas:
                    self.slot += 1
                    lat.measure(cp, self.slot)
                    nl += 1
            return nl

    runner = Runner()
    with torch.cuda.stream(stream):
        runner.sweeps(args.warmup, 1)
    lat.sync()
    step0 = args.warmup + 1

    ev_start = torch.cuda.Event(enable_timing=True)
    ev_end = torch.cuda.Event(enable_timing=True)
    pass_events = []
    barrier()
    with ClockSampler(local) as clocks:
        ev_start.record(stream)
        slot_first = runner.slot + 1
        launches = runner.sweeps(args.steps, step0, pass_events)
        ev_end.record(stream)
        ev_end.synchronize()
    barrier()
    slot = runner.slot
    ms = ev_start.elapsed_time(ev_end)
    a_ms = sum(e[0].elapsed_time(e[1]) for e in pass_events)
    b_ms = sum(e[1].elapsed_time(e[2]) for e in pass_events)
    t = torch.tensor([ms, a_ms, b_ms], device="cuda", dtype=torch.float64)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms, a_ms, b_ms = float(t[0]), float(t[1]), float(t[2])
    value = world * n * args.steps / (ms * 1e-3)
    pass_ms = (a_ms + b_ms) / (2 * args.steps)
    achieved_gbs = BYTES_PER_SITE_PASS * n / (pass_ms * 1e-3) / 1e9
    peak, peak_kind = _peaks()
    ctl = lat.control()
    rows = lat.read_rows(slot_first, slot - slot_first + 1) if slot >= slot_first \
        else np.zeros((0, 16))
    lat.close()
    del lat

    # e2e: the public API with host buffers (pinned), copies inside the timed region
    e2e = None
    if not args.no_e2e:
        sim = chll.ChLLSim(edge, edge, edge, KT, D0, KK, FIELD, 0.0, seed=SEED + rank,
                           boundary="periodic", verbose=False)
        pin = lambda dt: torch.empty((edge,) * 3, dtype=dt, pin_memory=True).numpy().T
        sim.nx, sim.ny, sim.nz = pin(torch.float64), pin(torch.float64), pin(torch.float64)
        sim.s, sim.dope = pin(torch.int32), pin(torch.int32)
        st = Lattice(edge, edge, edge, boundary="periodic")
        st.init_random(SEED + rank)
        x, y, z, sp = st.download_f64()
        st.close()
        sim.nx[...], sim.ny[...], sim.nz[...], sim.s[...] = x, y, z, sp
        del x, y, z, sp
        nsw = max(args.e2e_sweeps, NOUT)
        sim.run(NOUT, NOUT)  # warm-up: allocations and graph capture
        barrier()
        with ClockSampler(local) as e2e_clocks:
            t0 = time.perf_counter()
            sim.run(nsw, NOUT)
            dt = time.perf_counter() - t0
        tt = torch.tensor([dt], device="cuda", dtype=torch.float64)
        if dist is not None:
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        dt = float(tt[0])
        h2d = n * (3 * 8 + 4)
        d2h = n * (3 * 8 + 4) + sim.rows.nbytes
        e2e = {"value": world * n * nsw / dt, "unit": UNIT,
               "h2d_bytes_per_step": h2d / nsw, "d2h_bytes_per_step": d2h / nsw,
               "sweeps": nsw, "api": "ChLLSim.run -> chll_run_ex (C ABI), pinned FP64 host "
                                     "arrays, upload + pack + sweeps + measurements + unpack + "
                                     "download",
               "clocks": e2e_clocks.summary()}

    batched = None
    if not args.no_batched:
        batched = batched_vs_plain(args, rank, torch)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_sample(args.cpu_seconds)

    clk = clocks.summary()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: directors uniform on the sphere, chiralities +-1 p=1/2 "
                "(Philox seed 11 + rank); state FP32, observables FP64",
        "config": {"workload": WORKLOAD if edge == L_EDGE else WORKLOAD.replace(
                       f"{L_EDGE}^3", f"{edge}^3"), "lattice": [edge, edge, edge],
                   "boundary": "periodic", "kT": KT, "K": KK, "h": FIELD, "eps": EPS,
                   "d0": D0, "nout": NOUT, "parallelism": f"replicas x{world}",
                   "l2": f"lattice {16 * n / 1e9:.2f} GB vs 126 MB L2; no flush"},
        "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": peak, "unit": "GB/s",
                     "frac": achieved_gbs / peak,
                     "traffic": (TRAFFIC_BYTES_PER_SITE_PASS * n / 1e9
                                 if TRAFFIC_BYTES_PER_SITE_PASS else None),
                     "traffic_unit": "GB per launch (ncu, 256^3 launch scaled by sites)",
                     "kernel": "fused_pass_kernel A and B (2 launches per step)",
                     "bytes_per_launch": BYTES_PER_SITE_PASS * n,
                     "limiter": "instruction issue (ncu on 256^3: ~245 instructions per site, "
                                "issue 65-66%, DRAM 46-47%, load waits hidden by an L1 prefetch); "
                                "bytes are the algorithmic 24 B/site",
                     "ms_per_launch": pass_ms, "ms_pass_a": a_ms / args.steps,
                     "ms_pass_b": b_ms / args.steps, "peak_kind": peak_kind,
                     "four_half_sweep_equiv_gbs": 4 * BYTES_PER_SITE_PASS * n / (ms * 1e-3)
                     * args.steps / 1e9},
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": launches,
        "clocks": clk,
        "batched": batched,
        "final_control": ctl,
        "last_row": {"energy_per_site": float(rows[-1][5] / n) if len(rows) else None,
                     "eta": float(rows[-1][1]) if len(rows) else None},
    }
    print(json.dumps(line), flush=True)
    return 0


def batched_vs_plain(args, rank, torch):
    """Phase-diagram grid: 64 replicas (kT on 8 points in 0.1-2.0 x h on 8 points
    in 0.0-3.0, K=1, edges drawn from {32, 48, 64}, seed 1 + replica) for
    `batched_sweeps` sweeps with FP64 measurements every BATCH_NOUT sweeps, as
    one persistent launch versus the same points run one after another with the
    plain kernels (graph-captured BATCH_NOUT-sweep chunks + a measurement each)."""
    import numpy as np

    from chllmodel_b200.batched import Batch, phase_grid
    from chllmodel_b200.lattice import Lattice, coupling

    nsw = args.batched_sweeps
    specs = phase_grid(np.linspace(0.1, 2.0, 8), np.linspace(0.0, 3.0, 8), [32, 48, 64],
                       K=1.0, seed=1 + 1000 * rank, size_seed=12345)
    stream = torch.cuda.Stream()
    b = Batch(specs)
    b.set_stream(stream.cuda_stream)
    b.init_random()
    if args.batched_shape:
        t, c = (int(x) for x in args.batched_shape.split("x"))
        b.set_tuning(t, c, args.batched_wave_mb << 20)
        tune = {"threads": t, "ctas_per_sm": c, "wave_bytes": args.batched_wave_mb << 20,
                "trial_ms": None}
    else:
        tune = b.autotune(trial_sweeps=200)
    b.run(nsw, measure_every=BATCH_NOUT)   # warm-up: graph capture and first launch
    b.sync()
    b.close()
    b = Batch(specs)
    b.set_stream(stream.cuda_stream)
    b.init_random()
    b.set_tuning(tune["threads"], tune["ctas_per_sm"], tune["wave_bytes"])
    b.sync()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.run(nsw, measure_every=BATCH_NOUT)
    e1.record(stream)
    e1.synchronize()
    t_batched = e0.elapsed_time(e1) * 1e-3
    summ = b.summary()
    info = b.info()
    info_tune = b.tuning()
    b.close()

    t_plain = float("nan")
    for sp in ([] if args.no_plain_grid else specs):
        if t_plain != t_plain:
            t_plain = 0.0
        lat = Lattice(sp["ni"], sp["nj"], sp["nk"], boundary=sp["boundary"])
        lat.set_stream(stream.cuda_stream)
        lat.init_random(sp["seed"], sp["replica"])
        lat.set_control(sp["d"], step=1)
        lat.reserve_rows(nsw // BATCH_NOUT + 1)
        cp = coupling(sp["kT"], sp["K"], sp["g"], sp["eps"])
        lat.sweep(cp, BATCH_NOUT, seed=sp["seed"], replica=sp["replica"])  # capture the graph
        lat.sync()
        lat.init_random(sp["seed"], sp["replica"])
        lat.set_control(sp["d"], step=1)
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        for c in range(nsw // BATCH_NOUT):
            lat.sweep(cp, BATCH_NOUT, seed=sp["seed"], replica=sp["replica"])
            lat.measure(cp, c)
        a1.record(stream)
        a1.synchronize()
        t_plain += a0.elapsed_time(a1) * 1e-3
        lat.close()
    # The same points as the reference's phase-diagram driver runs them: one
    # ChLLSim per point, run(nsweeps, BATCH_NOUT) through the C ABI with host
    # arrays (scripts/phase_diagram.py:25-31), wall time of each run summed.
    t_sim = float("nan")
    if not args.no_plain_grid:
        from chllmodel_b200 import chll

        t_sim = 0.0
        for sp in specs:
            sim = chll.ChLLSim(sp["ni"], sp["nj"], sp["nk"], sp["kT"], sp["d"], sp["K"], sp["g"],
                               0.0, seed=sp["seed"], boundary=sp["boundary"], epsilon=sp["eps"],
                               verbose=False)
            sim.init_random_directors(np.random.default_rng(sp["seed"]))
            sim.init_rand_s()
            t_sim += sim.run(nsw, BATCH_NOUT)
    total = info["total_sites"]
    return {"workload": "64 replicas, edges {32,48,64}^3, kT x h grid 8x8, K=1, "
                        f"{nsw} sweeps, FP64 measurements every {BATCH_NOUT} sweeps",
            "replicas": len(specs), "total_sites": total, "sweeps": nsw,
            "time_to_grid_s": t_batched, "sequential_plain_s": t_plain,
            "speedup_vs_sequential_plain": t_plain / t_batched,
            "sequential_chllsim_s": t_sim,
            "speedup_vs_sequential_chllsim": t_sim / t_batched,
            "site_updates_per_s": total * nsw / t_batched,
            "tuning": dict({k: tune[k] for k in ("threads", "ctas_per_sm", "trial_ms")},
                           **{"waves": info_tune["waves"],
                              "wave_MiB": info_tune["wave_bytes"] / 2 ** 20}),
            "grid_ctas": info["grid"],
            "mean_S_lowest_kT": float(np.mean([r["S"] for r in summ if r["kT"] < 0.2])),
            "mean_S_highest_kT": float(np.mean([r["S"] for r in summ if r["kT"] > 1.9]))}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-sweeps", type=int, default=E2E_SWEEPS,
                    help="sweeps of the end-to-end ChLLSim.run (default: the workload's 10000)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--batched-sweeps", type=int, default=2000)
    ap.add_argument("--batched-shape", default="",
                    help="THREADSxCTAS_PER_SM for the batched launch instead of autotuning")
    ap.add_argument("--batched-wave-mb", type=int, default=0,
                    help="wave size with --batched-shape (0: all replicas in one wave)")
    ap.add_argument("--no-plain-grid", action="store_true",
                    help="skip the sequential plain-kernel grid (profiling runs)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--edge", type=int, default=L_EDGE,
                    help="lattice edge (480 is the benchmark; smaller edges for profiling)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return reference_arm(args)
    return gpu_arm(args)


if __name__ == "__main__":
    sys.exit(main())
