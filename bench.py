"""Benchmark of the plain checkerboard sweep: site updates/s and HBM roofline.

Workload (one "step" = one full checkerboard sweep: director trials and
chirality flips on both colours, run as the library's two fused passes):
  480^3 periodic lattice, eps=1, K=1, h=0, kT=0.3, directors uniform on the
  sphere and chiralities +-1 (Philox seed 11 + rank), d0 = 0.1 with the
  reference's adaptation, FP64 observables every 100 sweeps.  The float4
  lattice is 1.77 GB, far above the 126 MB L2, so no L2 flush is needed.

The line also carries, under "configs", the other benchmark configurations
of the path, each timed on the GPU through the public API and on the host
cores through the oracle port: the 32^3 reference-size run, the 128^3
anneal, the 64^3 differentiation workflow and the batched 64-replica
phase grid against the same points run one after another.

Modes and arms:
  default            the CUDA library, one 480^3 replica per GPU (seed 11 +
                     rank), no collective on the data path: weak scaling
  --mode slab        ONE lattice split into z-slabs, one per rank; each
                     pass stores its boundary planes into the neighbours'
                     halos over peer memory (CUDA IPC) and the per-pass
                     accept counts are summed with NCCL: strong scaling
  --impl reference   the reference algorithm on the host cores (the C
                     oracle port, OpenMP over each colour), each step one
                     sweep of the same 480^3 lattice; rank 0 only.

Prints ONE JSON line (rank 0).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
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
# ncu figures of the fused pass kernels A and B on the 480^3 benchmark lattice
# (one capture of two launches, mean of A and B; profiles/fused_pass_kernel_480cube_metrics.md):
# DRAM bytes read + written per site and launch (A 2653.0 MB, B 2651.2 MB
# for 110.6 M sites), and warp-level instructions x 32 per updated site
# (A 344.8 M, B 339.6 M warp instructions; a launch updates half the sites).
PASS_PROFILE = {"traffic_bytes_per_site": 23.98, "thread_instr_per_updated_site": 198.0,
                "source": "ncu dram__bytes_read+write at 480^3"}
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


# ---------------------------------------------------------------------------
# Clock record of a timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    """SM clock and clock-event reasons while a region runs.

    NVML is polled from a thread every `period` seconds (2 ms: a 20-sweep
    region of the 480^3 workload lasts ~25 ms), plus one sample on entry and
    one on exit; without NVML, nvidia-smi -lms 100 is the fallback.  The GPU
    is found by its PCI bus id, which NVML and CUDA share whatever
    CUDA_VISIBLE_DEVICES says."""

    REASON_BITS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
                   "hw_thermal_slowdown": 0x40, "sw_power_cap": 0x4}
    SMI_FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                  "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                  "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    SMI_REASONS = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, device: int, period: float = 0.002):
        self.device = device
        self.period = period
        self.samples: list[tuple[float, int]] = []  # (sm MHz, reason bits)
        self.sm_max = None
        self.source = None
        self._nvml = None
        self._stop = threading.Event()
        self._thread = None
        self._smi = None
        self._smi_path = None
        self._summary = None

    def _bus_id(self):
        try:
            import torch

            p = torch.cuda.get_device_properties(self.device)
            return f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
        except Exception:  # noqa: BLE001
            return None

    def _sample(self):
        n, h = self._nvml, self._handle
        sm = n.nvmlDeviceGetClockInfo(h, n.NVML_CLOCK_SM)
        reasons = n.nvmlDeviceGetCurrentClocksEventReasons(h)
        self.samples.append((float(sm), int(reasons)))

    def _poll(self):
        while not self._stop.is_set():
            try:
                self._sample()
            except Exception:  # noqa: BLE001
                return
            time.sleep(self.period)

    def __enter__(self):
        bus = self._bus_id()
        try:
            import pynvml as n

            n.nvmlInit()
            self._nvml = n
            self._handle = (n.nvmlDeviceGetHandleByPciBusId(bus) if bus
                            else n.nvmlDeviceGetHandleByIndex(self.device))
            self.sm_max = float(n.nvmlDeviceGetMaxClockInfo(self._handle, n.NVML_CLOCK_SM))
            self.source = "nvml"
            self._sample()
            self._thread = threading.Thread(target=self._poll, daemon=True)
            self._thread.start()
        except Exception:  # noqa: BLE001 - no NVML: nvidia-smi, then nothing
            self._nvml = None
            self._start_smi(bus)
        return self

    def _start_smi(self, bus):
        ClockSampler._count = getattr(ClockSampler, "_count", 0) + 1
        self._smi_path = os.path.join("/tmp", f"chll_clocks_{os.getpid()}_{ClockSampler._count}.csv")
        try:
            self._fh = open(self._smi_path, "w")
            self._smi = subprocess.Popen(
                ["nvidia-smi", f"--id={bus or self.device}", f"--query-gpu={self.SMI_FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self._fh, stderr=subprocess.DEVNULL)
            self.source = "nvidia-smi"
        except Exception:  # noqa: BLE001
            self._smi = None

    def __exit__(self, *exc):
        if self._nvml is not None:
            self._stop.set()
            if self._thread is not None:
                self._thread.join(timeout=5)
            try:
                self._sample()
                self._nvml.nvmlShutdown()
            except Exception:  # noqa: BLE001
                pass
        if self._smi is not None:
            self._smi.terminate()
            try:
                self._smi.wait(timeout=5)
            except Exception:  # noqa: BLE001
                self._smi.kill()
            self._fh.close()

    @classmethod
    def parse_smi_csv(cls, path):
        """(samples [(sm MHz, reason bits)], max SM MHz) of an nvidia-smi CSV."""
        samples, smax = [], None
        for line in open(path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm = float(parts[1])
                smax = float(parts[2])
            except ValueError:
                continue
            bits = 0
            for name, v in zip(cls.SMI_REASONS, parts[5:9]):
                if v.lower() == "active":
                    bits |= cls.REASON_BITS[name]
            samples.append((sm, bits))
        return samples, smax

    def summary(self):
        if self._summary is None:
            if self._smi_path and os.path.exists(self._smi_path):
                self.samples, self.sm_max = self.parse_smi_csv(self._smi_path)
                os.unlink(self._smi_path)
            if not self.samples:
                self._summary = {"sm_mhz": None, "sm_max_mhz": self.sm_max, "reasons": [],
                                 "samples": 0, "source": self.source or "unavailable"}
            else:
                sm = sorted(s for s, _ in self.samples)
                bits = 0
                for _, b in self.samples:
                    bits |= b
                self._summary = {
                    "sm_mhz": sm[len(sm) // 2], "sm_max_mhz": self.sm_max,
                    "reasons": sorted(n for n, m in self.REASON_BITS.items() if bits & m),
                    "samples": len(sm), "source": self.source}
        return self._summary


# ---------------------------------------------------------------------------
# CPU arm: the oracle port of the reference algorithm on the host cores
# ---------------------------------------------------------------------------
def _oracle_lattice(edge, seed=SEED):
    from oracle import oracle as O

    cfg = O.make_cfg(edge, edge, edge, periodic=True, kT=KT, K=KK, g=FIELD, eps=EPS, seed=seed)
    return O, cfg, O.init_random(cfg)


def cpu_sample(nsweeps: int, seconds: float, edge: int = L_EDGE):
    """Reference sweeps of the workload's edge^3 periodic lattice on the host
    cores: `nsweeps` of them (10 at 480^3, about 15 s on 16 cores), stopping
    early once `seconds` have elapsed (at least one sweep)."""
    O, cfg, (nx, ny, nz, s) = _oracle_lattice(edge)
    n = edge ** 3
    sweeps, t0, step = 0, time.perf_counter(), 1
    while True:
        for p in range(4):
            O.run_pass(cfg, p, step, D0, nx, ny, nz, s)
        step += 1
        sweeps += 1
        dt = time.perf_counter() - t0
        if sweeps >= nsweeps or dt >= seconds:
            break
    return {"value": n * sweeps / dt, "unit": UNIT, "cores": O.max_threads(), "kind": "port",
            "sample": f"{sweeps} sweep(s) of the workload's {edge}^3 periodic lattice "
                      f"({n} sites), {dt:.1f} s, FP64 reference arithmetic"}


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    edge = args.edge
    O, cfg, (nx, ny, nz, s) = _oracle_lattice(edge)
    cores = O.max_threads()
    n = edge ** 3
    step = 1
    for _ in range(args.warmup):
        for p in range(4):
            O.run_pass(cfg, p, step, D0, nx, ny, nz, s)
        step += 1
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        for p in range(4):
            O.run_pass(cfg, p, step, D0, nx, ny, nz, s)
        times.append(time.perf_counter() - t0)
        step += 1
    tot = sum(times)
    value = n * args.steps / tot
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": _workload(edge), "lattice": [edge, edge, edge],
                   "sample": f"each step one sweep of the whole {edge}^3 periodic lattice"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{args.steps} sweeps of the {edge}^3 periodic lattice "
                                   f"({n} sites); the reference's Fortran/OpenACC build "
                                   f"needs nvfortran, absent here, so its C restatement runs"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def _workload(edge):
    return WORKLOAD if edge == L_EDGE else WORKLOAD.replace(f"{L_EDGE}^3", f"{edge}^3")


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def _dist_init(torch, local):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world <= 1:
        return None
    import datetime

    import torch.distributed as dist

    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                            device_id=torch.device("cuda", local))
    return dist


def gpu_arm(args):
    import numpy as np
    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = _dist_init(torch, local)

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
    clk = clocks.summary()

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
        with ClockSampler(local, period=0.05) as e2e_clocks:
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

    configs = {}
    if rank == 0 and world == 1 and not args.no_configs:
        configs = other_configs(args, torch)
    if not args.no_batched:
        configs["batched_64_replicas"] = batched_vs_plain(args, rank, torch)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_sample(args.cpu_sweeps, args.cpu_seconds, edge)

    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    # Issue roofline: every SM issues at most one warp instruction per cycle
    # and scheduler (4 per SM), so a pass updating n/2 sites at I thread
    # instructions each can update at most SMs * 4 * 32 * f / I sites per second.
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    instr = PASS_PROFILE["thread_instr_per_updated_site"]
    f_hz = (clk["sm_mhz"] or clk["sm_max_mhz"] or 1965.0) * 1e6
    issue_ceiling = sms * 4 * 32 * f_hz / instr
    updated_per_s = (n / 2) / (pass_ms * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: directors uniform on the sphere, chiralities +-1 p=1/2 "
                "(Philox seed 11 + rank); state FP32, observables FP64",
        "config": {"workload": _workload(edge), "lattice": [edge, edge, edge],
                   "boundary": "periodic", "kT": KT, "K": KK, "h": FIELD, "eps": EPS,
                   "d0": D0, "nout": NOUT,
                   "measurements_in_timed_region": sum(
                       1 for t in range(step0, step0 + args.steps) if t % NOUT == 0),
                   "measurement_note": f"a measurement every {NOUT} sweeps, counted by sweep "
                                       f"number: a region of fewer sweeps may hold none; the "
                                       f"e2e leg's {max(args.e2e_sweeps, NOUT)} sweeps hold "
                                       f"their share",
                   "parallelism": f"replicas x{world}",
                   "l2": f"lattice {16 * n / 1e9:.2f} GB vs 126 MB L2; no flush"},
        "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": peak, "unit": "GB/s",
                     "frac": achieved_gbs / peak,
                     "traffic": PASS_PROFILE["traffic_bytes_per_site"] * n / 1e9,
                     "traffic_unit": f"GB per launch ({PASS_PROFILE['source']})",
                     "kernel": "fused_pass_kernel A and B (2 launches per step)",
                     "bytes_per_launch": BYTES_PER_SITE_PASS * n,
                     "ms_per_launch": pass_ms, "ms_pass_a": a_ms / args.steps,
                     "ms_pass_b": b_ms / args.steps, "peak_kind": peak_kind,
                     "instructions_per_site": instr,
                     "issue_frac": updated_per_s / issue_ceiling,
                     "issue_note": "updated sites/s over SMs x 4 schedulers x 32 lanes x "
                                   "median sampled SM clock / thread instructions per updated "
                                   "site: the limiter of these passes"},
        "reference_form": {
            "note": "the reference's four half-sweeps move 96 B per site and sweep; the fused "
                    "form does the same trials in two passes of 24 B per site",
            "equiv_gbs_at_96_B_per_site_sweep": 4 * BYTES_PER_SITE_PASS * n / (ms * 1e-3)
            * args.steps / 1e9},
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": launches,
        "clocks": clk,
        "configs": configs,
        "final_control": ctl,
        "last_row": {"energy_per_site": float(rows[-1][5] / n) if len(rows) else None,
                     "eta": float(rows[-1][1]) if len(rows) else None},
    }
    print(json.dumps(line), flush=True)
    return 0


def _events(torch):
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def other_configs(args, torch):
    """The path's other benchmark configurations, each on the GPU through the
    public API and on the host cores through the oracle port."""
    import numpy as np

    from chllmodel_b200 import chll
    from chllmodel_b200.lattice import Lattice, coupling
    from chllmodel_b200.workflows import anneal, linear_schedule
    from oracle import oracle as O

    out = {}
    cores = O.max_threads()

    # 32^3, K=0.5, h=0, kT=0.5, seed 1, 1000 sweeps with a row every 100:
    # ChLLSim.run through chll_run_ex, host arrays, wall time of the call.
    e = 32
    lat = Lattice(e, e, e, boundary="periodic")
    lat.init_random(1)
    state = lat.download_f64()
    lat.close()
    sim = chll.ChLLSim(e, e, e, 0.5, 0.1, 0.5, 0.0, 0.0, seed=1, boundary="periodic",
                       verbose=False)
    runs = []
    for r in range(4):  # the first call captures the graph
        sim.nx[...], sim.ny[...], sim.nz[...], sim.s[...] = state
        sim.d = 0.1
        runs.append(sim.run(1000, 100))
    t_gpu = float(np.median(runs[1:]))
    cfg = O.make_cfg(e, e, e, periodic=True, kT=0.5, K=0.5, g=0.0, seed=1)
    ox, oy, oz, os_ = (np.asfortranarray(a) for a in state)
    t0 = time.perf_counter()
    O.run(cfg, 1, 1000, 100, 0.1, ox, oy, oz, os_)
    t_cpu = time.perf_counter() - t0
    out["plain_32"] = {
        "workload": "32^3 periodic, K=0.5, h=0, kT=0.5, d0=0.1, seed 1, 1000 sweeps, a "
                    "measurement row every 100 (ChLLSim.run, host FP64 arrays)",
        "seconds": t_gpu, "site_updates_per_s": e ** 3 * 1000 / t_gpu,
        "cpu_seconds": t_cpu, "cpu_site_updates_per_s": e ** 3 * 1000 / t_cpu,
        "cpu_cores": cores, "speedup_vs_cpu": t_cpu / t_gpu,
        "final_d": sim.d, "final_row": [float(x) for x in sim.m[-1]]}

    # 128^3 anneal: K=1, h=0.25, seed 7, kT 1.5 -> 0.1 in 20 stages of 500
    # sweeps, FP64 rows every 10 sweeps (workflows.anneal).
    e = 128
    lat = Lattice(e, e, e, boundary="periodic")
    sched = linear_schedule(1.5, 0.1, 20)
    for rep in range(2):  # the first pass captures the graphs
        lat.init_random(7)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        stages = anneal(lat, sched if rep else sched[:1], 500, K=1.0, g=0.25, seed=7,
                        measure_every=10, d0=0.1)
        lat.sync()
        t_gpu = time.perf_counter() - t0
    lat.close()
    cfg = O.make_cfg(e, e, e, periodic=True, kT=1.5, K=1.0, g=0.25, seed=7)
    ox, oy, oz, os_ = O.init_random(cfg)
    ncpu = 100
    t0 = time.perf_counter()
    for st in range(1, ncpu + 1):
        for p in range(4):
            O.run_pass(cfg, p, st, 0.1, ox, oy, oz, os_)
    t_cpu = (time.perf_counter() - t0) * 10000 / ncpu
    out["anneal_128"] = {
        "workload": "128^3 periodic, K=1, h=0.25, seed 7, kT 1.5 -> 0.1 linear in 20 stages of "
                    "500 sweeps, FP64 rows every 10 sweeps (workflows.anneal)",
        "seconds": t_gpu, "site_updates_per_s": e ** 3 * 10000 / t_gpu,
        "cpu_seconds_extrapolated": t_cpu, "cpu_sample": f"{ncpu} sweeps at kT=1.5, scaled to "
                                                          f"10000", "cpu_cores": cores,
        "speedup_vs_cpu": t_cpu / t_gpu,
        "last_stage": {k: stages[-1][k] for k in ("kT", "energy", "eta", "S", "C_v", "chi_c")}}

    # 64^3 differentiation: 500-sweep equilibration at kT=0.3, K=1, h=0.5
    # (seed 3), the energy adjoint (dE/dn and dE/d(eps, K, h)), a 2000-step
    # zero-temperature gradient quench.
    e = 64
    stream = torch.cuda.Stream()  # not the default stream, whose handle 0 means the lattice's own
    lat = Lattice(e, e, e, boundary="periodic")
    lat.set_stream(stream.cuda_stream)
    lat.init_random(3)
    lat.set_control(0.1, step=1)
    cpe = coupling(0.3, 1.0, 0.5)
    lat.sweep(cpe, 10, seed=3)  # graph capture
    lat.init_random(3)
    lat.set_control(0.1, step=1)
    a, b = _events(torch)
    a.record(stream)
    lat.sweep(cpe, 500, seed=3)
    b.record(stream)
    b.synchronize()
    t_eq = a.elapsed_time(b) * 1e-3
    with torch.cuda.stream(stream):
        grad = torch.empty((e ** 3, 4), dtype=torch.float32, device="cuda")
    cpq = coupling(0.0, 1.0, 0.5)
    lat.energy_grad(cpq, project=True, grad_ptr=grad.data_ptr())  # allocation
    reps = 20
    a.record(stream)
    for _ in range(reps):
        _, out4 = lat.energy_grad(cpq, project=True, grad_ptr=grad.data_ptr())
    b.record(stream)
    b.synchronize()
    t_adj = a.elapsed_time(b) * 1e-3 / reps
    x, y, z, s = lat.download_f64()
    e_before = float(out4[0])
    lat.quench(cpq, 0.05, 2)
    lat.sync()
    a.record(stream)
    lat.quench(cpq, 0.05, 2000)
    b.record(stream)
    b.synchronize()
    t_q = a.elapsed_time(b) * 1e-3
    _, out4q = lat.energy_grad(cpq)
    lat.close()
    cfg = O.make_cfg(e, e, e, periodic=True, kT=0.0, K=1.0, g=0.5, seed=3)
    ox, oy, oz, os_ = (np.asfortranarray(v) for v in (x, y, z, s))
    t0 = time.perf_counter()
    O.energy_grad(cfg, ox, oy, oz, os_, project=True)
    t_cadj = time.perf_counter() - t0
    cfg = O.make_cfg(e, e, e, periodic=True, kT=0.3, K=1.0, g=0.5, seed=3)
    t0 = time.perf_counter()
    for st in range(1, 51):
        for p in range(4):
            O.run_pass(cfg, p, st, 0.1, ox, oy, oz, os_)
    t_ceq = (time.perf_counter() - t0) * 10
    out["differentiation_64"] = {
        "workload": "64^3 periodic, 500-sweep equilibration at kT=0.3, K=1, h=0.5 (seed 3); "
                    "energy adjoint (tangent-projected dE/dn, dE/d(eps,K,h)); 2000-step "
                    "gradient quench at kT=0, step 0.05",
        "equilibration_seconds": t_eq, "equilibration_site_updates_per_s": e ** 3 * 500 / t_eq,
        "adjoint_ms": t_adj * 1e3, "quench_seconds": t_q,
        "quench_site_steps_per_s": e ** 3 * 2000 / t_q,
        "energy_before_quench": e_before, "energy_after_quench": float(out4q[0]),
        "cpu_adjoint_ms": t_cadj * 1e3, "cpu_equilibration_seconds_extrapolated": t_ceq,
        "cpu_cores": cores}
    return out


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
        paired = None if args.batched_pairs < 0 else bool(args.batched_pairs)
        pooled = None if args.batched_pooled < 0 else bool(args.batched_pooled)
        b.set_tuning(t, c, args.batched_wave_mb << 20, paired, pooled)
        tune = {"threads": t, "ctas_per_sm": c, "wave_bytes": args.batched_wave_mb << 20,
                "paired": b.tuning()["paired"], "pooled": b.tuning()["pooled"],
                "trial_ms": None}
    else:
        tune = b.autotune(trial_sweeps=200)
    b.run(nsw, measure_every=BATCH_NOUT)   # warm-up: graph capture and first launch
    b.sync()
    b.close()
    b = Batch(specs)
    b.set_stream(stream.cuda_stream)
    b.init_random()
    b.set_tuning(tune["threads"], tune["ctas_per_sm"], tune["wave_bytes"], tune["paired"],
                 tune["pooled"])
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

    # The same points one after another: the plain kernels launched pass by
    # pass ("fused", the comparison the batched launch is measured against),
    # and the library's default form per point ("auto": the resident cluster
    # launch for the 32^3 points, the fused passes for the others).
    t_seq = {"fused": float("nan"), "auto": float("nan")}
    for kind, sp in [(k, sp) for k in t_seq for sp in ([] if args.no_plain_grid else specs)]:
        if t_seq[kind] != t_seq[kind]:
            t_seq[kind] = 0.0
        lat = Lattice(sp["ni"], sp["nj"], sp["nk"], boundary=sp["boundary"])
        lat.set_stream(stream.cuda_stream)
        lat.set_kernel(kind)
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
        t_seq[kind] += a0.elapsed_time(a1) * 1e-3
        lat.close()
    t_plain = t_seq["fused"]
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
            "sequential_default_form_s": t_seq["auto"],
            "speedup_vs_sequential_default_form": t_seq["auto"] / t_batched,
            "sequential_chllsim_s": t_sim,
            "speedup_vs_sequential_chllsim": t_sim / t_batched,
            "site_updates_per_s": total * nsw / t_batched,
            "tuning": dict({k: tune[k] for k in ("threads", "ctas_per_sm", "paired", "pooled",
                                                 "trial_ms")},
                           **{"waves": info_tune["waves"],
                              "wave_MiB": info_tune["wave_bytes"] / 2 ** 20}),
            "grid_ctas": info["grid"],
            "mean_S_lowest_kT": float(np.mean([r["S"] for r in summ if r["kT"] < 0.2])),
            "mean_S_highest_kT": float(np.mean([r["S"] for r in summ if r["kT"] > 1.9]))}


# ---------------------------------------------------------------------------
# Slab mode: one lattice split over the ranks
# ---------------------------------------------------------------------------
def slab_arm(args):
    """One edge^3 periodic lattice in z-slabs, one per rank.  Every pass
    stores the slab's boundary planes into the neighbours' halo planes over
    peer memory (CUDA IPC mappings; a single rank is its own neighbour) and
    the per-pass counts are summed with NCCL, which also orders the passes
    across ranks.  Timed: the sweeps with their closing flip pass, halo
    stores and count all-reduces, on the device (CUDA events), max over ranks."""
    import numpy as np
    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world == 1:  # a one-rank group: the slab's halos are its own planes
        import socket

        with socket.socket() as s:
            s.bind(("127.0.0.1", 0))
            os.environ.setdefault("MASTER_PORT", str(s.getsockname()[1]))
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("RANK", "0")
        os.environ.setdefault("WORLD_SIZE", "1")
    import datetime

    import torch.distributed as dist

    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                            device_id=torch.device("cuda", local))
    from chllmodel_b200.lattice import coupling
    from chllmodel_b200.slab import SlabLattice, TorchPeerHalo, split_planes, sweep_slabs

    edge = args.edge
    n = edge ** 3
    z0, nkl = split_planes(edge, world)[rank]
    cp = coupling(KT, KK, FIELD, EPS)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        sl = SlabLattice(edge, edge, edge, z0, nkl, boundary="periodic")
        sl.init_random(SEED)
        sl.set_control(D0, step=1)
        halo = TorchPeerHalo.for_slab(sl)
        sweep_slabs([sl], halo, cp, args.warmup, seed=SEED)
        torch.cuda.synchronize()
        dist.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clocks:
            e0.record(stream)
            sweep_slabs([sl], halo, cp, args.steps, seed=SEED)
            e1.record(stream)
            e1.synchronize()
        ms = e0.elapsed_time(e1)
        ctl = sl.control()
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t[0])
        halo.close()
        sl.close()
    torch.cuda.synchronize()
    dist.barrier()
    dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": n * args.steps / (ms * 1e-3), "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: directors uniform on the sphere, chiralities +-1 p=1/2 (Philox "
                "seed 11); state FP32",
        "config": {"workload": f"one {edge}^3 periodic lattice in {world} z-slab(s), the "
                               f"{_workload(edge)} minus its measurements",
                   "mode": "slab", "lattice": [edge, edge, edge],
                   "slab_planes": [list(p) for p in split_planes(edge, world)],
                   "transport": "boundary planes stored into the neighbours' halos by the "
                                "passes (CUDA IPC peer memory), counts summed with NCCL",
                   "parallelism": f"z-slabs x{world}",
                   "l2": f"lattice {16 * n / 1e9:.2f} GB vs 126 MB L2; no flush"},
        "e2e": None, "e2e_note": "slab mode times device-resident sweeps only",
        "gpu_launches": None, "clocks": clocks.summary(), "final_control": ctl,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--mode", default="replicas", choices=["replicas", "slab"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-sweeps", type=int, default=E2E_SWEEPS,
                    help="sweeps of the end-to-end ChLLSim.run (default: the workload's 10000)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the 32^3, 128^3 anneal and 64^3 differentiation configurations")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--batched-sweeps", type=int, default=2000)
    ap.add_argument("--batched-shape", default="",
                    help="THREADSxCTAS_PER_SM for the batched launch instead of autotuning")
    ap.add_argument("--batched-wave-mb", type=int, default=0,
                    help="wave size with --batched-shape (0: all replicas in one wave)")
    ap.add_argument("--batched-pooled", type=int, default=-1,
                    help="with --batched-shape: 1 pooled passes, 0 the persistent launch "
                         "(default: the library's)")
    ap.add_argument("--batched-pairs", type=int, default=-1,
                    help="with --batched-shape: 1 replica groups of two alternating replicas, "
                         "0 one replica per group (default: the library's)")
    ap.add_argument("--no-plain-grid", action="store_true",
                    help="skip the sequential plain-kernel grid (profiling runs)")
    ap.add_argument("--cpu-sweeps", type=int, default=10)
    ap.add_argument("--cpu-seconds", type=float, default=30.0)
    ap.add_argument("--edge", type=int, default=L_EDGE,
                    help="lattice edge (480 is the benchmark; smaller edges for profiling)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return reference_arm(args)
    if args.mode == "slab":
        return slab_arm(args)
    return gpu_arm(args)


if __name__ == "__main__":
    sys.exit(main())
