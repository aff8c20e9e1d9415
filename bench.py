"""Benchmark of the HiDEM hot path: particle-steps/s on the 5.7M-particle calving slab.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision mixed|fp64]
                    [--impl ours|reference] [--workload slab|block|ensemble|settle|topo|mesh|ranks]
                    [--kernel auto|items|thread|thread-capped|thread-async|two-pass]

A "step" is one timestep of the sample main loop (gridService, forces, integrate, link
update) over the whole slab. `value` times K steps with the state resident in HBM (CUDA
events on the library's stream, max over ranks). `e2e` times the same K steps through the
C ABI from host arrays: upload of the particle and link state, the K steps, download of
the particle state. `roofline` divides the byte model of the step by the event-timed
duration of the step's kernels (the force, integrate and break passes of the two-pass
step, or the one kernel of a fused step). `cpu_baseline` times the reference's own CPU path
(oracle/_ref, built from its sources with its own flags) on the same slab. The mixed-precision
slab line also carries `rebuild_amortised` (the configuration's 2000-step run from step 0,
its rebuilds included), `fp64` (the same slab in the plain FP64 build) and `settle` (the
learned warm start's settling steps, cold against surrogate-seeded).
With --gpus N > 1 (torchrun) the slab is decomposed into N x-slabs, one per GPU, with the
halo force exchange over NCCL (strong scaling); --replicas runs N independent copies instead.
--impl reference times the reference's CPU implementation on this host's cores.
--workload ensemble: 256 independent FCC blocks of 5k-80k particles advanced by one
batched launch per timestep (runs of launches replayed from CUDA graphs); with --gpus N
the blocks are split across the ranks by particle count (strong scaling, no exchange).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

# best published single-device figure for this metric (mixed, 5.7M MeshBlock slab,
# RTX 5090, HiDEM/Docs/Performance.md:68): 5,723,826 particles x 5000 steps / 25.83 s
PUBLISHED_MIXED = 5723826 * 5000 / 25.83

# step kernels of the library (hidem_set_step_kernel)
KERNELS = {"auto": 0, "items": 1, "thread": 2, "thread-capped": 3, "thread-async": 4, "two-pass": 5}
KERNEL_NAMES = {v: k for k, v in KERNELS.items()}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["slab", "block", "ensemble", "settle", "topo", "mesh", "ranks",
                                           "meshblock", "surrogate"], default="slab")
    ap.add_argument("--surrogate-batch", type=int, default=65536, help="surrogate: rows per Adam step")
    ap.add_argument("--config", default=None,
                    help="meshblock: the reference's run config (default data/meshblock_5700k/config_mesh_5700k.toml)")
    ap.add_argument("--particle-file", default=None,
                    help="meshblock: the File lattice's HDF5 points (default: particles.h5 beside the config)")
    ap.add_argument("--meshblock-start", type=int, default=25000,
                    help="meshblock: untimed steps before the timed ones (the published run times 25000-30000)")
    ap.add_argument("--ranks", type=int, default=2,
                    help="ranks: slab ranks held as contexts of this process (one GPU)")
    ap.add_argument("--topo", default="1200,200,150",
                    help="topo: slab size in metres on the Fourier-mode bed (the 50M configuration)")
    ap.add_argument("--train-tongues", type=int, default=256, help="settle: training geometries")
    ap.add_argument("--surrogate-inputs", choices=["lattice", "coords"], default="lattice",
                    help="settle: the surrogate's inputs (lattice neighbourhood, or 5 coordinates)")
    ap.add_argument("--test-tongues", type=int, default=16, help="settle: held-out geometries")
    ap.add_argument("--train-steps", type=int, default=20000, help="settle: surrogate Adam steps")
    ap.add_argument("--tongue", default="40,12", help="settle: tongue plan size in metres x,y")
    ap.add_argument("--tongue-thickness", type=float, default=6.0, help="settle: base ice thickness (m)")
    ap.add_argument("--tongue-amplitude", type=float, default=2.0,
                    help="settle: total amplitude of each heightfield's 8 Fourier modes (m)")
    ap.add_argument("--settle-max-steps", type=int, default=40000, help="settle: step cap of each settle")
    ap.add_argument("--settle-check", type=int, default=20, help="settle: steps between kinetic-energy reads")
    ap.add_argument("--max-train-rows", type=int, default=None,
                    help="settle: seeded sample of at most this many training rows")
    ap.add_argument("--lattice-offsets", default="1.5,3,6",
                    help="settle: distances (m) at which the surrogate's inputs sample the heightfields")
    ap.add_argument("--blocks", type=int, default=256, help="ensemble: number of blocks")
    ap.add_argument("--no-graphs", action="store_true", help="ensemble: plain launches")
    ap.add_argument("--kernel", choices=["auto", "items", "thread", "thread-capped", "thread-async", "two-pass"],
                    default="auto", help="step kernel (auto: timed on the first steps)")
    ap.add_argument("--slab", default="400,100,100",
                    help="slab size in metres x,y,z (smaller slabs for profiling captures)")
    ap.add_argument("--replicas", action="store_true",
                    help="slab with --gpus N > 1: N independent replicas instead of the x-slab decomposition")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-numa-bind", action="store_true",
                    help="run the end-to-end job on every allowed CPU, not only the GPU's NUMA node")
    ap.add_argument("--no-fp64", action="store_true", help="slab: skip the plain-FP64 run")
    ap.add_argument("--no-settle", action="store_true", help="slab: skip the warm-start settling experiment")
    ap.add_argument("--amortised-steps", type=int, default=2000,
                    help="slab: steps of the run with its rebuilds (the configuration's 2000; 0 skips)")
    return ap.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def make_workload(args):
    from hidem_b200 import abi, workloads
    prec = abi.PREC_MIXED if args.precision == "mixed" else abi.PREC_FP64
    if args.workload == "slab":
        size = tuple(float(v) for v in args.slab.split(","))
        P, p, l = workloads.calving_slab(size=size, precision=prec, jitter=0.0)
        cells = tuple(max(1, int(round(s / workloads.SQRT2))) for s in size)
        name = (f"calving slab {size[0]:g}x{size[1]:g}x{size[2]:g} m FCC d=1 m "
                f"({cells[0]}x{cells[1]}x{cells[2]} cells), bed, water 90 m, 1% pre-broken")
    else:
        P, p, l = workloads.ice_block(cells=(20, 20, 20), precision=prec)
        name = "ice block 20^3 FCC cells, jitter 0.01 d, bottom fixed"
    return prec, P, p, l, name


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,"
              "utilization.gpu")
    PERIOD_MS = 50

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", str(self.PERIOD_MS)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict | None:
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, busy, mx, reasons = [], [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
                if len(f) > 9 and float(f[9]) >= 50.0:
                    busy.append(float(f[1]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        under_load = busy if busy else sm
        return {"sm_mhz": float(np.median(under_load)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "samples_under_load": len(busy), "period_ms": self.PERIOD_MS,
                "span": "from the warm-up through the timed steps and the rebuild-amortised run"}


def measured_peak():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        d = json.loads(f.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def step_label(kernel: int, extra: str = "") -> str:
    """What one step launches, for roofline.kernel."""
    if kernel == KERNELS["two-pass"]:
        return f"step passes (k_step force pass, k_integrate{extra}, k_link_break), two-pass kernel"
    return f"fused step{extra}, " + KERNEL_NAMES.get(kernel, "?") + " kernel"


def profile_traffic(precision: str, two_pass: bool = True):
    """DRAM bytes per particle-step of the step's kernels from the committed ncu summary
    (profiles/step_passes_slab_*.md for the two-pass step, profiles/fused_step_slab_*.md
    for the fused one; line `dram_bytes_per_particle_step: X`)."""
    stem = "step_passes_slab" if two_pass else "fused_step_slab"
    f = ROOT / "profiles" / f"{stem}_{precision}.md"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.strip().startswith("dram_bytes_per_particle_step:"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


def cpu_model() -> str:
    """The host CPU's model name (for the CPU baseline's record)."""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline(P, p, l, n):
    """The reference's CPU path (oracle/_ref fast build, all host threads) on a bounded
    sample of the same workload: a few timesteps of the whole slab after one warm-up."""
    from oracle import oracle
    if oracle.reference_available(int(P.precision), fast=True):
        sess = oracle.RefSession(P, p, l, fast=True)
        kind = "reference"
        cores = sess.threads()
        t1 = sess.advance(1)  # warm-up (includes nothing of the setup)
        k = int(max(1, min(10, 15.0 / max(t1, 1e-3))))
        secs = sess.advance(k)
        sess.close()
        return {"value": n * k / secs, "unit": "particle-steps/s", "cores": cores, "kind": kind,
                "cpu": cpu_model(), "host_threads": os.cpu_count(),
                "sample": f"{k} timesteps of the full workload ({n} particles) after 1 warm-up step, "
                          f"reference CPU path built with -O3 -ffast-math -march=x86-64-v3 -fopenmp"}
    port = oracle.port()
    _, _, _, _, _, secs = port.run(P, p, l, 3)
    return {"value": n * 3 / secs, "unit": "particle-steps/s", "cores": port.threads(),
            "kind": "port", "sample": f"3 timesteps of the full workload ({n} particles)"}


def make_workload_np(args):
    """make_workload's slab or block built in numpy (hidem_b200.inputs_np), so that the
    reference arm's process maps none of this library's native code; the arrays and
    parameters are the same bit for bit."""
    from hidem_b200 import abi, inputs_np, workloads
    prec = abi.PREC_MIXED if args.precision == "mixed" else abi.PREC_FP64
    if args.workload == "slab":
        size = tuple(float(v) for v in args.slab.split(","))
        P, p, l = inputs_np.calving_slab(size=size, precision=prec, jitter=0.0)
        cells = tuple(max(1, int(round(s / workloads.SQRT2))) for s in size)
        name = (f"calving slab {size[0]:g}x{size[1]:g}x{size[2]:g} m FCC d=1 m "
                f"({cells[0]}x{cells[1]}x{cells[2]} cells), bed, water 90 m, 1% pre-broken")
        return prec, P, p, l, name
    p = inputs_np.fcc_particles(20, 20, 20, prec, jitter=0.01, seed=1)
    z0 = p["zCord"].min()
    p["type"][p["zCord"] < z0 + 0.25 * workloads.SQRT2] |= abi.TYPE_FIXED
    l = inputs_np.distance_links(p, prec, 1.01)
    P = inputs_np.default_params(**workloads.block_overrides(prec, useFixed=1))
    return prec, P, p, l, "ice block 20^3 FCC cells, jitter 0.01 d, bottom fixed"


def run_reference(args):
    """--impl reference: the reference's CPU implementation (oracle/_ref, its own sources
    and flags, all host threads), timed steps after W warm-up, on inputs built without this
    library."""
    world, rank, _ = dist_env()
    if rank != 0:
        return
    from oracle import oracle
    prec, P, p, l, name = make_workload_np(args)
    n = p["xCord"].shape[0]
    fast_ok = oracle.reference_available(prec, fast=True)
    sess = oracle.RefSession(P, p, l, fast=True) if fast_ok else None
    if sess is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built"}))
        return
    warm_n = max(args.warmup, 1)
    warm_s = sess.advance(warm_n) / warm_n
    # timed steps bounded to about a minute of host time (the rate is what is reported)
    timed = int(min(args.steps, max(3, 60.0 / max(warm_s, 1e-6))))
    secs = sess.advance(timed)
    cores = sess.threads()
    sess.close()
    value = n * timed / secs
    line = {
        "metric": slab_metric(args),
        "value": value, "unit": "particle-steps/s", "n_gpus": args.gpus, "steps": timed,
        "steps_requested": args.steps, "warmup": warm_n, "ms_per_step": 1e3 * secs / timed,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64pos" if prec == 1 else "f64", "data": "synthetic",
        "config": slab_config(args, name, n, int(l["state"].shape[0]), world),
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": cores,
                         "kind": "reference", "cpu": cpu_model(), "host_threads": os.cpu_count(),
                         "sample": f"{timed} timesteps of the full workload (of the {args.steps} asked, "
                                   f"bounded to about a minute) after {warm_n} warm-up; inputs "
                                   f"generated in numpy (hidem_b200.inputs_np)"},
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def run_reference_meshblock(args):
    """--impl reference --workload meshblock: the reference's CPU path on its own benchmark
    input, timed steps from the initial state (its per-step cost does not depend on the step
    reached; the GPU arm's state at step 25,000 cannot be handed to this process without
    this library). The input is read by the C restatement's harness-free numpy path."""
    world, rank, _ = dist_env()
    if rank != 0:
        return
    print(json.dumps({"impl": "reference", "unavailable":
                      "the meshblock line carries the reference CPU path on the same state in cpu_baseline; "
                      "reading its HDF5 input needs this library's reader"}))


def run_reference_ensemble(args):
    """--impl reference --workload ensemble: the reference's CPU path block after block on
    a bounded sample (the first blocks of the ensemble), particle-steps/s."""
    world, rank, _ = dist_env()
    if rank != 0:
        return
    from hidem_b200 import abi, workloads
    from oracle import oracle
    prec = abi.PREC_MIXED if args.precision == "mixed" else abi.PREC_FP64
    if not oracle.reference_available(prec, fast=True):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built"}))
        return
    blocks = workloads.ensemble(args.blocks, prec)
    sample = blocks[:8]
    tot_ps, tot_s, cores = 0, 0.0, 1
    for P, p, l in sample:
        sess = oracle.RefSession(P, p, l, fast=True)
        sess.advance(max(args.warmup, 1))
        secs = sess.advance(args.steps)
        cores = sess.threads()
        sess.close()
        tot_ps += p["xCord"].shape[0] * args.steps
        tot_s += secs
    value = tot_ps / tot_s
    n_all = sum(b[1]["xCord"].shape[0] for b in blocks)
    line = {
        "metric": "particle-steps/s (256-block ensemble)", "value": value,
        "unit": "particle-steps/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * n_all / value, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None,
        "dtype": "f32+f64pos" if prec == 1 else "f64", "data": "synthetic",
        "config": {"workload": f"ensemble of {len(blocks)} FCC blocks, 5k-80k particles",
                   "particles": n_all, "precision": args.precision},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": cores,
                         "kind": "reference",
                         "sample": f"{args.steps} timesteps of each of the first {len(sample)} blocks"},
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main_ensemble(args):
    import torch
    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist
    from hidem_b200 import abi, workloads
    from hidem_b200.hidemlib import HiDEMBatch, HiDEMLib

    prec = abi.PREC_MIXED if args.precision == "mixed" else abi.PREC_FP64
    all_blocks = workloads.ensemble(args.blocks, prec)
    n_all = sum(b[1]["xCord"].shape[0] for b in all_blocks)
    mine = workloads.ensemble_shard([b[1]["xCord"].shape[0] for b in all_blocks], world, rank)
    blocks = [all_blocks[i] for i in mine]
    n = sum(b[1]["xCord"].shape[0] for b in blocks)
    L = sum(b[2]["state"].shape[0] for b in blocks)
    kernel = KERNELS[args.kernel]

    def open_all(src):
        libs = []
        for P, p, l in src:
            lib = HiDEMLib(P, device=local)
            lib.set_particles(p)
            lib.set_links(l)
            libs.append(lib)
        if kernel != abi.STEP_KERNEL_AUTO:
            libs[0].set_step_kernel(kernel)
        return libs

    libs = open_all(blocks)
    batch = HiDEMBatch(libs, graphs=not args.no_graphs)
    stream = torch.cuda.ExternalStream(batch.stream_handle)
    batch.step(args.warmup)
    st0 = [lib.stats() for lib in libs]
    c0 = batch.counts()
    pairs = sum(s["num_neighbour_pairs"] for s in st0)

    clocks = ClockSampler(local)
    clocks.start()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    libs[0].profile(True)
    e0.record(stream)
    batch.step(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    kern_ms, kern_n = libs[0].profile_read()
    libs[0].profile(False)
    clk = clocks.stop()
    c1 = batch.counts()
    st1 = [lib.stats() for lib in libs]
    launches = int(sum(b["kernel_launches"] for b in st1) - sum(a["kernel_launches"] for a in st0))
    broken = [s["broken_links"] / max(1, s["num_links"]) for s in st1]
    if pg:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = float(t.item())
        pg.barrier()
    batch.close()
    for lib in libs:
        lib.close()

    value = n_all * args.steps / (ms / 1e3)
    bytes_step = workloads.algorithmic_bytes(n, L, pairs, prec)["total"]
    # kernel time per step from the event pairs around each run of launches
    kern_step_s = kern_ms / 1e3 / max(1, args.steps)
    peak, peak_kind = measured_peak()
    achieved = bytes_step / kern_step_s / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": None, "peak_source": peak_kind,
                "kernel": ("batched two-pass step (k_force_batch, k_integrate_batch, k_break_batch)"
                           if kernel in (abi.STEP_KERNEL_AUTO, abi.STEP_KERNEL_TWO_PASS)
                           else "k_step_batch (" + KERNEL_NAMES[kernel] + ")"),
                "kernel_ms": kern_step_s * 1e3,
                "algorithmic_bytes_per_launch": bytes_step}

    e2e = None
    if not args.no_e2e:
        def pinned(a):
            t = torch.empty(a.shape, dtype=torch.from_numpy(a[:1]).dtype, pin_memory=True)
            out = t.numpy()
            out[...] = a
            return out, t
        keep, host = [], []
        for P, p, l in blocks:
            pp, ll, oo = {}, {}, {}
            for k, v in p.items():
                pp[k], t = pinned(v)
                keep.append(t)
            for k, v in l.items():
                ll[k], t = pinned(v)
                keep.append(t)
            for k, v in abi.empty_particles(p["xCord"].shape[0], prec).items():
                oo[k], t = pinned(v)
                keep.append(t)
            host.append((P, pp, ll, oo))
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        t0 = time.perf_counter()
        libs2 = open_all([(P, pp, ll) for P, pp, ll, _ in host])
        b2 = HiDEMBatch(libs2, graphs=not args.no_graphs)
        b2.step(args.steps)
        for lib, (_, _, _, oo) in zip(libs2, host):
            lib.get_particles(oo)
        for lib in libs2:
            lib.synchronize()
        el = time.perf_counter() - t0
        b2.close()
        for lib in libs2:
            lib.close()
        if pg:
            t = torch.tensor([el], device="cuda", dtype=torch.float64)
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            el = float(t.item())
        h2d = sum(v.nbytes for _, pp, ll, _ in host for v in list(pp.values()) + list(ll.values()))
        d2h = sum(v.nbytes for _, _, _, oo in host for v in oo.values())
        e2e = {"value": n_all * args.steps / el, "unit": "particle-steps/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "step": f"one C-ABI job per rank from pinned host arrays: create {len(blocks)} "
                       f"contexts, upload, {args.steps} batched timesteps, download particles"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            from oracle import oracle
            P, p, l = blocks[0]
            if oracle.reference_available(prec, fast=True):
                sess = oracle.RefSession(P, p, l, fast=True)
                sess.advance(1)
                k = 20
                secs = sess.advance(k)
                cores = sess.threads()
                sess.close()
                nb = p["xCord"].shape[0]
                cpu = {"value": nb * k / secs, "unit": "particle-steps/s", "cores": cores,
                       "kind": "reference",
                       "sample": f"{k} timesteps of block 0 ({nb} particles) after 1 warm-up"}
        except Exception as ex:
            cpu = {"value": None, "unit": "particle-steps/s", "cores": None, "kind": "reference",
                   "sample": f"failed: {ex}"}

    if pg:
        pg.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": "particle-steps/s (256-block ensemble)", "value": value,
        "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None,
        "dtype": "f32+f64pos" if prec == abi.PREC_MIXED else "f64", "data": "synthetic",
        "config": {"workload": f"ensemble of {len(all_blocks)} FCC blocks, 5k-80k particles "
                               f"log-uniform, maxLoad lognormal(5e-4, 0.3)",
                   "particles": n_all, "particles_rank0": n, "links_rank0": L,
                   "precision": args.precision, "parallelism": f"blocks split over {world} ranks",
                   "graphs": not args.no_graphs,
                   "graph_replays": c1["graph_launches"] - c0["graph_launches"],
                   "entry_uploads": c1["uploads"] - c0["uploads"],
                   "rebuilds_in_timed_steps": int(sum(b["regen_count"] for b in st1) - sum(a["regen_count"] for a in st0)),
                   "l2": "inputs larger than L2 (records + link ends > 126 MB)",
                   "broken_fraction_rank0": {"min": float(np.min(broken)),
                                             "median": float(np.median(broken)),
                                             "max": float(np.max(broken))}},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
        "clocks": clk,
    }
    print(json.dumps(line))


def main_settle(args):
    """Learned warm start: settling steps of held-out glacier tongues, cold vs surrogate-
    seeded, both judged by the plain method's convergence test (kinetic energy per particle
    below 1e-6 J over the last 200 steps); plus the surrogate's tensor-core throughput."""
    import dataclasses
    import torch
    from hidem_b200 import settle
    from hidem_b200 import surrogate as sg
    world, rank, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    size = tuple(float(v) for v in args.tongue.split(","))
    thick, amp = args.tongue_thickness, args.tongue_amplitude
    rep = settle.warm_start_experiment(n_train=args.train_tongues, n_test=args.test_tongues, size=size,
                                       base_thickness=thick, amplitude=amp, train_steps=args.train_steps,
                                       inputs=args.surrogate_inputs, max_steps=args.settle_max_steps,
                                       max_train_rows=args.max_train_rows, check=args.settle_check,
                                       offsets=tuple(float(v) for v in args.lattice_offsets.split(",")))
    # tensor-core forward throughput of the trained network's shape on 2M rows
    lattice = args.surrogate_inputs == "lattice"
    nin = settle.n_lattice_inputs(tuple(float(v) for v in args.lattice_offsets.split(","))) if lattice else 5
    cfg = sg.default_config(inputs=nin, fourier_bands=4 if lattice else 6)
    k0 = sg.feature_width(nin, cfg.fourier_bands)
    rows = 1 << 21
    u = np.random.default_rng(0).uniform(-1, 1, (rows, nin)).astype(np.float32)
    with sg.Surrogate(cfg) as net:
        net.predict(u[:16384])
        t0 = time.perf_counter()
        net.predict(u)
        el = time.perf_counter() - t0
        # the same rows resident in device memory: features + the fused network, CUDA events
        du = torch.from_numpy(u).cuda()
        dy = torch.empty((rows, 3), dtype=torch.float32, device="cuda")
        stream = torch.cuda.ExternalStream(net.stream_handle)
        dev = float("inf")
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            net.predict_device(du.data_ptr(), rows, dy.data_ptr())
            e1.record(stream)
            torch.cuda.synchronize()
            dev = min(dev, e0.elapsed_time(e1) / 1e3)
    flops = 2.0 * rows * (k0 * cfg.width + (cfg.hidden_layers - 1) * cfg.width * cfg.width + 3 * cfg.width)
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = float(peaks.get("bf16_tflops", 1590.0))
    d = dataclasses.asdict(rep)
    line = {
        "metric": "settle steps, cold / surrogate-warm (KE < 1e-6 J per particle)",
        "value": d["step_ratio"], "unit": "x fewer steps", "n_gpus": 1, "steps": None,
        "warmup": None, "higher_is_better": True, "scaling": "none", "vs_baseline": None,
        "dtype": "f32+f64pos (settling), bf16/f32-accumulate (surrogate)", "data": "synthetic",
        "config": {"workload": f"glacier tongues {size[0]:g} x {size[1]:g} m plan, base thickness {thick:g} m, "
                               f"bed and surface 8 Fourier modes each (total amplitude {amp:g} m), "
                               f"FCC d = 1 m; {args.train_tongues} training, {args.test_tongues} held out",
                   "particles_per_tongue": d["particles_per_tongue"], "train_samples": d["train_samples"],
                   "surrogate": f"{nin} inputs ({args.surrogate_inputs}), {k0} Fourier features, "
                                f"4 x 256 SiLU MLP, BF16 tcgen05 GEMMs",
                   "train_steps": args.train_steps},
        "cold_steps": d["cold_steps"], "warm_steps": d["warm_steps"],
        "prediction_rel_error": d["prediction_rel_error"],
        "settled_error_over_d": d["settled_error_over_d"],
        "converged": {"cold": d["cold_converged"], "warm": d["warm_converged"]},
        "final_train_loss": d["final_loss"], "seconds": d["seconds"],
        "surrogate_forward": {"rows": rows, "seconds": el, "tflops": flops / el / 1e12,
                              "includes": "pageable host-device copies of inputs and outputs, features, the fused network",
                              "device_seconds": dev, "device_tflops": flops / dev / 1e12,
                              "device_frac_of_bf16_peak": flops / dev / 1e12 / peak,
                              "device_includes": "features and the fused network (k_mlp_pp), inputs in device memory"},
    }
    print(json.dumps(line))


def main_surrogate(args):
    """The learned warm start's network alone, at the settle experiment's shape (82 lattice
    inputs, 4 Fourier bands -> 768 features, 4 x 256 SiLU, 3 outputs): Adam training steps
    of --surrogate-batch rows (features, the fused forward pass that keeps activations, the
    backward GEMMs k_umma_gemm, the CUDA-core reductions and Adam) and the forward pass alone
    on 2M device-resident rows; tensor-core FLOP/s against the measured BF16 peak."""
    import torch
    from hidem_b200 import settle
    from hidem_b200 import surrogate as sg
    world, rank, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    nin = settle.N_LATTICE_INPUTS
    batch = args.surrogate_batch
    cfg = sg.default_config(inputs=nin, fourier_bands=4, batch=batch)
    k0 = sg.feature_width(nin, cfg.fourier_bands)
    W, Lh = cfg.width, cfg.hidden_layers
    rng = np.random.default_rng(0)
    rows = max(4 * batch, 1 << 18)
    x = rng.uniform(-1, 1, (rows, nin)).astype(np.float32)
    y = rng.normal(0, 0.1, (rows, 3)).astype(np.float32)
    fwd_flops = 2.0 * (k0 * W + (Lh - 1) * W * W + 3 * W)
    # backward: data gradients of layers 1.. and weight gradients of every layer
    bwd_flops = 2.0 * ((Lh - 1) * W * W + 3 * W) + 2.0 * (k0 * W + (Lh - 1) * W * W + 3 * W)
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = float(peaks.get("bf16_tflops", 1590.0))
    with sg.Surrogate(cfg) as net:
        net.set_data(x, y)
        net.train(max(args.warmup, 3))
        stream = torch.cuda.ExternalStream(net.stream_handle)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        loss = net.train(args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
        train_s = e0.elapsed_time(e1) / 1e3
        n_fwd = 1 << 21
        u = rng.uniform(-1, 1, (n_fwd, nin)).astype(np.float32)
        du = torch.from_numpy(u).cuda()
        dy = torch.empty((n_fwd, 3), dtype=torch.float32, device="cuda")

        def fwd_seconds():
            net.predict_device(du.data_ptr(), n_fwd, dy.data_ptr())
            t = float("inf")
            for _ in range(3):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                a.record(stream)
                net.predict_device(du.data_ptr(), n_fwd, dy.data_ptr())
                b.record(stream)
                torch.cuda.synchronize()
                t = min(t, a.elapsed_time(b) / 1e3)
            return t
        from hidem_b200 import abi
        best = fwd_seconds()  # the default: the persistent ping-pong pass for width 256
        net.set_forward(abi.SURROGATE_FORWARD_BLOCK)
        best_block = fwd_seconds()
        net.set_forward(abi.SURROGATE_FORWARD_AUTO)
    step_flops = batch * (fwd_flops + bwd_flops)
    value = step_flops * args.steps / train_s / 1e12
    line = {
        "metric": "surrogate training TFLOP/s (BF16 tensor cores, FP32 accumulation)", "value": value,
        "unit": "TFLOP/s", "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 3),
        "ms_per_step": 1e3 * train_s / args.steps, "higher_is_better": True, "scaling": "none",
        "vs_baseline": None, "dtype": "bf16 (f32 accumulate)", "data": "synthetic",
        "config": {"workload": f"surrogate {nin} inputs -> {k0} Fourier features -> {Lh} x {W} SiLU -> 3, "
                               f"Adam steps of {batch} rows", "rows": rows, "batch": batch},
        "frac_of_bf16_peak": value / peak, "final_loss": loss,
        "forward": {"rows": n_fwd, "seconds": best, "tflops": n_fwd * fwd_flops / best / 1e12,
                    "frac_of_bf16_peak": n_fwd * fwd_flops / best / 1e12 / peak,
                    "includes": "features (k_features) and the fused network (k_mlp_pp, the persistent "
                                "ping-pong pass), inputs in device memory",
                    "one_cta_per_block": {"seconds": best_block,
                                          "tflops": n_fwd * fwd_flops / best_block / 1e12,
                                          "includes": "features and k_mlp_fwd"}},
        "roofline": {"bound": "tensor", "achieved": value, "peak": peak, "unit": "TFLOP/s",
                     "frac": value / peak, "traffic": None,
                     "peak_source": "measured" if peaks else "fallback",
                     "kernel": "training step (k_mlp_pp, k_umma_gemm, CUDA-core kernels)"},
    }
    print(json.dumps(line))


def main_topo(args):
    """The large slab on bed topography (mixed precision): particle-steps/s of the fused step
    with the bed as a GlacierDem map; and the mixed-precision error against an FP64 run of
    a ~1M-particle sub-slab of the same construction after 1000 steps."""
    import torch
    from hidem_b200 import abi, workloads
    from hidem_b200.hidemlib import HiDEMLib
    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    size = tuple(float(v) for v in args.topo.split(","))
    t0 = time.perf_counter()
    P, p, l, bed_v, ext = workloads.slab_on_bed(size=size, precision=abi.PREC_MIXED)
    gen_s = time.perf_counter() - t0
    n, L = p["xCord"].shape[0], l["state"].shape[0]
    bed, keep = abi.map2d(bed_v, *ext, abi.PREC_MIXED)
    lib = HiDEMLib(P, device=local)
    lib.set_bed_maps(bed, None)
    t0 = time.perf_counter()
    lib.set_particles(p)
    lib.set_links(l)
    del p, l
    warm = max(args.warmup, 15)
    lib.step(warm)
    lib.synchronize()
    setup_s = time.perf_counter() - t0
    st0 = lib.stats()
    stream = torch.cuda.ExternalStream(lib.stream_handle)
    clocks = ClockSampler(local)
    clocks.start()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    lib.profile(True)
    e0.record(stream)
    lib.step(args.steps)
    e1.record(stream)
    lib.synchronize()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    kern_ms, kern_n = lib.profile_read()
    clk = clocks.stop()
    st1 = lib.stats()
    kernel = lib.step_kernel()
    free, total = torch.cuda.mem_get_info()
    lib.close()
    value = n * args.steps / (ms / 1e3)
    bytes_step = workloads.algorithmic_bytes(n, L, st0["num_neighbour_pairs"], abi.PREC_MIXED)["total"]
    kern_avg_s = (kern_ms / max(kern_n, 1)) / 1e3
    peak, peak_kind = measured_peak()
    achieved = bytes_step / kern_avg_s / 1e9
    # mixed vs FP64 on a ~1M sub-slab of the same construction
    sub = (200.0, 80.0, 45.0)
    res = {}
    for prec in (abi.PREC_MIXED, abi.PREC_FP64):
        Ps, ps, ls, bvs, exs = workloads.slab_on_bed(size=sub, precision=prec, amplitude=15.0 * sub[2] / 150.0,
                                                     water_level=135.0 * sub[2] / 150.0)
        m, k2 = abi.map2d(bvs, *exs, prec)
        sl = HiDEMLib(Ps, device=local)
        sl.set_bed_maps(m, None)
        sl.set_particles(ps)
        sl.set_links(ls)
        sl.step(1000)
        res[prec] = (sl.get_particles(), ps)
        sl.close()
    a, b = res[abi.PREC_MIXED][0], res[abi.PREC_FP64][0]
    dx = np.sqrt(sum((a[k] - b[k]) ** 2 for k in ("xCord", "yCord", "zCord")))
    disp = np.sqrt(sum((b[k] - res[abi.PREC_FP64][1][k]) ** 2 for k in ("xCord", "yCord", "zCord")))
    line = {
        "metric": "particle-steps/s (large slab on bed topography)", "value": value,
        "unit": "particle-steps/s", "n_gpus": 1, "steps": args.steps, "warmup": warm,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64pos", "data": "synthetic",
        "config": {"workload": f"slab {size[0]:g} x {size[1]:g} x {size[2]:g} m FCC d = 1 m on a bed of 8 "
                               f"Fourier modes (amplitude 15 m) as a GlacierDem bed map, water 135 m, "
                               f"front pressure, 1% pre-broken",
                   "particles": n, "links": L, "contact_pairs": st0["num_neighbour_pairs"],
                   "generation_s": gen_s, "upload_and_warmup_s": setup_s,
                   "device_memory_used_gb": (total - free) / 1e9,
                   "l2": "inputs larger than L2"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None, "peak_source": peak_kind,
                     "kernel": step_label(kernel),
                     "kernel_ms": kern_ms / max(kern_n, 1), "algorithmic_bytes_per_launch": bytes_step},
        "mixed_vs_fp64_1M_subslab_1000_steps": {
            "particles": int(dx.shape[0]), "max_err_over_d": float(dx.max()),
            "rms_err_over_d": float(np.sqrt((dx ** 2).mean())),
            "err_over_displacement": float(np.linalg.norm(dx) / max(np.linalg.norm(disp), 1e-30)),
            "max_displacement_m": float(disp.max())},
        "gpu_launches": int(st1["kernel_launches"] - st0["kernel_launches"]), "clocks": clk,
    }
    print(json.dumps(line))


def main_mesh(args):
    """The calving slab in a fjord-shaped collision mesh (the MeshConstrainedDem setting):
    particle-steps/s of the fused step with the closest-triangle query in its integrate,
    the same slab without the mesh beside it, and the reference's CPU path with the same
    mesh on a bounded sample."""
    import torch
    from hidem_b200 import abi, workloads
    from hidem_b200.hidemlib import HiDEMLib
    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    prec = abi.PREC_MIXED if args.precision == "mixed" else abi.PREC_FP64
    size = tuple(float(v) for v in args.slab.split(","))
    P, p, l, md = workloads.slab_in_fjord(size=size, precision=prec)
    mesh, keep = abi.mesh(md["vertices"], md["normals"], md["cell_size"], prec, md["mesh_force"], md["mesh_drag"])
    n, L = p["xCord"].shape[0], l["state"].shape[0]

    def timed(with_mesh: bool):
        lib = HiDEMLib(P, device=local)
        lib.set_step_kernel(KERNELS[args.kernel])
        if with_mesh:
            lib.set_collision_mesh(mesh)
        lib.set_particles(p)
        lib.set_links(l)
        warm = max(args.warmup, 15) if args.kernel == "auto" else args.warmup
        lib.step(warm)
        lib.synchronize()
        st0 = lib.stats()
        stream = torch.cuda.ExternalStream(lib.stream_handle)
        clocks = ClockSampler(local)
        clocks.start()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        lib.profile(True)
        e0.record(stream)
        lib.step(args.steps)
        e1.record(stream)
        lib.synchronize()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        kern_ms, kern_n = lib.profile_read()
        lib.profile(False)
        clk = clocks.stop()
        st1 = lib.stats()
        out = {"ms": ms, "kernel_ms": kern_ms / max(kern_n, 1), "kernel": lib.step_kernel(),
               "launches": int(st1["kernel_launches"] - st0["kernel_launches"]),
               "rebuilds": int(st1["regen_count"] - st0["regen_count"]) if "regen_count" in st1 else None,
               "pairs": st1["num_neighbour_pairs"], "clocks": clk, "warm": warm}
        if with_mesh:
            g = lib.mesh_accel()
            face = lib.mesh_face_forces()
            nonempty = g["sizes"][g["sizes"] > 0]
            out["grid"] = {"cells": int(g["sizes"].shape[0]), "counts": g["counts"].tolist(),
                           "nonempty_cells": int(nonempty.shape[0]),
                           "mean_triangles_per_nonempty_cell": float(nonempty.mean()) if nonempty.size else 0.0,
                           "faces_pushed": int((np.abs(face).sum(axis=1) > 0).sum())}
        lib.close()
        return out

    with_mesh = timed(True)
    plain = timed(False)
    value = n * args.steps / (with_mesh["ms"] / 1e3)
    bytes_step = workloads.algorithmic_bytes(n, L, with_mesh["pairs"], prec)["total"]
    peak, peak_kind = measured_peak()
    achieved = bytes_step / (with_mesh["kernel_ms"] / 1e3) / 1e9
    cpu = None
    if not args.no_cpu_baseline:
        try:
            from oracle import oracle
            if not oracle.reference_available(prec, fast=True):
                raise RuntimeError("oracle/_ref not built")
            ref = oracle.reference(prec, fast=True)
            ref.set_mesh(mesh)
            cpu = cpu_baseline(P, p, l, n)
            ref.set_mesh(None)
            cpu["sample"] += ", with the same collision mesh (the reference's MeshAccel)"
        except Exception as ex:  # reported, not fatal
            cpu = {"value": None, "unit": "particle-steps/s", "cores": None, "kind": "reference",
                   "sample": f"failed: {ex}"}
    line = {
        "metric": "particle-steps/s (slab in a collision mesh)", "value": value, "unit": "particle-steps/s",
        "n_gpus": 1, "steps": args.steps, "warmup": with_mesh["warm"],
        "ms_per_step": with_mesh["ms"] / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64pos" if prec == abi.PREC_MIXED else "f64", "data": "synthetic",
        "config": {"workload": f"calving slab {size[0]:g}x{size[1]:g}x{size[2]:g} m in a fjord mesh "
                               f"(bed of {md['vertices'].shape[0] - 6} triangles, 3 walls, open front), "
                               f"MeshAccel cells {md['cell_size']:g} m",
                   "particles": n, "links": L, "triangles": int(md["vertices"].shape[0]),
                   "precision": args.precision, "parallelism": "replicas x1",
                   "l2": "inputs larger than L2 (records + link ends > 126 MB)"},
        "mesh_grid": with_mesh["grid"],
        "without_mesh": {"value": n * args.steps / (plain["ms"] / 1e3), "ms_per_step": plain["ms"] / args.steps},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_source": peak_kind,
                     "kernel": step_label(with_mesh["kernel"], " with the mesh query"),
                     "kernel_ms": with_mesh["kernel_ms"], "algorithmic_bytes_per_launch": bytes_step},
        "cpu_baseline": cpu, "gpu_launches": with_mesh["launches"], "rebuilds_in_timed_steps": with_mesh["rebuilds"],
        "clocks": with_mesh["clocks"],
    }
    print(json.dumps(line))


def main_slab_decomposed(args):
    """The default slab line on N > 1 GPUs (torchrun, one rank per GPU): the slab is
    decomposed into N x-slabs (hidem_b200.slab, the reference's MPI distribution with its
    halo force exchange, HiDEMDistribution.h:99-234), NCCL point-to-point for the halo
    forces and all-reduces for gridService. Strong scaling: the whole 5.7M slab over N GPUs;
    `value` = particles x steps / the slowest rank's time."""
    import datetime
    import torch
    import torch.distributed as dist
    from hidem_b200 import abi, slab
    from hidem_b200.hidemlib import HiDEMLib
    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    prec, P, p, l, name = make_workload(args)
    n, L = p["xCord"].shape[0], l["state"].shape[0]
    comm = slab.DistComm()
    kernel = KERNELS["thread-capped" if prec == abi.PREC_MIXED else "thread-async"]

    def timed(body, steps):
        torch.cuda.synchronize()
        dist.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        body(steps)
        torch.cuda.synchronize()
        e1.record()
        e1.synchronize()
        t = torch.tensor([e0.elapsed_time(e1)], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    lib = HiDEMLib(P, device=local)
    lib.set_step_kernel(kernel)
    run = slab.SlabRun(comm, [lib], p, l)
    run.step(max(args.warmup, 3))
    st0 = lib.stats()
    red0, ex0 = run.redistributions, run.exchanged
    clocks = ClockSampler(local)
    clocks.start()
    ms = timed(run.step, args.steps)
    clk = clocks.stop()
    st1 = lib.stats()
    launches = int(st1["kernel_launches"] - st0["kernel_launches"])
    held = int(st1["num_particles"])
    lib.close()

    e2e = None
    if not args.no_e2e:
        # a fresh decomposed job: this rank's share uploaded from host arrays, K steps,
        # this rank's particles downloaded; the slowest rank's wall time
        lib2 = HiDEMLib(P, device=local)
        lib2.set_step_kernel(kernel)
        torch.cuda.synchronize()
        dist.barrier()
        t0 = time.perf_counter()
        run2 = slab.SlabRun(comm, [lib2], p, l)
        run2.step(args.steps)
        out = lib2.get_particles()
        lib2.synchronize()
        el = time.perf_counter() - t0
        t = torch.tensor([el], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        el = float(t.item())
        held2 = int(lib2.stats()["num_particles"])
        nb = torch.tensor([held2 * 77.0, sum(v.nbytes for v in out.values())], device="cuda", dtype=torch.float64)
        dist.all_reduce(nb)
        lib2.close()
        e2e = {"value": n * args.steps / el, "unit": "particle-steps/s",
               "h2d_bytes_per_step": int(nb[0].item()), "d2h_bytes_per_step": int(nb[1].item()),
               "step": f"one decomposed job over {world} ranks: partition, each rank's share uploaded "
                       f"from host arrays, {args.steps} timesteps with halo exchanges, each rank's "
                       f"particles downloaded"}
    halo = torch.tensor([held - 0.0], device="cuda", dtype=torch.float64)
    dist.all_reduce(halo)
    dist.destroy_process_group()
    if rank != 0:
        return
    value = n * args.steps / (ms / 1e3)
    cfg = slab_config(args, name, n, L, world)
    line = {
        "metric": slab_metric(args), "value": value, "unit": "particle-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "strong",
        "vs_baseline": (value / PUBLISHED_MIXED) if (prec == abi.PREC_MIXED and args.workload == "slab") else None,
        "dtype": "f32+f64pos" if prec == abi.PREC_MIXED else "f64", "data": "synthetic",
        "config": cfg,
        "decomposition": {"transport": "NCCL point-to-point (halo forces), all-reduce (gridService)",
                          "particles_held_all_ranks": int(halo.item()),
                          "halo_fraction": float(halo.item()) / n - 1.0,
                          "force_records_rank0_per_step": (run.exchanged - ex0) / max(args.steps, 1),
                          "redistributions_in_timed_steps": run.redistributions - red0},
        "roofline": None, "cpu_baseline": None, "e2e": e2e, "gpu_launches": launches,
        "clocks": clk,
    }
    print(json.dumps(line))


def main_ranks(args):
    """The slab decomposed over ranks (hidem_b200.slab): with one process, --ranks contexts
    on its GPU exchange halo forces by device copies; under torchrun, one rank per GPU over
    NCCL. Times K decomposed timesteps (gridService, forces, halo exchange, integrate, link
    update) and, on one GPU, the same K steps of one context through the same separate
    calls and through the fused step, so the cost of the decomposition shows."""
    import torch
    from hidem_b200 import abi, slab, workloads
    from hidem_b200.hidemlib import HiDEMLib
    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    prec = abi.PREC_MIXED if args.precision == "mixed" else abi.PREC_FP64
    size = tuple(float(v) for v in args.slab.split(","))
    P, p, l = workloads.calving_slab(size=size, precision=prec)
    n, L = p["xCord"].shape[0], l["state"].shape[0]
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        comm = slab.DistComm()
        nranks = world
    else:
        comm = slab.LocalComm(args.ranks)
        nranks = args.ranks

    def region(body, steps):
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        body(steps)
        torch.cuda.synchronize()
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        if world > 1:
            t = torch.tensor([ms], device="cuda")
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    single = {}
    if world == 1:
        for mode in ("split", "fused"):
            lib = HiDEMLib(P, device=local)
            lib.set_step_kernel(KERNELS["thread-capped" if prec == abi.PREC_MIXED else "thread-async"])
            lib.set_particles(p)
            lib.set_links(l)

            def body(k, lib=lib, mode=mode):
                for _ in range(k):
                    if mode == "fused":
                        lib.step(1)
                    else:
                        lib.timestep_split()
                lib.synchronize()
            body(args.warmup)
            single[mode] = region(body, args.steps) / args.steps
            lib.close()
            torch.cuda.empty_cache()
    libs = [HiDEMLib(P, device=local) for _ in comm.ranks]
    for lib in libs:
        lib.set_step_kernel(KERNELS["thread-capped" if prec == abi.PREC_MIXED else "thread-async"])
    run = slab.SlabRun(comm, libs, p, l)
    run.step(args.warmup)
    st0 = [lib.stats() for lib in libs]
    red0, ex0 = run.redistributions, run.exchanged
    clocks = ClockSampler(local)
    clocks.start()
    ms = region(run.step, args.steps) / args.steps
    clk = clocks.stop()
    st1 = [lib.stats() for lib in libs]
    held = [int(s["num_particles"]) for s in st1]
    launches = sum(int(b["kernel_launches"] - a["kernel_launches"]) for a, b in zip(st0, st1))
    # one redistribution of the current state, outside the timed steps: what it costs to
    # recut the slabs and move what changes hands (wall time, every rank)
    redist_s = {}
    for mode in (True, False):
        run.device_redistribution = mode
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        run._redistribute()
        for lib in libs:
            lib.synchronize()
        redist_s["device" if mode else "host"] = time.perf_counter() - t0
    run.device_redistribution = True
    if rank == 0:
        lay = run.layout
        halo = int(sum(len(lay.local[r]) for r in range(nranks)) - n)
        line = {
            "metric": "particle-steps/s (slab decomposed over ranks)", "value": n / (ms / 1e3),
            "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f32+f64pos" if prec == abi.PREC_MIXED else "f64", "data": "synthetic",
            "config": {"workload": f"calving slab {size[0]:g}x{size[1]:g}x{size[2]:g} m in {nranks} x-slabs",
                       "particles": n, "links": L, "ranks": nranks,
                       "transport": "NCCL point-to-point" if world > 1 else "device copies between contexts of one process",
                       "parallelism": f"slabs{nranks}", "precision": args.precision,
                       "l2": "inputs larger than L2 (records + link ends > 126 MB)"},
            "halo": {"halo_particles": halo, "halo_fraction": halo / n,
                     "force_records_per_step": (run.exchanged - ex0) / max(args.steps, 1),
                     "exchange_bytes_per_step": (run.exchanged - ex0) / max(args.steps, 1) * 6 * (4 if prec == abi.PREC_MIXED else 8),
                     "particles_held_per_rank": held if world == 1 else None},
            "redistributions_in_timed_steps": run.redistributions - red0,
            "redistribution_s": dict(redist_s, what="one recut of the current state after the timed "
                                     "steps, with the state kept in device memory and through host "
                                     "arrays: held sets read back, moves packed and exchanged, new "
                                     "held sets installed (their rebuild comes at the next step)"),
            "one_context_ms_per_step": single or None,
            "gpu_launches": launches, "clocks": clk,
        }
        print(json.dumps(line))
    for lib in libs:
        lib.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def slab_config(args, name: str, n: int, L: int, world: int) -> dict:
    """The `config` of the slab line, identical in both arms at the same N."""
    par = f"x-slabs{world}" if (world > 1 and not args.replicas) else f"replicas x{world}"
    return {"workload": name, "particles": n, "links": L, "precision": args.precision,
            "parallelism": par, "l2": "inputs larger than L2 (records + link ends > 126 MB)"}


def slab_metric(args) -> str:
    return "particle-steps/s (5.7M slab)" if args.workload == "slab" else "particle-steps/s (32k block)"


def timed_steps(lib, stream, steps: int, pg=None):
    """K timesteps between CUDA events on the library's stream (a barrier and device
    synchronisation on both sides); returns (ms, step-kernel ms per step, launches, stats
    before, stats after)."""
    import torch
    st0 = lib.stats()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    lib.profile(True)
    e0.record(stream)
    lib.step(steps)
    e1.record(stream)
    lib.synchronize()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    kern_ms, kern_n = lib.profile_read()
    lib.profile(False)
    st1 = lib.stats()
    return ms, kern_ms / max(kern_n, 1), int(st1["kernel_launches"] - st0["kernel_launches"]), st0, st1


def roofline_of(n, L, pairs, prec, kern_step_ms, precision: str, step_kernel: int) -> dict:
    from hidem_b200 import workloads
    bytes_step = workloads.algorithmic_bytes(n, L, pairs, prec)["total"]
    peak, peak_kind = measured_peak()
    achieved = bytes_step / (kern_step_ms / 1e3) / 1e9
    dpps = profile_traffic(precision, step_kernel == KERNELS["two-pass"])
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": (dpps * n) if dpps else None,
            "peak_source": peak_kind, "kernel": step_label(step_kernel),
            "kernel_ms": kern_step_ms, "algorithmic_bytes_per_launch": bytes_step}


def main_slab(args):
    """The default line: the calving slab in the requested precision (K timed steps, the
    end-to-end job through the C ABI, the 2000-step run of the configuration with its
    rebuilds, the roofline, the CPU baseline); with mixed precision also the plain-FP64 run
    of the same slab and the learned warm start's settling experiment, the two other halves
    of the metric."""
    import torch
    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist
    from hidem_b200 import abi
    from hidem_b200.hidemlib import HiDEMLib

    prec, P, p, l, name = make_workload(args)
    n = p["xCord"].shape[0]
    L = l["state"].shape[0]

    clocks = ClockSampler(local)
    clocks.start()
    lib = HiDEMLib(P, device=local)
    lib.set_step_kernel(KERNELS[args.kernel])
    lib.set_particles(p)
    lib.set_links(l)
    stream = torch.cuda.ExternalStream(lib.stream_handle)
    # warm-up: at least the autotuner's rounds, so the timed steps use its choice
    warm = max(args.warmup, 15) if args.kernel == "auto" else args.warmup
    lib.step(warm)
    lib.synchronize()
    ms, kern_step_ms, launches, st0, st1 = timed_steps(lib, stream, args.steps, pg)
    pairs = st1["num_neighbour_pairs"]
    step_kernel = lib.step_kernel()
    if pg:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = float(t.item())
        pg.barrier()
    lib.close()
    value = world * n * args.steps / (ms / 1e3)
    roofline = roofline_of(n, L, pairs, prec, kern_step_ms, args.precision, step_kernel)

    # the configuration's whole run (2000 steps from step 0, its rebuilds included), the
    # step kernel fixed to the tuned one
    amortised = None
    if args.amortised_steps > 0:
        lib = HiDEMLib(P, device=local)
        lib.set_step_kernel(step_kernel)
        lib.set_particles(p)
        lib.set_links(l)
        s2 = torch.cuda.ExternalStream(lib.stream_handle)
        ams, akern, alaunch, a0, a1 = timed_steps(lib, s2, args.amortised_steps, pg)
        if pg:
            t = torch.tensor([ams], device="cuda", dtype=torch.float64)
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            ams = float(t.item())
        lib.close()
        amortised = {"steps": args.amortised_steps, "value": world * n * args.amortised_steps / (ams / 1e3),
                     "ms_per_step": ams / args.amortised_steps,
                     "rebuilds": int(a1["regen_count"] - a0["regen_count"]),
                     "step_kernel_ms_per_step": akern, "gpu_launches": alaunch,
                     "what": "a fresh context: steps 0..K-1 of the configuration's run, the first "
                             "step's rebuild and the rebuild policy's later ones included"}
    clk = clocks.stop()

    e2e = None
    if not args.no_e2e:
        e2e = e2e_job(args, P, p, l, prec, step_kernel, local, pg, world, n)

    fp64 = None
    if args.precision == "mixed" and args.workload == "slab" and not args.no_fp64:
        a64 = argparse.Namespace(**{**vars(args), "precision": "fp64"})
        prec64, P64, p64, l64, _ = make_workload(a64)
        lib = HiDEMLib(P64, device=local)
        lib.set_step_kernel(KERNELS[args.kernel])
        lib.set_particles(p64)
        lib.set_links(l64)
        s64 = torch.cuda.ExternalStream(lib.stream_handle)
        lib.step(warm)
        lib.synchronize()
        ms64, k64, la64, _, b64 = timed_steps(lib, s64, args.steps, pg)
        sk64 = lib.step_kernel()
        if pg:
            t = torch.tensor([ms64], device="cuda", dtype=torch.float64)
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            ms64 = float(t.item())
        lib.close()
        del p64, l64
        v64 = world * n * args.steps / (ms64 / 1e3)
        fp64 = {"value": v64, "unit": "particle-steps/s", "ms_per_step": ms64 / args.steps,
                "mixed_over_fp64": value / v64, "gpu_launches": la64,
                "roofline": roofline_of(n, L, b64["num_neighbour_pairs"], prec64, k64, "fp64", sk64),
                "what": "the same slab and steps in the plain FP64 build (lp = ct = double)"}

    settle = None
    if args.precision == "mixed" and args.workload == "slab" and not args.no_settle and rank == 0:
        settle = settle_summary(args)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(P, p, l, n)
        except Exception as ex:  # reported, not fatal
            cpu = {"value": None, "unit": "particle-steps/s", "cores": None, "kind": "reference",
                   "sample": f"failed: {ex}"}

    if pg:
        pg.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": slab_metric(args),
        "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": warm, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": (value / PUBLISHED_MIXED) if (prec == abi.PREC_MIXED and args.workload == "slab") else None,
        "dtype": "f32+f64pos" if prec == abi.PREC_MIXED else "f64", "data": "synthetic",
        "config": slab_config(args, name, n, L, world),
        "contact_pairs": pairs,
        "baseline_number": "RTX 5090 1.108e9 particle-steps/s, HiDEM/Docs/Performance.md:68",
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
        "rebuilds_in_timed_steps": int(st1["regen_count"] - st0["regen_count"]),
        "rebuild_amortised": amortised, "fp64": fp64, "settle": settle,
        "clocks": clk,
    }
    print(json.dumps(line))


def gpu_local_cpus(device: int):
    """The host CPUs next to the GPU (NVML's CPU affinity of the device: its NUMA node) that
    this process may run on; None when NVML cannot tell or when they are all of them."""
    try:
        import pynvml
        pynvml.nvmlInit()
        h = pynvml.nvmlDeviceGetHandleByIndex(device)
        words = ((os.cpu_count() or 64) + 63) // 64
        mask = pynvml.nvmlDeviceGetCpuAffinity(h, words)
        cpus = {w * 64 + b for w, m in enumerate(mask) for b in range(64) if (int(m) >> b) & 1}
        allowed = os.sched_getaffinity(0)
        cpus &= allowed
        return cpus if cpus and cpus != allowed else None
    except Exception:
        return None


def e2e_job(args, P, p, l, prec, step_kernel, local, pg, world, n, start_step: int = 0):
    """The same K steps through the C ABI from pinned host buffers: upload of the particle
    and link state, K steps, download of the particle state; wall time, devices synchronised
    on both sides."""
    import torch
    from hidem_b200 import abi
    from hidem_b200.hidemlib import HiDEMLib
    # the job's host side on the CPUs next to the GPU, so that its pinned buffers sit in that
    # NUMA node's memory and the copies do not cross between sockets (the affinity a serving
    # process would take; restored after the job)
    near = None if getattr(args, "no_numa_bind", False) else gpu_local_cpus(local)
    prev = os.sched_getaffinity(0)
    if near:
        os.sched_setaffinity(0, near)
    try:
        return _e2e_job(args, P, p, l, prec, step_kernel, local, pg, world, n, start_step,
                        len(near) if near else len(prev), bool(near))
    finally:
        if near:
            os.sched_setaffinity(0, prev)


def _e2e_job(args, P, p, l, prec, step_kernel, local, pg, world, n, start_step, host_cpus, bound):
    import torch
    from hidem_b200 import abi
    from hidem_b200.hidemlib import HiDEMLib

    def pinned(a):
        t = torch.empty(a.shape, dtype=torch.from_numpy(a[:1]).dtype, pin_memory=True)
        out = t.numpy()
        out[...] = a
        return out, t
    keep = []
    pp, ll = {}, {}
    for k, v in p.items():
        pp[k], t = pinned(v)
        keep.append(t)
    # a fresh job's link ends carry no history (CT all zero): like the reference's own
    # start, which generates its links in place, it uploads none (the library zeroes CT)
    fresh = not any(l[k].any() for k in ("CT0", "CT1", "CT2", "CT3", "CT4", "CT5") if k in l)
    for k, v in l.items():
        if fresh and k.startswith("CT"):
            continue
        ll[k], t = pinned(v)
        keep.append(t)
    outp = {}
    for k, v in abi.empty_particles(n, prec).items():
        outp[k], t = pinned(v)
        keep.append(t)
    # one untimed job first (the warm-up of the end-to-end leg: the GPU leaves its idle
    # clocks, the memory pool holds the context's buffers), then the timed one
    warm = HiDEMLib(P, device=local)
    warm.set_step_kernel(step_kernel)
    if start_step:
        warm.set_timestep(start_step)
    warm.set_particles(pp)
    warm.set_links(ll)
    warm.step(min(args.steps, 5))
    warm.get_particles(outp)
    warm.close()
    lib2 = HiDEMLib(P, device=local)
    lib2.set_step_kernel(step_kernel)
    if start_step:
        lib2.set_timestep(start_step)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    t0 = time.perf_counter()
    lib2.set_particles(pp)
    ta = time.perf_counter()
    lib2.set_links(ll)
    tb = time.perf_counter()
    lib2.step(args.steps)
    tc = time.perf_counter()
    lib2.get_particles(outp)
    lib2.synchronize()
    t1 = time.perf_counter()
    el = t1 - t0
    parts = {"set_particles_s": ta - t0, "set_links_s": tb - ta, "steps_s": tc - tb,
             "get_particles_s": t1 - tc}
    if pg:
        t = torch.tensor([el], device="cuda", dtype=torch.float64)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        el = float(t.item())
    lib2.close()
    h2d = sum(v.nbytes for v in pp.values()) + sum(v.nbytes for v in ll.values())
    d2h = sum(v.nbytes for v in outp.values())
    return {"value": world * n * args.steps / el, "unit": "particle-steps/s",
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "warmup": "one untimed job (5 steps) before the timed one",
            "step": f"one C-ABI job from pinned host arrays: upload state (particles, links"
                    f"{'; side history zero, not uploaded' if fresh else ', side history'}), "
                    f"{args.steps} timesteps, download particles", "breakdown": parts,
            "host_cpus": host_cpus, "bound_to_gpu_numa_node": bound}


def settle_summary(args) -> dict:
    """The learned warm start's experiment (the settle workload's defaults): held-out
    tongues settled cold and from the surrogate's prediction, steps to the plain method's
    convergence test."""
    import dataclasses
    from hidem_b200 import settle
    size = tuple(float(v) for v in args.tongue.split(","))
    t0 = time.perf_counter()
    rep = settle.warm_start_experiment(n_train=args.train_tongues, n_test=args.test_tongues, size=size,
                                       base_thickness=6.0, amplitude=2.0, train_steps=args.train_steps,
                                       inputs=args.surrogate_inputs)
    d = dataclasses.asdict(rep)
    return {"metric": "settle steps, cold / surrogate-warm (KE < 1e-6 J per particle)",
            "step_ratio": d["step_ratio"],
            "cold_steps_mean": float(np.mean(d["cold_steps"])),
            "warm_steps_mean": float(np.mean(d["warm_steps"])),
            "prediction_rel_error_mean": float(np.mean(d["prediction_rel_error"])),
            "settled_error_over_d_max": float(np.max(d["settled_error_over_d"])),
            "all_converged": {"cold": bool(d["cold_converged"]), "warm": bool(d["warm_converged"])},
            "tongues": {"size_m": list(size), "train": args.train_tongues, "held_out": args.test_tongues,
                        "particles_per_tongue": d["particles_per_tongue"]},
            "seconds": time.perf_counter() - t0}


def meshblock_paths(args):
    cfg = Path(args.config) if args.config else ROOT / "data" / "meshblock_5700k" / "config_mesh_5700k.toml"
    pf = Path(args.particle_file) if args.particle_file else cfg.parent / "particles.h5"
    if not cfg.exists() or not pf.exists():
        raise SystemExit(f"meshblock: {cfg} / {pf} not found: copy HiDEM/Benchmark/5700k/"
                         f"{{config_mesh_5700k.toml,particles.h5}} of the reference there, or pass "
                         f"--config / --particle-file")
    return cfg, pf


def main_meshblock(args):
    """The reference's own benchmark run (HiDEM/Benchmark/5700k: MeshBlock sample, File
    lattice of 5,723,826 particles, config_mesh_5700k.toml): the run advances untimed to
    --meshblock-start (the reference's published time covers steps 25,000-30,000, with link
    breaking active from t = breakTime), then K timesteps are timed. vs_baseline divides by
    the published RTX 5090 figure of that run (HiDEM/Docs/Performance.md:68)."""
    import torch
    from hidem_b200 import abi, workloads
    from hidem_b200.hidemlib import HiDEMLib
    world, rank, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    cfg, pf = meshblock_paths(args)
    prec = abi.PREC_MIXED if args.precision == "mixed" else abi.PREC_FP64
    t0 = time.perf_counter()
    P, p, l, info = workloads.meshblock(str(cfg), str(pf), prec)
    gen_s = time.perf_counter() - t0
    n, L = p["xCord"].shape[0], l["state"].shape[0]
    clocks = ClockSampler(local)
    lib = HiDEMLib(P, device=local)
    lib.set_step_kernel(KERNELS[args.kernel])
    lib.set_particles(p)
    lib.set_links(l)
    stream = torch.cuda.ExternalStream(lib.stream_handle)
    start = max(args.meshblock_start, args.warmup, 15 if args.kernel == "auto" else 0)
    t0 = time.perf_counter()
    lib.step(start)
    lib.synchronize()
    adv_s = time.perf_counter() - t0
    # the state where the timed region starts, for the legs that start there (untimed)
    sp, sl = lib.get_particles(), lib.get_links()
    clocks.start()
    ms, kern_ms, launches, st0, st1 = timed_steps(lib, stream, args.steps)
    clk = clocks.stop()
    step_kernel = lib.step_kernel()
    state_p = lib.get_particles()
    state_l = lib.get_links()
    lib.close()
    value = n * args.steps / (ms / 1e3)
    pairs = st1["num_neighbour_pairs"]
    roofline = roofline_of(n, L, pairs, prec, kern_ms, args.precision, step_kernel)
    roofline["traffic"] = None  # the committed DRAM figures are of the synthetic slab

    e2e = None
    if not args.no_e2e:
        # the job from host arrays: the state at the timed region's start uploaded (particles,
        # links with their CT history), K steps, the particle state downloaded
        e2e = e2e_job(args, P, sp, sl, prec, step_kernel, local, None, 1, n, start_step=start)

    cpu = None
    if not args.no_cpu_baseline:
        try:
            from oracle import oracle
            if not oracle.reference_available(prec, fast=True):
                raise RuntimeError("oracle/_ref not built")
            sess = oracle.RefSession(P, sp, sl, fast=True, start_step=start)
            sess.advance(1)
            k = 5
            secs = sess.advance(k)
            cpu = {"value": n * k / secs, "unit": "particle-steps/s", "cores": sess.threads(),
                   "kind": "reference", "cpu": cpu_model(), "host_threads": os.cpu_count(),
                   "sample": f"{k} timesteps from step {start + 1} of the same run (the GPU's state at "
                             f"step {start} handed over) after 1 warm-up step, reference CPU path built with "
                             f"-O3 -ffast-math -march=x86-64-v3 -fopenmp"}
            sess.close()
        except Exception as ex:  # reported, not fatal
            cpu = {"value": None, "unit": "particle-steps/s", "cores": None, "kind": "reference",
                   "sample": f"failed: {ex}"}
    broken = int((state_l["state"] == 0).sum())
    line = {
        "metric": "particle-steps/s (MeshBlock 5700k benchmark run)", "value": value,
        "unit": "particle-steps/s", "n_gpus": 1, "steps": args.steps, "warmup": start,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": value / PUBLISHED_MIXED if prec == abi.PREC_MIXED else None,
        "dtype": "f32+f64pos" if prec == abi.PREC_MIXED else "f64",
        "data": "the reference's own benchmark input (HiDEM/Benchmark/5700k/particles.h5, config_mesh_5700k.toml)",
        "config": {"workload": f"MeshBlock File lattice {pf.parent.name}: steps {start}-{start + args.steps}",
                   "particles": n, "links": L, "precision": args.precision, "parallelism": "replicas x1",
                   "l2": "inputs larger than L2 (records + link ends > 126 MB)"},
        "baseline_number": "RTX 5090 25.83 s for steps 25000-30000 = 1.108e9 particle-steps/s, HiDEM/Docs/Performance.md:68",
        "contact_pairs": pairs, "broken_links_at_end": broken,
        "rebuilds_in_timed_steps": int(st1["regen_count"] - st0["regen_count"]),
        "rebuilds_total": int(st1["regen_count"]),
        "setup_s": {"read_and_links": gen_s, "advance_to_start": adv_s},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
        "clocks": clk,
    }
    print(json.dumps(line))


def main():
    args = parse()
    if args.workload == "surrogate":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable":
                              "the reference has no learned warm start"}))
        else:
            main_surrogate(args)
        return
    if args.workload == "meshblock":
        if args.impl == "reference":
            run_reference_meshblock(args)
        else:
            main_meshblock(args)
        return
    if args.workload == "ranks":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable":
                              "the reference's ranks are MPI processes; its CPU path is timed by the slab workload"}))
        else:
            main_ranks(args)
        return
    if args.workload == "mesh":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable":
                              "the mesh workload reports the reference CPU path in its own line (cpu_baseline)"}))
        else:
            main_mesh(args)
        return
    if args.workload == "topo":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable":
                              "the reference CPU path on the 50M-particle slab exceeds the bench's time bound"}))
        else:
            main_topo(args)
        return
    if args.workload == "settle":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable":
                              "the reference has no learned warm start; its settling is the cold start"}))
        else:
            main_settle(args)
        return
    if args.workload == "ensemble":
        if args.impl == "reference":
            run_reference_ensemble(args)
        else:
            main_ensemble(args)
        return
    if args.impl == "reference":
        run_reference(args)
        return
    if dist_env()[0] > 1 and not args.replicas:
        main_slab_decomposed(args)
        return
    main_slab(args)


if __name__ == "__main__":
    main()
