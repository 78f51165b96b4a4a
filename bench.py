"""Benchmark: explicit BPM uniaxial compression, particle-steps/s.

Workload: a 198,061-particle seeded lattice cylinder (D 52 mm x H 104 mm, particle
radius 0.5 mm) of the reference's granite bonded-particle model (parameters of
mp_determineconjgradient.cu:15-38), loaded by the uniaxial platens, reference
precision (FP32 state). One bench "step" is STEPS_PER_BENCH_STEP explicit DEM steps
of the whole specimen (bin/list maintenance, bond and contact forces with break
check, platen, integration, cut, load reduction).

value : particle-steps/s of the fused engine, state resident in HBM, timed with
        CUDA events on the engine's stream (max over ranks for N > 1).
e2e   : the same metric through the reference-facing driver call
        md_CalculationUniaxialCompression with host buffers (pinned upload of the
        positions, build of cells/rows/bonds, the steps, download of the result),
        timed on the host around each call.
--impl reference : the reference's own CPU force path (h_CalculateForceElastic,
        md_calculateforcesbpm_cpu.cpp, built from its source into oracle/_ref) on
        the same specimen's bonds, all host threads (one specimen copy per thread).

Multi-GPU: independent specimens per rank (different seeds), no data-path
collective; only the elapsed time is max-reduced.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "rockfit-dem_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np

STEPS_PER_BENCH_STEP = 1000
DIAMETER, HEIGHT = 52.0, 104.0
METRIC = "particle-steps/s"
WORKLOAD = "explicit BPM uniaxial compression, 198k-particle lattice cylinder D52xH104 mm, granite, fp32 state"


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_per_particle_step():
    """dram read+write bytes per particle-step of the step kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "k_step_uniaxial-200k.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("traffic_bytes_per_particle_step:"):
            return float(line.split(":")[1])
    return None


class Clocks:
    """nvidia-smi sampler running during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev = dev
        self.proc = None
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        self.f.flush()
        rows = [l.strip().split(",") for l in open(self.f.name) if l.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for n, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(n)
            except Exception:
                pass
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return 0, 1, None
    import torch
    import torch.distributed as dist
    rank = int(os.environ["RANK"])
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", rank)))
    import datetime
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return rank, ws, dist


def max_over_ranks(x, dist):
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x, dist):
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def cpu_reference(task, R, reps, threads):
    """The reference's own h_CalculateForceElastic over the specimen's bond slots.
    Rows come from the oracle's restatement of the reference's initial build."""
    import ctypes as C
    import oracle
    L = oracle.load()
    ref = oracle.ref_cpu()
    N, K = int(task.N), int(task.K)
    CN = int(task.C.N)
    CI, CIs, pnC = np.zeros(N, np.uint64), np.zeros(2 * N, np.uint64), np.zeros(2 * CN, np.uint64)
    L.rfo_cell_distribution_f(R.ctypes.data, N, CI.ctypes.data, CIs.ctypes.data, pnC.ctypes.data, CN, task.C._1d_a,
                              task.C.Nr)
    IL = np.zeros(N * K, np.uint64)
    L.rfo_construct_list_f(R.ctypes.data, N, CIs.ctypes.data, pnC.ctypes.data, IL.ctypes.data, K, task.C.a,
                           task.C._1d_a, task.aacut, task.C.Nr, CN)
    ty, iL = np.zeros(N * K, np.uint8), np.zeros(N * K, np.float32)
    z = np.zeros(3 * N * K, np.float32)
    L.rfo_construct_bonds_f(R.ctypes.data, N, IL.ctypes.data, ty.ctypes.data, iL.ctypes.data, z.ctypes.data,
                            z.ctypes.data, z.ctypes.data, z.ctypes.data, K, float(np.float32(task.Po.b_dd)))
    bonds = int(((IL != np.uint64(2 ** 64 - 1)) & (ty == 1)).sum())
    if ref is None:
        return None, bonds
    IL32 = IL.astype(np.uint32)
    IL32[IL == np.uint64(2 ** 64 - 1)] = np.uint32(0xFFFFFFFF)
    V = np.zeros(3 * N, np.float32)
    W = np.zeros(3 * N, np.float32)
    f = lambda x: float(np.float32(x))
    P = task.Po
    ev = C.c_uint64(0)
    secs = ref.ref_cpu_bond_forces(R.ctypes.data, V.ctypes.data, W.ctypes.data, IL32.ctypes.data, ty.ctypes.data,
                                   iL.ctypes.data, N, K, f(P.dt), f(P.m_E), f(P.m_G), f(P.b_r), f(P.m_Ec), f(P.m_Gc),
                                   reps, threads, C.byref(ev))
    return secs, bonds


def run_reference(args):
    rank, ws, dist = dist_init()
    if rank != 0:
        return
    import rfdem
    t, R = rfdem.make_test(rfdem.RF_TEST_UNIAXIAL, DIAMETER, HEIGHT, seed=0xB2000000 + 2000, max_strain=1.0)
    threads = os.cpu_count() or 1
    cpu_reference(t, R, 1, 1)                      # builds rows once (and warms the library)
    secs_w, _ = cpu_reference(t, R, max(args.warmup, 1), threads)
    if secs_w is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libmdref_cpu.so not built (reference tree absent at build time)"}))
        return
    secs, bonds = cpu_reference(t, R, args.steps, threads)
    N = int(t.N)
    value = threads * N * args.steps / secs
    sample = ("reference h_CalculateForceElastic (md_calculateforcesbpm_cpu.cpp:20-288, bond slots only) over all "
              "%d directed bond slots of the %d-particle specimen, %d passes per thread, %d threads each on its own "
              "specimen copy; one pass = one particle-step of every particle" % (bonds, N, args.steps, threads))
    out = {"metric": METRIC, "value": value, "unit": "particle-steps/s", "impl": "reference", "n_gpus": ws,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": {"workload": WORKLOAD, "particles": N, "cpu_threads": threads},
           "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": threads, "kind": "reference",
                            "sample": sample},
           "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def run_engine(args):
    import torch
    rank, ws, dist = dist_init()
    dev = torch.cuda.current_device()
    import rfdem
    S = STEPS_PER_BENCH_STEP
    t, R = rfdem.make_test(rfdem.RF_TEST_UNIAXIAL, DIAMETER, HEIGHT, seed=0xB2000000 + 2000 + rank, max_strain=1.0)
    N = int(t.N)
    e = rfdem.Engine(t, R)
    stream = torch.cuda.ExternalStream(e.stream())
    for _ in range(args.warmup):
        e.step(S)
    torch.cuda.synchronize()
    c0 = e.counters()
    clocks = Clocks(dev)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        e.step(S)
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop()
    if dist is not None:
        dist.barrier()
    ms = ev0.elapsed_time(ev1)
    c1 = e.counters()
    done_steps = c1["steps"] - c0["steps"]
    if done_steps != S * args.steps:
        raise SystemExit("bench: the specimen finished early (%d of %d steps)" % (done_steps, S * args.steps))
    ms_max = max_over_ranks(ms, dist)
    total_particles = sum_over_ranks(float(N), dist)
    value = total_particles * S * args.steps / (ms_max * 1e-3)
    bbar, cbar = c1["bonds"] / N, c1["contacts"] / N
    K = int(t.K)
    # algorithmic bytes per particle-step (fused explicit step, FP32 state, K slots)
    b_step = 72 + 5 * K + 32 + 105 * bbar + 24 * cbar
    per_step_s = (ms * 1e-3) / (S * args.steps)
    achieved = b_step * N / per_step_s / 1e9
    peak, peak_kind = peaks()
    tr = traffic_per_particle_step()
    rebuilds = c1["rebuilds"] - c0["rebuilds"]
    launches = S * args.steps + 7 * rebuilds + 2 * args.steps

    # e2e through the reference-facing driver call with host buffers
    graph_used = e.uses_graph()
    e.close()
    e2e_steps = S
    pinned = torch.from_numpy(R).pin_memory()
    Rout = torch.empty_like(pinned).pin_memory()
    curve = torch.empty(3 * e2e_steps, dtype=torch.float64).pin_memory()
    import ctypes as C
    e2e_calls = 0 if args.no_e2e else 3

    def e2e_call():
        tt = rfdem.Task.from_buffer_copy(t)
        res = rfdem.RunResult()
        rfdem.check(rfdem.lib.md_CalculationUniaxialCompression(C.byref(tt), pinned.data_ptr(), e2e_steps,
                                                                 curve.data_ptr(), e2e_steps, Rout.data_ptr(),
                                                                 C.byref(res)), "e2e")
        return res
    e2e_value = None
    if e2e_calls:
        e2e_call()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_calls):
            e2e_call()
        torch.cuda.synchronize()
        e2e_s = max_over_ranks(time.perf_counter() - t0, dist)
        e2e_value = total_particles * e2e_steps * e2e_calls / e2e_s

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        reps = 3
        secs, bonds = cpu_reference(t, R, reps, threads)
        if secs is not None:
            cpu = {"value": threads * N * reps / secs, "unit": "particle-steps/s", "cores": threads,
                   "kind": "reference",
                   "sample": "reference h_CalculateForceElastic (bond slots only) over the %d bond slots of the "
                             "same specimen, %d passes x %d threads, one specimen copy per thread" % (bonds, reps,
                                                                                                     threads)}
    if rank != 0:
        return
    out = {"metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": ws, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": {"workload": WORKLOAD, "particles": N, "explicit_steps_per_bench_step": S, "slots_K": K,
                      "bonds_per_particle": round(bbar, 3), "contacts_per_particle": round(cbar, 3),
                      "l2": "inputs larger than L2 (state %.0f MB)" % ((N * K * 57 + N * 100) / 1e6),
                      "parallelism": "specimen-per-gpu" if ws > 1 else "single"},
           "e2e": {"value": e2e_value, "unit": "particle-steps/s", "h2d_bytes_per_step": 12 * N,
                   "d2h_bytes_per_step": 12 * N + 24 * e2e_steps,
                   "path": "md_CalculationUniaxialCompression, %d explicit steps per call incl. build" % e2e_steps},
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                        "traffic": (tr * N) if tr else None, "peak_source": peak_kind,
                        "kernel": "k_step (fused explicit step)",
                        "bytes_per_particle_step": round(b_step, 1)},
           "cpu_baseline": cpu,
           "gpu_launches": launches,
           "rebuilds": rebuilds,
           "clocks": clk}
    out["config"]["graph"] = graph_used
    print(json.dumps(out))
    if dist is not None:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the driver-call leg (profiling runs)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_engine(args)


if __name__ == "__main__":
    main()
