"""Benchmark: particle-steps/s of the explicit bonded-particle step, and wall time per
relaxed quasi-static load step (FIRE, warm-started vs plain).

Explicit workload (the large polydisperse uniaxial configuration): 4,000,000 particles
packed on the GPU, radii log-uniform in [0.5, 1.5] x 0.25 mm (radius ratio 3), a cylinder
of aspect 2 (D 65.7 x H 131.4 mm at packing fraction 0.58), bonded where the gap is below
0.05 r_min, kn = 1e11 N/m^3, ks = kn / 2.5, Weibull(m = 5) tensile / shear strengths with
scales 10 / 30 MPa, FP64 positions and FP32 forces, dt = 1e-8 s, platen strain rate
0.1/s, pairs listed within min(a_farcut, r_i + r_j + 0.25 r0). With these bonds a bond
fails only near 20 % stretch, which loading at 0.1/s does not reach in a benchmark's
steps; so the specimen is first pre-strained (rf_engine_affine_strain: +20 % laterally,
-3 % axially) and the timed steps run in that damaged state: bonds break and contacts
carry load in the window (both reported in config). One bench "step" is
STEPS_PER_BENCH_STEP explicit steps of the whole specimen (list maintenance, bond and
contact forces with the break check, platen, integration, cut, load reduction).

value : particle-steps/s of the fused engine, state resident in HBM, CUDA events on the
        engine's stream (max over ranks for N > 1).
e2e   : the same metric through the public API with host buffers: rf_engine_create_ext
        from pinned host positions and radii (bond construction included), the pre-strain,
        the steps, and the FP64 positions read back.
batch : 64 Brazilian discs of 5k-80k particles advanced by one step kernel
        (rf_engine_create_batch) vs one engine per specimen, particle-steps/s of both.
fire  : quasi-static load increments (strain 2.5e-5) of a 1M-particle cylinder (radii
        U[0.8, 1.2] x 0.25 mm) relaxed by FIRE to a residual of 1e-6 x the mean normal pair
        force: plain FIRE vs FIRE warm-started by the MLP trained on plain-FIRE pairs, and
        warm-started by the last increment's displacements; wall time per load step of each.
--impl reference : the reference's own CPU force path (h_CalculateForceElastic,
        md_calculateforcesbpm_cpu.cpp, built from its source into oracle/_ref) over the
        bond slots of a committed sample of the same specimen (a contiguous block of
        SAMPLE_N particles from the middle of the spatially numbered 4M specimen, which
        the engine arm checks bit for bit against its own), all host threads. It needs no
        part of the engine: bonds are found with scipy.

Multi-GPU: independent specimens per rank (different seeds), no data-path
collective; only the elapsed time is max-reduced.
"""
import argparse
import ctypes as C
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
R0_MM, PHI, ASPECT = 0.25, 0.58, 2.0
N_PARTICLES, RMIN, RMAX, RADII = 4000000, 0.5, 1.5, "log-uniform"
LIST_GAP = 0.25                          # x r0
PRESTRAIN = (0.2, 0.2, -0.03)            # lateral, lateral, axial
FIRE_PARTICLES = 1000000                 # the quasi-static configuration (radii U[0.8, 1.2] x r0)
FIRE_BATCH_SPECIMENS, FIRE_BATCH_INC = 8, 3   # quasi-static batch: specimens, timed increments
FIRE_PRE, FIRE_COLLECT, FIRE_EVAL = 1, 2, 20
SAMPLE_N = 65536                         # particles of the committed specimen sample
SAMPLE_FILE = os.path.join(ROOT, "oracle", "data", "bench_sample_4m.npz")
DIAMETER, HEIGHT = 52.0, 104.0           # the reference-model lattice specimen (198,061 particles)
METRIC = "particle-steps/s; wall time per relaxed load step, warm-start vs plain FIRE"


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_per_particle_step(name):
    """dram read+write bytes per particle-step of the step kernel from a committed ncu summary."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("traffic_bytes_per_particle_step:"):
            return float(line.split(":")[1])
    return None


def workload_name(args):
    dist = "U[%g,%g]" % (args.rmin, args.rmax) if args.radii == "uniform" else \
        "log-uniform [%g,%g]" % (args.rmin, args.rmax)
    pre = ("pre-strained %+g/%+g/%+g (x/y/z) into the damage regime" % tuple(args.prestrain)) if any(args.prestrain) \
        else "no pre-strain"
    return ("explicit BPM uniaxial compression, %d-particle polydisperse cylinder (radii %s x 0.25 mm, aspect 2, "
            "packing 0.58), gap < 0.05 r_min bonds, kn 1e11 N/m^3, ks kn/2.5, Weibull(5) strengths 10/30 MPa, "
            "FP64 positions / FP32 forces, dt 1e-8 s, 0.1/s, %s" % (args.particles, dist, pre))


def sample_block(N):
    """Index range of the specimen sample: SAMPLE_N consecutive particles from the middle
    of the spatially numbered specimen (a slab across the cylinder)."""
    n = min(SAMPLE_N, N)
    a = N // 2 - n // 2
    return a, a + n


def sample_bonds(R, rad, K=32, gap_frac=0.05, lam=0.330015):
    """Bond rows of a specimen sample by the extended model's rule (gap < gap_frac * min
    radius), in the reference's row layout, with each slot's bond radius lam * min(r_i, r_j)
    and 1/L0; found with a k-d tree (scipy), no part of the engine."""
    from scipy.spatial import cKDTree
    n = rad.size
    X = np.ascontiguousarray(R.reshape(3, n).T)
    tree = cKDTree(X)
    pairs = tree.query_pairs(2.0 * rad.max() * (1.0 + gap_frac), output_type="ndarray")
    i, j = pairs[:, 0], pairs[:, 1]
    d = np.sqrt(((X[i] - X[j]) ** 2).sum(1))
    keep = d - rad[i] - rad[j] < gap_frac * np.minimum(rad[i], rad[j])
    i, j, d = i[keep], j[keep], d[keep]
    a = np.concatenate([i, j])
    b = np.concatenate([j, i])
    dd = np.concatenate([d, d])
    order = np.lexsort((b, a))
    a, b, dd = a[order], b[order], dd[order]
    first = np.searchsorted(a, np.arange(n))
    slot = np.arange(a.size) - first[a]
    ok = slot < K
    IL = np.full(n * K, 0xFFFFFFFF, np.uint32)
    ty = np.zeros(n * K, np.uint8)
    iL = np.zeros(n * K, np.float32)
    br = np.zeros(n * K, np.float32)
    k = a[ok] * K + slot[ok]
    IL[k] = b[ok]
    ty[k] = 1
    iL[k] = (1.0 / dd[ok]).astype(np.float32)
    br[k] = (lam * np.minimum(rad[a[ok]], rad[b[ok]])).astype(np.float32)
    return IL, ty, iL, br, int(ok.sum())


def run_reference(args):
    """The reference's own CPU force path on the committed sample of the benchmark's
    specimen, all host threads (one sample copy per thread: the function walks a whole
    specimen). Loads only oracle/_ref/libmdref_cpu.so; nothing of the engine."""
    rank, ws, dist = dist_init()
    if rank != 0:
        return
    import oracle
    ref = oracle.ref_cpu()
    if ref is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libmdref_cpu.so not built "
                                                               "(reference tree absent at build time)"}))
        return
    if not os.path.exists(SAMPLE_FILE):
        print(json.dumps({"impl": "reference", "unavailable": "specimen sample %s missing" % SAMPLE_FILE}))
        return
    z = np.load(SAMPLE_FILE)
    R, rad = z["R"], z["radius"]
    n, K = rad.size, 32
    IL, ty, iL, br, bonds = sample_bonds(R, rad, K)
    Rf = R.astype(np.float32)
    V = np.zeros(3 * n, np.float32)
    W = np.zeros(3 * n, np.float32)
    # model units (mm, mg, us): stiffness per area kn = 1e11 N/m^3 -> E = kn * L0 at the mean
    # rest length; strengths 10 / 30 MPa; dt 1e-8 s
    kn = 1e11 / 1e12
    E = kn * float(np.mean(1.0 / iL[ty == 1]))
    G = E / 2.494
    threads = os.cpu_count() or 1
    ev = C.c_uint64(0)
    call = lambda reps: ref.ref_cpu_bond_forces_rb(Rf.ctypes.data, V.ctypes.data, W.ctypes.data, IL.ctypes.data,
                                                   ty.ctypes.data, iL.ctypes.data, n, K, 0.01, E, G, br.ctypes.data,
                                                   0.01, 0.03, reps, threads, C.byref(ev))
    call(1)
    for _ in range(max(args.warmup, 1) - 1):
        call(1)
    secs = call(args.steps)
    value = threads * n * args.steps / secs
    sample = ("reference h_CalculateForceElastic (md_calculateforcesbpm_cpu.cpp:20-288; bond slots only, no "
              "contacts, lists or integration) over all %d directed bond slots of the committed %d-particle "
              "sample of the benchmark specimen (particles %d..%d of the 4M specimen), per-bond radius "
              "0.330015 min(r_i, r_j), %d passes per thread, %d threads each on its own sample copy; one pass = "
              "one particle-step of every sample particle" % (bonds, n, int(z["first"]), int(z["first"]) + n - 1,
                                                              args.steps, threads))
    out = {"metric": METRIC, "value": value, "unit": "particle-steps/s", "impl": "reference", "n_gpus": ws,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": {"workload": workload_name(args), "particles": args.particles, "sample_particles": n,
                      "cpu_threads": threads, "same_specimen": "committed sample of the engine arm's specimen"},
           "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": threads, "kind": "reference",
                            "sample": sample},
           "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def ext_specimen(rfdem, N, seed, dist, rmin, rmax):
    R0, rad, D, H, mo = rfdem.pack_cylinder(N, R0_MM, rmin=rmin, rmax=rmax, aspect=ASPECT, phi=PHI, seed=seed,
                                            dist=dist)
    v = -0.1 * H * 1e-6                        # strain rate 0.1/s in mm per microsecond
    # the reference's fracture stop (stress above MinStress, then below ZeroStress) is kept
    # out of reach: a timed window is a fixed number of steps of the damaged specimen
    t, R = rfdem.make_test_ext(rfdem.RF_TEST_UNIAXIAL, R0, rad, R0_MM, dt=0.01, v_load=v, max_strain=1.0,
                               min_stress=1e30)
    return t, R, rad, D, H


def ext_bytes_per_particle_step(K, bbar, cbar):
    """Algorithmic bytes per particle-step of the fused extended-model step: FP64
    position (32 B) and FP32 velocity and spin (32 B) read and written, the K-slot row
    (id + type) once, the binning share, per bond record its partner id and slot (5),
    state read and written (96), rest length and strengths (16), per active contact its
    tangential overlap read and written (24)."""
    return 128 + 5 * K + 32 + 117 * bbar + 24 * cbar


def run_explicit(rfdem, torch, t, R, rad, x, args, dist):
    S = STEPS_PER_BENCH_STEP
    e = rfdem.Engine(t, R, ext=x, radius=rad)
    stream = torch.cuda.ExternalStream(e.stream())
    if any(args.prestrain):
        e.affine_strain(*args.prestrain)
    tuned = e.autotune(200) if not args.no_autotune else (0, [0.0, 0.0, 0.0])   # trials on a snapshot
    for _ in range(args.warmup):
        e.step(S)
    torch.cuda.synchronize()
    c0 = e.counters()
    _, r0 = e.sync()
    clocks = Clocks(torch.cuda.current_device())
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
    _, res = e.sync()
    done_steps = c1["steps"] - c0["steps"]
    if done_steps != S * args.steps:
        raise SystemExit("bench: the specimen finished early (%d of %d steps)" % (done_steps, S * args.steps))
    if res.error:
        raise SystemExit("bench: engine error %d (%s)" % (res.error, rfdem.STATUS.get(res.error, "?")))
    graph = e.uses_graph()
    e.close()
    return dict(ms=ms, c0=c0, c1=c1, clocks=clk, graph=graph, tuned=tuned,
                broken_window=int(res.broken_bonds - r0.broken_bonds), broken_total=int(res.broken_bonds),
                bonds_initial=int(res.bonds_initial))


def run_fire(rfdem, torch, seed, n_eval):
    """Quasi-static load steps of the 1M-particle cylinder: two engines in lockstep take
    FIRE_PRE + FIRE_COLLECT plain increments (the MLP is trained on the plain engine's
    FIRE_COLLECT relaxation pairs), then n_eval increments each: one plain, one
    warm-started by the MLP. Wall time per relaxed load step of each. A third engine,
    warm-started by its own last increment's displacements (rotations from zero), is the
    predictor-free reference the MLP has to beat."""
    from rfdem.warm import WarmStart
    t, R, rad, D, H = ext_specimen(rfdem, FIRE_PARTICLES, seed, "uniform", 0.8, 1.2)
    x = rfdem.ext_params_si()
    x.list_gap = LIST_GAP * R0_MM
    FIRE_N = int(t.N)
    A = rfdem.Engine(rfdem.Task.from_buffer_copy(t), R, ext=x, radius=rad)
    B = rfdem.Engine(rfdem.Task.from_buffer_copy(t), R, ext=x, radius=rad)
    Cn = rfdem.Engine(rfdem.Task.from_buffer_copy(t), R, ext=x, radius=rad)
    p = A.relax_params(max_iter=60000)
    ws = WarmStart(FIRE_N, p.strain_inc, seed=seed)
    for k in range(FIRE_PRE + FIRE_COLLECT):
        collect = k >= FIRE_PRE
        if collect:
            ws.features(A)
        A.load_increment(p)
        B.load_increment(p)
        Cn.load_increment(p)
        if collect:
            ws.collect(A)
    t0 = time.perf_counter()
    losses = ws.train()
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    plain, warm, last = [], [], []
    for k in range(n_eval):
        t0 = time.perf_counter()
        ra = A.load_increment(p)
        ta = time.perf_counter() - t0
        # MLP warm start behind its gate (the gate's scoring of the increment is timed too)
        t0 = time.perf_counter()
        Y = ws.predict(B)
        rb = B.load_increment_pred(p, Y, 16)
        ws.observe(B)
        tb = time.perf_counter() - t0
        # the last increment's motion alone (exact, from the device)
        t0 = time.perf_counter()
        Yc = ws.predict(Cn, use_mlp=False)
        rc = Cn.load_increment_pred(p, Yc, 16)
        tc = time.perf_counter() - t0
        plain.append((ta, ra.iterations, ra.converged, ra.stress))
        warm.append((tb, rb.iterations, rb.converged, rb.stress))
        last.append((tc, rc.iterations, rc.converged, rc.stress))
    A.close(); B.close(); Cn.close(); ws.close()
    tp = sum(a[0] for a in plain) / n_eval
    tw = sum(a[0] for a in warm) / n_eval
    tl = sum(a[0] for a in last) / n_eval
    mpa = lambda v: [round(a[3] * rfdem.STRESS * 1e-6, 6) for a in v]     # platen stress, MPa
    return {"workload": "quasi-static uniaxial load steps of strain %.1e of a %d-particle cylinder (radii "
                        "U[0.8,1.2] x 0.25 mm, D %.1f x H %.1f mm), FIRE (stiffness-scaled masses) to RMS net force "
                        "<= 1e-6 x mean normal pair force" % (p.strain_inc, FIRE_N, D, H),
            "particles": FIRE_N, "evaluated_increments": n_eval,
            "wall_s_per_load_step_plain": tp, "wall_s_per_load_step_warm": tw, "speedup_warm_vs_plain": tp / tw,
            "wall_s_per_load_step_last_increment_warm": tl, "speedup_last_increment_vs_plain": tp / tl,
            "iterations_plain": [a[1] for a in plain], "iterations_warm": [a[1] for a in warm],
            "iterations_last_increment_warm": [a[1] for a in last],
            "converged_plain": [a[2] for a in plain], "converged_warm": [a[2] for a in warm],
            "converged_last_increment_warm": [a[2] for a in last],
            "stress_mpa_plain": mpa(plain), "stress_mpa_warm": mpa(warm), "stress_mpa_last_increment_warm": mpa(last),
            "mlp_error_over_last_increment_error": [round(r, 4) for r, _ in ws.log],
            "mlp_used": [int(u) for _, u in ws.log],
            "last_increment_relative_error": [round(v, 5) for v in ws.base_error],
            "training_pairs": ws.pairs(), "training_loss": [losses[0], losses[-1]], "training_s": t_train,
            "warm_start_includes": "feature build + last-increment motion + MLP forward (tcgen05 BF16) + gate "
                                   "scoring per load step"}


def run_fire_long(n_inc):
    """A long quasi-static run of the FIRE specimen: one plain increment, then n_inc
    increments warm-started by each particle's last-increment motion; per increment its
    iterations, convergence, platen stress (MPa) and wall time."""
    import torch
    import rfdem
    from rfdem.warm import WarmStart
    seed = 0xB2000000 + 3000
    t, R, rad, D, H = ext_specimen(rfdem, FIRE_PARTICLES, seed, "uniform", 0.8, 1.2)
    x = rfdem.ext_params_si()
    x.list_gap = LIST_GAP * R0_MM
    e = rfdem.Engine(rfdem.Task.from_buffer_copy(t), R, ext=x, radius=rad)
    p = e.relax_params(max_iter=60000)
    ws = WarmStart(int(t.N), p.strain_inc, seed=seed)
    r0 = e.load_increment(p)
    rows = []
    t_all = time.perf_counter()
    for k in range(n_inc):
        t0 = time.perf_counter()
        r = e.load_increment_pred(p, ws.predict(e, use_mlp=False), 16)
        rows.append((r.iterations, r.converged, r.stress * rfdem.STRESS * 1e-6, time.perf_counter() - t0))
    wall = time.perf_counter() - t_all
    e.close(); ws.close()
    print(json.dumps({"record": "quasi-static run, last-increment warm start",
                      "workload": "%d-particle cylinder (radii U[0.8,1.2] x 0.25 mm, D %.1f x H %.1f mm), %d increments "
                                  "of strain %.1e after one plain increment (%d iterations)"
                                  % (int(t.N), D, H, n_inc, p.strain_inc, r0.iterations),
                      "increments": n_inc, "wall_s": wall, "wall_s_per_increment": wall / n_inc,
                      "all_converged": int(min(a[1] for a in rows)),
                      "iterations": [a[0] for a in rows], "stress_mpa": [round(a[2], 6) for a in rows],
                      "iterations_total": sum(a[0] for a in rows)}))


def run_fire_batch(rfdem, torch, seed):
    """Quasi-static load steps of a batch: FIRE_BATCH_SPECIMENS uniaxial cylinders (particle
    counts log-uniform in [50k, 200k], radii U[0.8, 1.2] x 0.25 mm, own seeds) relaxed
    together (rf_engine_load_increment_batch, each specimen on its own FIRE scalars), plain
    and warm-started by each particle's last-increment motion, against the same specimens
    one engine each, one after the other. Wall time per load step of the whole set."""
    from rfdem.warm import WarmStart
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(np.log(50000), np.log(200000), FIRE_BATCH_SPECIMENS)).astype(int)
    tasks, params, Rs, rads = [], [], [], []
    x = rfdem.ext_params_si()
    x.list_gap = LIST_GAP * R0_MM
    t0 = time.perf_counter()
    for q in range(FIRE_BATCH_SPECIMENS):
        t, R, rad, D, H = ext_specimen(rfdem, int(counts[q]), seed + q, "uniform", 0.8, 1.2)
        tasks.append(t); params.append(x); Rs.append(R); rads.append(rad)
    t_pack = time.perf_counter() - t0
    ntot = int(sum(int(t.N) for t in tasks))
    P = rfdem.BatchEngine(tasks, params, Rs, rads)          # plain
    W = rfdem.BatchEngine(tasks, params, Rs, rads)          # warm-started
    p = P.relax_params(max_iter=60000)
    ws = WarmStart(ntot, p.strain_inc, seed=seed)
    for E in (P, W):
        E.load_increment(p)                                # one increment before: the warm start's base
    plain, warm = [], []
    for k in range(FIRE_BATCH_INC):
        t0 = time.perf_counter()
        rp = P.load_increment(p)
        plain.append((time.perf_counter() - t0, [r.iterations for r in rp], min(r.converged for r in rp)))
        t0 = time.perf_counter()
        rw = W.load_increment_pred(p, ws.predict(W, use_mlp=False), 16)
        warm.append((time.perf_counter() - t0, [r.iterations for r in rw], min(r.converged for r in rw)))
    P.close(); W.close(); ws.close()
    seq, seq_it, seq_conv = 0.0, [], 1
    for q in range(FIRE_BATCH_SPECIMENS):
        e = rfdem.Engine(rfdem.Task.from_buffer_copy(tasks[q]), Rs[q], ext=params[q], radius=rads[q])
        e.load_increment(p)
        its = []
        for k in range(FIRE_BATCH_INC):
            t0 = time.perf_counter()
            r = e.load_increment(p)
            seq += time.perf_counter() - t0
            its.append(r.iterations)
            seq_conv = min(seq_conv, r.converged)
        seq_it.append(its)
        e.close()
    tb = sum(a[0] for a in plain) / FIRE_BATCH_INC
    tw = sum(a[0] for a in warm) / FIRE_BATCH_INC
    ts = seq / FIRE_BATCH_INC
    return {"workload": "%d uniaxial cylinders, %d particles in all (%d to %d each, log-uniform), quasi-static load "
                        "steps of strain %.1e, FIRE to RMS net force <= 1e-6 x mean normal pair force"
                        % (FIRE_BATCH_SPECIMENS, ntot, int(counts.min()), int(counts.max()), p.strain_inc),
            "evaluated_increments": FIRE_BATCH_INC, "packing_s": t_pack,
            "wall_s_per_load_step_batched_plain": tb, "wall_s_per_load_step_batched_warm": tw,
            "wall_s_per_load_step_one_engine_each": ts,
            "speedup_batched_vs_one_engine_each": ts / tb, "speedup_batched_warm_vs_one_engine_each": ts / tw,
            "iterations_batched_plain": [a[1] for a in plain], "iterations_batched_warm": [a[1] for a in warm],
            "iterations_one_engine_each": seq_it,
            "all_converged": int(min([a[2] for a in plain] + [a[2] for a in warm] + [seq_conv])),
            "warm_start": "each particle's last-increment motion (WarmStart.predict(use_mlp=False))"}


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
    """One process per GPU under torchrun (NCCL); gloo when no GPU is present (tests)."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return 0, 1, None
    import torch
    import torch.distributed as dist
    rank = int(os.environ["RANK"])
    backend = "nccl" if torch.cuda.is_available() else "gloo"
    if backend == "nccl":
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", rank)))
    import datetime
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return rank, ws, dist


def _reduce(x, dist, op):
    if dist is None:
        return x
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(x, dist):
    return x if dist is None else _reduce(x, dist, dist.ReduceOp.MAX)


def sum_over_ranks(x, dist):
    return x if dist is None else _reduce(x, dist, dist.ReduceOp.SUM)


def rank_seed(rank):
    """Each rank packs its own specimen: weak scaling, no data-path collective."""
    return 0xB2000000 + 2000 + rank


BATCH_SPECIMENS, BATCH_STEPS, BATCH_FULL_CAP = 64, 1000, 300000


def run_batch_to_failure(rfdem, torch, tasks, params, Rs, rads, counts, t_pack, cap=BATCH_FULL_CAP):
    """The batch run to completion: every specimen to its 50 % post-peak load drop (or
    the step cap), one step kernel for all; device time of the whole run and each
    specimen's stop step, peak stress and broken bonds."""
    be = rfdem.BatchEngine(tasks, params, Rs, rads)
    s = torch.cuda.ExternalStream(be.stream())
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    chunk, done_steps, ms = 20000, 0, 0.0
    while done_steps < cap:
        a.record(s)
        be.step(chunk)
        b.record(s)
        b.synchronize()
        ms += a.elapsed_time(b)
        done_steps += chunk
        res = [be.sync_spec(q)[1] for q in range(len(tasks))]
        if all(r.Fracture or r.steps < done_steps for r in res):
            break
    res = [be.sync_spec(q)[1] for q in range(len(tasks))]
    be.close()
    ps = sum(int(tasks[q].N) * int(res[q].steps) for q in range(len(tasks)))
    return {"workload": "%d Brazilian discs run to a 50 %% post-peak load drop, %d particles in all (%d to %d each, "
                        "log-uniform), own seeds and Weibull moduli U[3,10], platens 0.05 m/s, dt 1e-8 s"
                        % (len(tasks), int(sum(int(t.N) for t in tasks)), int(counts.min()), int(counts.max())),
            "device_s": ms * 1e-3, "specimen_particle_steps_per_s": ps / (ms * 1e-3),
            "stopped_post_peak": int(sum(1 for r in res if r.Fracture)), "step_cap": cap,
            "stop_steps": [int(r.steps) for r in res],
            "peak_stress_MPa": [round(r.FractureStress * 1e3, 3) for r in res],
            "broken_bonds": [int(r.broken_bonds) for r in res], "packing_s": t_pack}


def run_batch(rfdem, torch, seed, full=False):
    """The batched-disc workload: BATCH_SPECIMENS Brazilian discs (thickness = D/2) with
    particle counts log-uniform in [5k, 80k], radii U[0.8, 1.2] x 0.25 mm, Weibull
    modulus U[3, 10] per specimen (own seed each), platens at 0.05 m/s, dt 1e-8 s; all
    advanced by one step kernel per step (rf_engine_create_batch) vs the same specimens
    one engine each, run one after the other. Particle-steps/s of both."""
    import ctypes as C
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(np.log(5000), np.log(80000), BATCH_SPECIMENS)).astype(int)
    ms = rng.uniform(3.0, 10.0, BATCH_SPECIMENS)
    tasks, params, Rs, rads = [], [], [], []
    t0 = time.perf_counter()
    for q in range(BATCH_SPECIMENS):
        R0, rad, D, H, mo = rfdem.pack_cylinder(int(counts[q]), R0_MM, aspect=0.5, phi=PHI, seed=seed + q)
        t, R = rfdem.make_test_ext(rfdem.RF_TEST_BRAZIL, R0, rad, R0_MM, dt=0.01, v_load=-5e-5, max_strain=1.0)
        x = rfdem.ext_params_si(weibull_m=float(ms[q]), seed=seed + 1000 + q)
        x.post_peak_drop = 0.5                    # each specimen stops after a 50 % post-peak load drop
        tasks.append(t); params.append(x); Rs.append(R); rads.append(rad)
    t_pack = time.perf_counter() - t0
    ntot = int(sum(int(t.N) for t in tasks))
    if full:
        return run_batch_to_failure(rfdem, torch, tasks, params, Rs, rads, counts, t_pack)
    be = rfdem.BatchEngine(tasks, params, Rs, rads)
    s = torch.cuda.ExternalStream(be.stream())
    be.step(BATCH_STEPS)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(s)
    for _ in range(3):
        be.step(BATCH_STEPS)
    b.record(s)
    b.synchronize()
    ms_batch = a.elapsed_time(b)
    steps_done = [be.sync_spec(q)[1].steps for q in range(BATCH_SPECIMENS)]
    be.close()
    done_batch = sum(int(tasks[q].N) * (steps_done[q] - BATCH_STEPS) for q in range(BATCH_SPECIMENS))
    ms_seq = 0.0
    done_seq = 0
    for q in range(BATCH_SPECIMENS):
        e = rfdem.Engine(rfdem.Task.from_buffer_copy(tasks[q]), Rs[q], ext=params[q], radius=rads[q])
        sq = torch.cuda.ExternalStream(e.stream())
        e.step(100)
        torch.cuda.synchronize()
        a.record(sq)
        e.step(BATCH_STEPS)
        b.record(sq)
        b.synchronize()
        ms_seq += a.elapsed_time(b)
        done_seq += int(tasks[q].N) * (e.counters()["steps"] - 100)
        e.close()
    v_b = done_batch / (ms_batch * 1e-3)
    v_s = done_seq / (ms_seq * 1e-3)
    return {"workload": "%d Brazilian discs, %d particles in all (%d to %d each, log-uniform), own seeds and "
                        "Weibull moduli U[3,10]" % (BATCH_SPECIMENS, ntot, int(counts.min()), int(counts.max())),
            "batched_particle_steps_per_s": v_b, "one_engine_each_particle_steps_per_s": v_s,
            "speedup_batched": v_b / v_s, "batched_ms_per_step": ms_batch / (3 * BATCH_STEPS),
            "packing_s": t_pack, "specimens_finished_early": int(sum(1 for q in range(BATCH_SPECIMENS)
                                                                     if steps_done[q] < 4 * BATCH_STEPS))}


def run_fit_step(rfdem):
    """One step of the material fitter at the reference's specimen sizes (cylinder D 12.5 x
    H 25 mm, disc D 25 x 10 mm, p_r 0.5 mm): its 12 simulations to fracture, all engines
    launched before any is waited on vs one after the other; wall time of each (engine
    creation included) and the simulations' particle-steps."""
    from rfdem import fit
    S = fit.Specimens()
    out = {}
    for mode, conc in (("concurrent", True), ("sequential", False)):
        T = fit.FitTask(2)
        T.calculate_start_parameters()
        t0 = time.perf_counter()
        steps = fit.evaluate(T, S, concurrent=conc)
        out[mode + "_s"] = time.perf_counter() - t0
        out["runs"] = len(steps)
        out["steps_per_run"] = sorted(steps.values())
        out["results_" + mode] = T.RFunction.tolist()
    out["speedup_concurrent"] = out["sequential_s"] / out["concurrent_s"]
    out["same_results"] = out["results_concurrent"] == out["results_sequential"]
    del out["results_sequential"]
    out["workload"] = ("one conjugate-gradient step of the reference's material fitter: 6 parameter sets x "
                       "(uniaxial + Brazilian) to fracture, reference model")
    return out


def check_sample(R, rad, write_path=None):
    """The specimen's sample block against the committed file (bit for bit), or written."""
    N = rad.size
    a, b = sample_block(N)
    P = R.reshape(3, N)[:, a:b]
    if write_path:
        os.makedirs(os.path.dirname(os.path.abspath(write_path)), exist_ok=True)
        np.savez_compressed(write_path, R=np.ascontiguousarray(P).reshape(-1), radius=rad[a:b].copy(), first=a,
                            total=N)
    if not os.path.exists(SAMPLE_FILE):
        return None
    z = np.load(SAMPLE_FILE)
    return bool(int(z["first"]) == a and int(z["total"]) == N and np.array_equal(z["R"], P.reshape(-1)) and
                np.array_equal(z["radius"], rad[a:b]))


def cpu_port_sample(rfdem, t, x, R, rad, prestrain):
    """The oracle's restatement of the extended-model step (the engine's arithmetic) on the
    committed sample block of the same specimen, pre-strained the same way, on all host
    threads; bond construction and pre-strain untimed."""
    import oracle
    N = rad.size
    a, b = sample_block(N)
    Rb = np.ascontiguousarray(R.reshape(3, N)[:, a:b]).reshape(-1)
    ts, Rs = rfdem.make_test_ext(rfdem.RF_TEST_UNIAXIAL, Rb, rad[a:b], R0_MM, dt=0.01, v_load=float(t.Compress.VLoad),
                                 max_strain=1.0, min_stress=1e30)
    threads = os.cpu_count() or 1
    secs, n = oracle.time_ext(rfdem.Task.from_buffer_copy(ts), x, Rs, rad[a:b], 2, threads, prestrain)
    steps = max(2, min(200, int(15.0 / max(secs / 2, 1e-3))))
    secs, n = oracle.time_ext(rfdem.Task.from_buffer_copy(ts), x, Rs, rad[a:b], steps, threads, prestrain)
    return {"value": (b - a) * n / secs, "unit": "particle-steps/s", "cores": threads, "kind": "port",
            "sample": "oracle restatement of the extended-model explicit step (float forces, FP64 positions, lists, "
                      "bonds, contacts, integration), %d steps of the %d-particle sample block of the same specimen "
                      "(its own platens), pre-strained the same way, on %d host threads (OpenMP); construction "
                      "untimed" % (n, b - a, threads)}


def run_engine(args):
    import torch
    rank, ws, dist = dist_init()
    import rfdem
    S = STEPS_PER_BENCH_STEP
    t0 = time.perf_counter()
    t, R, rad, Dm, Hm = ext_specimen(rfdem, args.particles, rank_seed(rank), args.radii, args.rmin, args.rmax)
    t_pack = time.perf_counter() - t0
    same_sample = check_sample(R, rad, args.write_sample if rank == 0 else None) if rank == 0 else None
    x = rfdem.ext_params_si()
    x.list_gap = args.list_gap * R0_MM
    N = int(t.N)
    K = int(t.K)
    r = run_explicit(rfdem, torch, rfdem.Task.from_buffer_copy(t), R, rad, x, args, dist)
    ms = r["ms"]
    ms_max = max_over_ranks(ms, dist)
    total_particles = sum_over_ranks(float(N), dist)
    value = total_particles * S * args.steps / (ms_max * 1e-3)
    c1, c0 = r["c1"], r["c0"]
    bbar = 0.5 * (c0["bonds"] + c1["bonds"]) / N
    cbar = 0.5 * (c0["contacts"] + c1["contacts"]) / N
    b_step = ext_bytes_per_particle_step(K, bbar, cbar)
    per_step_s = (ms * 1e-3) / (S * args.steps)
    achieved = b_step * N / per_step_s / 1e9
    peak, peak_kind = peaks()
    tr = traffic_per_particle_step("k_step_ext_uniaxial-4m-prestrained.md")
    rebuilds = c1["rebuilds"] - c0["rebuilds"]
    launches = S * args.steps + 7 * rebuilds + 2 * args.steps

    # e2e through the public API with host buffers (pinned): create, pre-strain, steps, read back
    import ctypes as C
    e2e_value = None
    e2e_calls = 0 if args.no_e2e else 3
    if e2e_calls:
        hR = torch.from_numpy(R).pin_memory()
        hrad = torch.from_numpy(rad).pin_memory()
        hout = torch.empty_like(hR).pin_memory()
        strain = (C.c_double * 3)(*args.prestrain)

        def e2e_call():
            tt = rfdem.Task.from_buffer_copy(t)
            h = rfdem.P()
            rfdem.check(rfdem.lib.rf_engine_create_ext(C.byref(tt), C.byref(x), hR.data_ptr(), hrad.data_ptr(),
                                                       C.byref(h)), "e2e create")
            if any(args.prestrain):
                rfdem.check(rfdem.lib.rf_engine_affine_strain(h, strain), "e2e pre-strain")
            rfdem.check(rfdem.lib.rf_engine_step(h, S), "e2e step")
            rfdem.check(rfdem.lib.rf_engine_positions_f64(h, hout.data_ptr()), "e2e positions")
            rfdem.lib.rf_engine_destroy(h)
        e2e_call()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        t1 = time.perf_counter()
        for _ in range(e2e_calls):
            e2e_call()
        torch.cuda.synchronize()
        e2e_s = max_over_ranks(time.perf_counter() - t1, dist)
        e2e_value = total_particles * S * e2e_calls / e2e_s

    # the reference's own model (mono-sized lattice, FP32 state), reference-exact engine
    refmodel = None
    if not args.no_reference_model:
        tr_, Rr = rfdem.make_test(rfdem.RF_TEST_UNIAXIAL, DIAMETER, HEIGHT, seed=0xB2000000 + 2000 + rank,
                                  max_strain=1.0)
        er = rfdem.Engine(tr_, Rr)
        sr = torch.cuda.ExternalStream(er.stream())
        for _ in range(args.warmup):
            er.step(S)
        torch.cuda.synchronize()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(sr)
        for _ in range(args.steps):
            er.step(S)
        a1.record(sr)
        a1.synchronize()
        mr = max_over_ranks(a0.elapsed_time(a1), dist)
        Nr = int(tr_.N)
        cr = er.counters()
        er.close()
        refmodel = {"workload": "reference model (mono-sized granite BPM, FP32 state, bit-exact with the reference), "
                                "198k-particle lattice cylinder D52xH104 mm",
                    "particles": Nr, "value": sum_over_ranks(float(Nr), dist) * S * args.steps / (mr * 1e-3),
                    "unit": "particle-steps/s", "ms_per_step": mr / args.steps,
                    "bytes_per_particle_step": round(72 + 5 * K + 32 + 105 * cr["bonds"] / Nr
                                                     + 24 * cr["contacts"] / Nr, 1)}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_port_sample(rfdem, t, x, R, rad, args.prestrain)

    batch = None
    if rank == 0 and ws == 1 and not args.no_batch:
        batch = run_batch(rfdem, torch, 0xB2000000 + 4000, full=args.batch_full)

    fitstep = None
    if rank == 0 and ws == 1 and args.fit:
        fitstep = run_fit_step(rfdem)

    fire = None
    if rank == 0 and ws == 1 and not args.no_fire:
        fire = run_fire(rfdem, torch, 0xB2000000 + 3000, args.fire_eval)
        fire["batch"] = run_fire_batch(rfdem, torch, 0xB2000000 + 5000)
    if rank != 0:
        return
    out = {"metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": ws, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32 forces, f64 positions", "data": "synthetic",
           "config": {"workload": workload_name(args), "particles": N, "specimen_mm": [round(Dm, 2), round(Hm, 2)],
                      "packing_s": round(t_pack, 1), "explicit_steps_per_bench_step": S, "slots_K": K,
                      "list_rule": ("pairs within min(a_farcut, r_i + r_j + %g mm)" % x.list_gap) if x.list_gap > 0
                      else "pairs within a_farcut (the reference's)",
                      "prestrain_xyz": list(args.prestrain),
                      "bonds_per_particle": round(bbar, 3), "contacts_per_particle": round(cbar, 3),
                      "bonds_broken_in_window": r["broken_window"], "bonds_broken_total": r["broken_total"],
                      "bond_slots_initial": r["bonds_initial"],
                      "sample_matches_committed_file": same_sample,
                      "l2": "inputs larger than L2 (state %.0f MB)" % ((N * K * 16 + N * 300 + c1["bonds"] * 129) / 1e6),
                      "parallelism": "specimen-per-gpu" if ws > 1 else "single", "graph": r["graph"],
                      "autotune": {"ctas_per_sm": r["tuned"][0],
                                   "ms_per_200_steps_for_8_6_5": [round(v, 3) for v in r["tuned"][1]]}},
           "e2e": {"value": e2e_value, "unit": "particle-steps/s", "h2d_bytes_per_step": 32 * N,
                   "d2h_bytes_per_step": 24 * N,
                   "path": "rf_engine_create_ext (host positions + radii, bond build) + rf_engine_affine_strain + %d "
                           "explicit steps + rf_engine_positions_f64 per call" % S},
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                        "traffic": (tr * N) if tr else None, "peak_source": peak_kind,
                        "kernel": "k_step_ext (fused explicit step, extended model)",
                        "bytes_per_particle_step": round(b_step, 1)},
           "cpu_baseline": cpu,
           "gpu_launches": launches,
           "rebuilds": rebuilds,
           "clocks": r["clocks"],
           "fire": fire,
           "batch": batch,
           "fit": fitstep,
           "reference_model": refmodel}
    print(json.dumps(out))
    if dist is not None:
        dist.destroy_process_group()


def main():
    global STEPS_PER_BENCH_STEP
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the driver-call leg (profiling runs)")
    ap.add_argument("--no-fire", action="store_true", help="skip the quasi-static FIRE comparison")
    ap.add_argument("--fire-eval", type=int, default=FIRE_EVAL, help="evaluated FIRE load increments")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-specimen comparison")
    ap.add_argument("--explicit-steps", type=int, default=STEPS_PER_BENCH_STEP,
                    help="explicit steps per bench step (profiling runs use fewer)")
    ap.add_argument("--no-reference-model", action="store_true", help="skip the reference-model line")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default step variant (profiling runs)")
    ap.add_argument("--particles", type=int, default=N_PARTICLES, help="particles of the benchmark specimen")
    ap.add_argument("--radii", default=RADII, choices=["uniform", "log-uniform"])
    ap.add_argument("--rmin", type=float, default=None, help="smallest radius / 0.25 mm (0.5; 0.8 uniform)")
    ap.add_argument("--rmax", type=float, default=None, help="largest radius / 0.25 mm (1.5; 1.2 uniform)")
    ap.add_argument("--list-gap", type=float, default=LIST_GAP,
                    help="list gap / 0.25 mm: pairs listed within min(a_farcut, r_i + r_j + gap) "
                         "(0 is the reference's uniform cutoff a_farcut)")
    ap.add_argument("--prestrain", type=float, nargs=3, default=list(PRESTRAIN),
                    help="homogeneous pre-strain x y z applied before the warm-up (0 0 0: none)")
    ap.add_argument("--write-sample", default=None, help="write the specimen's sample block to this .npz")
    ap.add_argument("--fit", action="store_true", help="time one material-fitter step (12 runs to fracture)")
    ap.add_argument("--fire-long", type=int, default=0,
                    help="only this many quasi-static increments of the 1M FIRE specimen, warm-started by the "
                         "last increment's motion; prints their iterations (a record run, not a bench line)")
    ap.add_argument("--batch-full", action="store_true",
                    help="run the 64-disc batch to every specimen's post-peak drop instead of the timed window")
    args = ap.parse_args()
    if args.rmin is None:
        args.rmin = 0.8 if args.radii == "uniform" else 0.5
    if args.rmax is None:
        args.rmax = 1.2 if args.radii == "uniform" else 1.5
    if args.warmup < 3:
        args.warmup = 3
    STEPS_PER_BENCH_STEP = max(1, args.explicit_steps)
    if args.impl == "reference":
        run_reference(args)
    elif args.fire_long > 0:
        run_fire_long(args.fire_long)
    else:
        run_engine(args)


if __name__ == "__main__":
    main()
