"""Benchmark: Dormand-Prince 5(4) attempts per second on the 64x64 two-band
electron-phonon workload, with the collision operator's HBM roofline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--layout auto|mc64|t64|t32] [--mixed]

A "step" is one DP45 attempt: six right-hand-side evaluations (collision
operator over all scattering channels + Vlasov drift + M^-1), the fused stage
combinations, the embedded error norm and the step-size controller, all on the
device (one CUDA graph launch).  Workload (synthetic, seeded): k-space
[-1,1]^2, 64x64 sections (8192 P1 triangles per band), bands parabola
E=|k|^2/2 and Dirac cone E=|k|+0.5 plus a dispersionless optical phonon
(hw = 0.2, Bose occupation at kT = 0.05), e-ph channels {el,pn,el} {in,in,out}
with unit coupling, drift field (0.1, 0), rtol 1e-8 / atol 1e-9, NMC = 50.
The four-leg e-e channel of that configuration is left out: at 64x64 it has
~9e10 surviving tuples per channel per RHS evaluation (measured scaling
~N^5.2), beyond any single GPU for a time integration.

Multi-GPU: runs are independent replicas (the path has no exchange step);
`value` is the aggregate over ranks, timed as the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DP45 steps/s & collision-op HBM GB/s, batched mixed vs plain FP64 GPU at ≤1e-8 rel err"
N_MESH = 64
T_END = 20.0
DENSE = T_END / 10.0


def workload(n_mesh=N_MESH):
    from tortoise_b200 import workloads as W
    mat = W.two_band_eph_drift(n_mesh)
    f0 = W.initial_status(mat, kT=0.1, seed=1).vec
    return mat, f0


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join(os.environ.get("TB_CLOCKS_DIR", tempfile.gettempdir()), "bench_clocks_%d.csv" % os.getpid())

    def __enter__(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if not self.proc or not os.path.exists(self.path):
            return None
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        loaded = [x for x in sm if x > 0.5 * (mx or max(sm))] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if args.impl == "ours" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=180))
        pg = dist
    return world, rank, local, pg


def reduce_max(pg, x, device):
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(world, steps_per_rank, t_max):
    """Whole-job throughput of replicas: every rank did steps_per_rank steps,
    the job took the slowest rank's time."""
    return world * steps_per_rank / t_max


WORKLOAD = "2-band e-ph + drift, 64x64 mesh (8192 triangles/band), NMC=50, rtol 1e-8"


def base_config(ntup, nch, ndofs, world):
    """The config object both arms print: the workload and its sizes only
    (kernel layouts and schedules go under "kernels")."""
    return {"workload": WORKLOAD, "tuples": int(ntup), "channels": int(nch), "dofs": int(ndofs),
            "parallelism": "replicas x%d" % world}


def cpu_rhs_full(o, f):
    """One whole right-hand side of the oracle (every tuple of every channel,
    drift, M^-1) on its threads; returns (seconds, dfdt)."""
    t0 = time.perf_counter()
    out = o.rhs(f, drift=True)
    return time.perf_counter() - t0, out


def cpu_rhs_sample(o, mat, f, frac):
    """One RHS evaluation of the oracle on the first `frac` of every channel's
    tuples plus the full drift term; returns seconds scaled to the full list."""
    t0 = time.perf_counter()
    acc = np.zeros(o.ndofs)
    t_coll = 0.0
    for ch in range(len(mat.channels)):
        n = o.num_tuples(ch)
        m = max(1, int(n * frac))
        a = time.perf_counter()
        o.channel_propagate(ch, f, 0, m, out=acc)
        t_coll += (time.perf_counter() - a) * (n / m)
    a = time.perf_counter()
    for b, band in enumerate(mat.bands):
        if band.drift_velocity != (0.0, 0.0):
            off = o.band_offset(b)
            o.vlasov(b, f[off:off + band.mesh.ne * 3])
    t_drift = time.perf_counter() - a
    return t_coll + t_drift, time.perf_counter() - t0


def reference_arm(args, world, rank):
    """The reference's CPU path (restated: the reference itself needs Eigen
    and oneTBB, which are absent), timed on all host cores.  A step is one
    DP45 attempt's six whole right-hand sides (every tuple of every channel,
    drift, M^-1), each timed; the stage combinations and the error norm cost
    microseconds beside them and are left out."""
    if rank != 0:
        return
    import oracle
    mat, f0 = workload()
    o = oracle.Oracle(mat, nthreads=os.cpu_count())
    nch = len(mat.channels)
    ntup = sum(o.num_tuples(c) for c in range(nch))
    times = []
    for i in range(args.warmup + args.steps):
        t_att = sum(cpu_rhs_full(o, f0)[0] for _ in range(6))
        if i >= args.warmup:
            times.append(t_att)
    v = len(times) / sum(times)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "DP45 steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded PCG64 bump on Fermi-Dirac, Bose phonons)",
            "config": base_config(ntup, nch, o.ndofs, world),
            "cpu_baseline": {"value": v, "unit": "DP45 steps/s", "cores": os.cpu_count(), "kind": "port",
                             "sample": "each step: 6 whole right-hand sides (all %d tuples, drift, M^-1), "
                                       "measured, not extrapolated" % ntup},
            "e2e": {"value": v, "unit": "DP45 steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def moment_bytes(L, layout):
    """Bytes of one tuple's stored moments: 3^L (1 + L) moments as FP64 (t64),
    FP32 (t32) or the upper 40 bits of FP64 (t40: a 4-byte word plus one
    byte, bytes packed four per word)."""
    nm = {2: 27, 3: 108, 4: 405}[L]
    return {"t64": 8 * nm, "t32": 4 * nm, "t40": 4 * (nm + (nm + 3) // 4),
            "t48": 4 * (nm + (nm + 1) // 2)}.get(layout, 0)


def mixed_flag(args):
    return {None: 0, "t32": 1, "t40": 2, "t48": 3}[args.mixed]


def ours(args, world, rank, local, pg):
    import torch
    from tortoise_b200 import engine as E
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    mat, f0 = workload()
    layout = {"auto": E.LAYOUT_AUTO, "mc64": E.LAYOUT_MC64, "t64": E.LAYOUT_T64, "t32": E.LAYOUT_T32,
              "t40": E.LAYOUT_T40, "t48": E.LAYOUT_T48}[args.layout]
    eng = E.Engine(mat, layout=layout, allow_fp32=mixed_flag(args), device=local, autotune=not args.no_tune,
                   shard=(rank, world) if args.shard else None)
    if args.shard:
        # one run, its tuples split over the ranks: every collision sum ends
        # with an NCCL all-reduce (one rank: the same call path)
        if pg is not None:
            from tortoise_b200 import shard
            shard.connect(eng, timeout_s=120.0)
        else:
            eng.shard_connect(E.shard_unique_id(), 120.0)
    nch = len(mat.channels)
    infos = [eng.channel_info(c) for c in range(nch)]
    ntup = sum(i["n_tuples"] for i in infos)
    stream = torch.cuda.ExternalStream(eng.stream_ptr(), device=dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    # ---- collision kernels alone (roofline) -----------------------------
    f = torch.tensor(f0, device=dev)
    acc = torch.zeros_like(f)
    torch.cuda.synchronize()
    for _ in range(3):
        eng.collision_accumulate(f.data_ptr(), acc.data_ptr())
    eng.synchronize()
    reps = 20
    ev0.record(stream)
    for _ in range(reps):
        eng.collision_accumulate(f.data_ptr(), acc.data_ptr())
    ev1.record(stream)
    ev1.synchronize()
    t_coll = ev0.elapsed_time(ev1) * 1e-3 / reps
    bytes_coll = 0
    for c, inf in zip(mat.channels, infos):
        L, n = c.nlegs, inf["n_tuples"]
        bytes_coll += n * moment_bytes(L, inf["layout"])
        bytes_coll += n * 4 * (L + 1)
    bytes_coll += eng.ndofs * 8 * 3   # f read once, accumulator read + written once
    hbm, peak_kind = peaks()
    achieved = bytes_coll / t_coll / 1e9

    # ---- DP45 attempts on the device ------------------------------------
    eng.dp45_begin(f0, 0.0, 1.0e9, DENSE, 0)
    eng.dp45_advance(args.warmup)
    eng.synchronize()
    with ClockSampler(local) as clk:
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize()
        ev0.record(stream)
        eng.dp45_advance(args.steps)
        ev1.record(stream)
        ev1.synchronize()
        torch.cuda.synchronize()
        if pg is not None:
            pg.barrier()
    t_dev = ev0.elapsed_time(ev1) * 1e-3
    st = eng.dp45_poll()
    t_max = reduce_max(pg, t_dev, dev)
    value = args.steps / t_max if args.shard else aggregate_rate(world, args.steps, t_max)
    drift_launch = 1 if any(b.drift_velocity != (0.0, 0.0) for b in mat.bands) else 0
    active = sum(1 for c, i in zip(mat.channels, infos) if c.amplitude != 0 and i["n_tuples"] > 0)
    launches = args.steps * (7 + 6 * (active + drift_launch) + 3)

    # ---- end to end through the C ABI with host buffers ------------------
    # tb_dp45_integrate from host memory to host memory (k1 evaluation, graph
    # launches, polling and the copies of the state and dense output inside).
    t_e2e_final = max(st["t"], 1e-3)
    y = np.ascontiguousarray(f0).copy()
    if pg is not None:
        pg.barrier()
    w0 = time.perf_counter()
    r = eng.dp45(y, 0.0, t_e2e_final, DENSE)
    w1 = time.perf_counter()
    e2e_t = reduce_max(pg, w1 - w0, dev)
    e2e_val = (1 if args.shard else world) * r["attempts"] / e2e_t
    h2d = eng.ndofs * 8 / max(1, r["attempts"])
    d2h = eng.ndofs * 8 * (1 + r["n_dense"]) / max(1, r["attempts"])

    # ---- CPU baseline and oracle parity (oracle on all host cores) ---------
    cpu, parity = None, None
    if rank == 0 and world == 1 and not args.no_cpu:
        import oracle
        o = oracle.Oracle(mat, nthreads=os.cpu_count())
        ref_rhs = cpu_rhs_full(o, f0)[1]   # warm-up: first touch of the tuple arrays, thread start-up
        samples = []
        for _ in range(3):
            t_rhs, ref_rhs = cpu_rhs_full(o, f0)
            samples.append(t_rhs)
        t_att = 6 * statistics.median(samples)
        cpu = {"value": 1.0 / t_att, "unit": "DP45 steps/s", "cores": os.cpu_count(), "kind": "port",
               "sample": "6 x one whole right-hand side (all %d tuples, drift, M^-1), median of 3 after one "
                         "warm-up: %.3f s each"
                         % (ntup, statistics.median(samples))}
        if not args.no_extras and args.mixed is None and not args.shard:
            parity = parity_measure(mat, f0, eng, o, ref_rhs)

    traffic = None
    tp = os.path.join(ROOT, "profiles", "collision_traffic.json")
    if os.path.exists(tp):
        d = json.load(open(tp))
        key = infos[0]["layout"]
        if key in d and d[key].get("bytes_per_tuple"):
            traffic = d[key]["bytes_per_tuple"] * ntup
    line = {"metric": METRIC, "value": value, "unit": "DP45 steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_max / args.steps, "higher_is_better": True,
            "scaling": "strong" if args.shard else "weak", "vs_baseline": None, "dtype": {None: "f64", "t32": "f32-storage/f64-accumulate",
                      "t40": "fp64-upper-40-bit-storage/f64-accumulate",
                      "t48": "fp64-upper-48-bit-storage/f64-accumulate"}[args.mixed],
            "data": "synthetic (seeded PCG64 bump on Fermi-Dirac, Bose phonons)",
            "config": dict(base_config(ntup, nch, eng.ndofs, world),
                           **({"parallelism": "tuple-shard x%d (NCCL all-reduce per RHS)" % world}
                              if args.shard else {})),
            "kernels": {"layouts": [i["layout"] for i in infos],
                        "schedules": [eng.schedule(c) for c in range(nch)],
                        "l2": "moment tensors (%.1f GB) exceed L2; no flush" % (bytes_coll / 1e9)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": traffic,
                         "kernel": "collision contraction, all channels, per RHS evaluation",
                         "algorithmic_bytes": bytes_coll, "seconds_per_launch": t_coll,
                         "peak_source": peak_kind},
            "cpu_baseline": cpu,
            "parity": parity,
            "e2e": {"value": e2e_val, "unit": "DP45 steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "attempts": r["attempts"], "seconds": e2e_t},
            "gpu_launches": launches,
            "dp45": {"t": st["t"], "dt": st["dt"], "attempts": st["attempts"], "rejected": st["rejected"],
                     "status": st["status"]}}
    clk_s = clk.summary()
    if clk_s:
        line["clocks"] = clk_s
    if rank == 0 and world == 1 and not args.no_extras and args.mixed is None and not args.shard:
        # the north-star comparison beside the FP64 headline: mixed-precision
        # storage on this workload, and the batched ensemble against
        # sequential single-run FP64
        line["mixed"] = mixed_measure(eng, mat, f0, args.steps, args.warmup, dev)
        eng.close()
        # 48-bit moments: in the FP64-bound batch they cost what 40-bit ones
        # do, and keep the ensemble at FP64's own run-to-run spread to t = 20
        line["batched"] = batched_measure(256, 10, 3, "t48")
        # the reference's own CPU case (one band, 16x16, four-leg e-e, t = 10)
        line["reference_cpu_case"] = small_ee_measure(args.no_cpu, args.no_tune)
        # the headline's two-band material with its six four-leg e-e
        # channels, streamed, at 16x16 (an extra: the line stands without it)
        try:
            line["ee_streamed"] = ee_streamed_measure(16)
        except Exception as ex:
            line["ee_streamed"] = {"error": str(ex)[:300]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    eng.close()


def fp64_instructions(L):
    """FP64-pipe instructions (an FMA counts once) of one instance-contraction
    of a tuple (contract_run / contract_tuple, tb_tensor.cu): the leg forms (6
    per leg); the gain + loss Kronecker vectors, whose products are shared over
    the leading legs (3^2 + .. + 3^L multiplies each) plus one add per entry;
    the constant-mode sum (3^L FMAs + 2 adds); the first-moment rows (6 FMAs
    per leg and entry of 3^(L-1)); the scaling (4 per leg).  L = 3: 320."""
    K = 3 ** L
    return 6 * L + 2 * sum(3 ** m for m in range(2, L + 1)) + K + (K + 2) + 6 * L * 3 ** (L - 1) + 4 * L


FP64_INSTR = {L: fp64_instructions(L) for L in (2, 3, 4)}

PARITY_T = 0.03          # DP45 span of the trajectory comparison with the oracle
PARITY_DENSE = 0.01


def parity_measure(mat, f0, eng64, o, ref_rhs):
    """The device path against the oracle (all host cores, every tuple) on the
    benchmarked 64x64 workload: one right-hand side with FP64 moments (the
    headline handle) and with 48-bit and 40-bit moments, relative L2 against
    the oracle's; then a DP45 from t = 0 to PARITY_T (dense step
    PARITY_DENSE, the same controller settings) by the oracle and by each
    device arm, compared dense output by dense output.  FP64 moments are held
    to the parity bar of the tests (1e-12 for one right-hand side); the
    reduced-precision storages to their stated bounds."""
    from tortoise_b200 import engine as E
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    out = {"oracle": "C++ restatement on %d host threads, every tuple" % os.cpu_count(),
           "rhs_rel_l2": {}, "rhs_bound": {"t64": 1e-12, "t48": 1e-10, "t40": 1e-8},
           "trajectory": {"t_end": PARITY_T, "dense_step": PARITY_DENSE, "arms": {}}}
    t0 = time.perf_counter()
    ro = o.dp45(f0, 0.0, PARITY_T, PARITY_DENSE)
    out["trajectory"]["oracle_seconds"] = time.perf_counter() - t0
    out["trajectory"]["oracle_attempts"] = [ro["attempts"], ro["accepted"], ro["rejected"]]
    engines = [("t64", eng64, False)]
    for name, flag in (("t48", 3), ("t40", 2)):
        engines.append((name, E.Engine(mat, allow_fp32=flag, autotune=False), True))
    for name, e, own in engines:
        out["rhs_rel_l2"][name] = rel(e.rhs(f0), ref_rhs)
        r = e.dp45(f0, 0.0, PARITY_T, PARITY_DENSE)
        k = min(len(r["dense"]), len(ro["dense"]))
        out["trajectory"]["arms"][name] = {
            "attempts": [r["attempts"], r["accepted"], r["rejected"]],
            "same_steps_as_oracle": [r["attempts"], r["accepted"], r["rejected"]] == out["trajectory"]["oracle_attempts"],
            "dense_rel_l2_max": max(rel(a, b) for a, b in zip(r["dense"][:k], ro["dense"][:k])) if k else None}
        if own:
            e.close()
    out["rhs_within_bound"] = all(out["rhs_rel_l2"][k] < out["rhs_bound"][k] for k in out["rhs_rel_l2"])
    return out


def batched_measure(n_runs, steps, warmup, mixed, layout_name="auto", tune=True):
    """Batched ensemble (ensemble_runs: N in {16..64}, per-run kT and
    couplings): n_runs runs in one handle, DP45 attempts of all runs per
    graph launch; value = run-attempts/s.  Baseline: the same run-attempts on
    the plain single-run FP64 path, one run at a time."""
    import torch
    from tortoise_b200 import engine as E
    from tortoise_b200 import workloads as W
    mats, states = W.ensemble_runs(n_runs)
    layout = {"auto": E.LAYOUT_AUTO, "mc64": E.LAYOUT_MC64, "t64": E.LAYOUT_T64, "t32": E.LAYOUT_T32,
              "t40": E.LAYOUT_T40, "t48": E.LAYOUT_T48}[layout_name]
    t0 = time.perf_counter()
    be = E.BatchEngine(mats, layout=layout, allow_fp32={None: 0, "t32": 1, "t40": 2, "t48": 3}[mixed], autotune=tune)
    t_setup = time.perf_counter() - t0
    f0 = np.concatenate(states)
    stream = torch.cuda.ExternalStream(be.stream_ptr())
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # collision phase alone
    f = torch.tensor(f0, device="cuda")
    acc = torch.zeros_like(f)
    be.collision_accumulate(f.data_ptr(), acc.data_ptr())
    be.synchronize()
    ev0.record(stream)
    for _ in range(5):
        be.collision_accumulate(f.data_ptr(), acc.data_ptr())
    ev1.record(stream)
    ev1.synchronize()
    t_coll = ev0.elapsed_time(ev1) * 1e-3 / 5
    be.dp45_begin(f0, 0.0, 1.0e9, DENSE, 0)
    be.dp45_advance(warmup)
    be.synchronize()
    with ClockSampler(0) as clk:
        ev0.record(stream)
        be.dp45_advance(steps)
        ev1.record(stream)
        ev1.synchronize()
    t = ev0.elapsed_time(ev1) * 1e-3
    Ns = sorted({m.bands[0].mesh.nsplit[0] for m in mats})
    groups = {}
    for m in mats:
        groups[m.bands[0].mesh.nsplit[0]] = groups.get(m.bands[0].mesh.nsplit[0], 0) + 1
    uniq = {}
    for r, m in enumerate(mats):
        N = m.bands[0].mesh.nsplit[0]
        if N not in uniq:
            uniq[N] = sum(be.channel_info(be.chan0[r] + c)["n_tuples"] for c in range(len(m.channels)))
    layouts = sorted({be.channel_info(c)["layout"] for c in range(be.channel_count())})
    # (stages, instance schedule, groups): schedule 0 one instance per thread,
    # 1 instance pairs, 2 / 3 / 4 / 5 run-minor with 32 / 8 / 4 / 16 runs per lane group
    cnt = {}
    for c in range(be.channel_count()):
        sc = be.schedule(c)
        k = (sc["stages"], {32: 2, 8: 3, 4: 4, 16: 5}[sc["runs"]] if sc["runs"] else sc["pair"])
        cnt[k] = cnt.get(k, 0) + 1
    scheds = [[k[0], k[1], v] for k, v in sorted(cnt.items())]
    ndofs = be.ndofs
    # FP64 roofline of the collision: every (tuple, run) pair of a shared
    # group is one contraction of FP64_INSTR[L] FP64-pipe instructions
    run_tuples = {}
    for r, m in enumerate(mats):
        for k, ch in enumerate(m.channels):
            if ch.amplitude != 0:
                L = ch.nlegs
                run_tuples[L] = run_tuples.get(L, 0) + be.channel_info(be.chan0[r] + k)["n_tuples"]
    be.close()
    instr = sum(n * FP64_INSTR[L] for L, n in run_tuples.items())
    fma_rate = E.fp64_fma_rate(0)
    roof64 = {"bound": "fp64", "achieved": instr / t_coll / 1e12, "peak": fma_rate / 1e12,
              "unit": "T FP64-pipe instructions/s", "frac": instr / t_coll / fma_rate,
              "run_tuples": run_tuples, "instructions_per_run_tuple": {L: FP64_INSTR[L] for L in run_tuples},
              "peak_source": "measured in this run: tb_fp64_fma_rate (register-resident DFMA chains on every SM, "
                             "CUDA events)",
              "floor_ms": 1e3 * instr / fma_rate}
    del f, acc
    # The same run-attempts done one run at a time on the plain single-run
    # FP64 path (one handle per structure; runs of equal N cost the same).
    seq = {}
    for N in Ns:
        r = next(i for i, m in enumerate(mats) if m.bands[0].mesh.nsplit[0] == N)
        eng = E.Engine(mats[r], layout=E.LAYOUT_AUTO, allow_fp32=False, autotune=tune)
        s1 = torch.cuda.ExternalStream(eng.stream_ptr())
        eng.dp45_begin(states[r], 0.0, 1.0e9, DENSE, 0)
        eng.dp45_advance(warmup)
        eng.synchronize()
        ev0.record(s1)
        eng.dp45_advance(steps)
        ev1.record(s1)
        ev1.synchronize()
        seq[N] = ev0.elapsed_time(ev1) * 1e-3 / steps
        eng.close()
    t_seq = sum(groups[N] * seq[N] for N in Ns)   # one attempt of every run
    return {"runs": n_runs, "mixed": mixed, "steps": steps,
            "run_attempts_per_s": n_runs * steps / t, "ms_per_attempt": 1e3 * t / steps,
            "collision_ms": 1e3 * t_coll, "setup_s": t_setup, "runs_per_N": groups,
            "tuples_per_structure": uniq, "dofs": ndofs, "layouts": layouts, "schedules": scheds,
            "sequential_fp64_ms_per_attempt_by_N": {N: 1e3 * seq[N] for N in Ns},
            "sequential_fp64_run_attempts_per_s": n_runs / t_seq,
            "speedup_vs_sequential_fp64": (n_runs * steps / t) / (n_runs / t_seq),
            "roofline_fp64": roof64,
            "clocks": clk.summary()}


def batched_to_end(n_runs, tune=True):
    """The ensemble of n_runs runs (ensemble_runs) integrated to t = 20 in one
    handle, every run with its own adaptive steps (dense output every 2):
    with FP64, 40-bit and 48-bit moments; the reduced-precision runs' dense
    outputs are compared with the FP64 runs' run by run.  The single-run FP64 path doing the same
    work one run at a time is projected from its measured time per attempt
    for each mesh size times every run's attempt count (the controllers are
    the same, so a run takes the same attempts alone)."""
    import torch
    from tortoise_b200 import engine as E
    from tortoise_b200 import workloads as W
    mats, states = W.ensemble_runs(n_runs)
    f0 = np.concatenate(states)
    arms, dense, attempts = {}, {}, {}
    # f64_repeat: the FP64 batch once more; its FP64 atomics add in another
    # order, so it measures how far two FP64 runs of the ensemble differ.
    # f64_det / f64_det_repeat: FP64 in the deterministic mode (exact sums),
    # twice: the two must agree bit for bit, and they are the yardstick of
    # the reduced-precision arms that no summation order moves
    for name, flag, det in (("f64", 0, False), ("t40", 2, False), ("t48", 3, False), ("f64_repeat", 0, False),
                            ("f64_det", 0, True), ("f64_det_repeat", 0, True), ("t48_det", 3, True)):
        t0 = time.perf_counter()
        be = E.BatchEngine(mats, allow_fp32=flag, autotune=tune, deterministic=det)
        setup = time.perf_counter() - t0
        be.dp45(f0, 0.0, 0.01, 0.01)   # warm-up: graph capture, first launches
        with ClockSampler(0) as clk:
            w0 = time.perf_counter()
            r = be.dp45(f0, 0.0, T_END, DENSE, max_dense=12)
            w1 = time.perf_counter()
        att = np.array([x["attempts"] for x in r["runs"]])
        arms[name] = {"seconds": w1 - w0, "setup_s": setup, "rc": r["rc"],
                      "all_reached_t_end": bool(all(x["t"] >= T_END for x in r["runs"])),
                      "statuses": sorted({int(x["status"]) for x in r["runs"]}),
                      "run_attempts": int(att.sum()), "attempts_per_run": [int(att.min()), int(np.median(att)),
                                                                          int(att.max())],
                      "run_attempts_per_s": float(att.sum() / (w1 - w0)), "clocks": clk.summary()}
        arms[name]["dense_outputs_per_run"] = [int(min(len(x["dense"]) for x in r["runs"])),
                                               int(max(len(x["dense"]) for x in r["runs"]))]
        print(json.dumps({"arm": name, **{k: arms[name][k] for k in ("seconds", "rc", "statuses",
                                                                     "dense_outputs_per_run")}}),
              file=sys.stderr, flush=True)
        dense[name] = [x["dense"] for x in r["runs"]]
        attempts[name] = att
        if name == "f64":
            attempts_f64 = att
        be.close()
    det_equal = (arms["f64_det"]["rc"] == 0 and arms["f64_det_repeat"]["rc"] == 0
                 and all(len(da) == len(db) > 0 and all(np.array_equal(a, b) for a, b in zip(da, db))
                         for da, db in zip(dense["f64_det"], dense["f64_det_repeat"]))
                 and np.array_equal(attempts["f64_det"], attempts["f64_det_repeat"]))
    for name in ("t40", "t48", "f64_repeat", "f64_det", "t48_det"):
        base = "f64_det" if name == "t48_det" else "f64"
        per_run = [max((float(np.linalg.norm(a - b) / np.linalg.norm(b)) for a, b in zip(da, db)), default=np.inf)
                   for da, db in zip(dense[name], dense[base])]
        if name == "t48_det":
            arms[name]["error_vs"] = "f64_det"
        arms[name]["error_vs_fp64"] = max(per_run)
        arms[name]["error_vs_fp64_median_run"] = float(np.median(per_run))
        arms[name]["runs_above_1e-8"] = int(sum(e > 1e-8 for e in per_run))
        # a run whose controller took another accept / reject path differs
        # from the FP64 run at the integrator's own tolerance (rtol 1e-8),
        # whatever the storage; the runs on the FP64 run's path show the
        # storage error alone
        same = attempts[name] == attempts[base]
        arms[name]["runs_on_another_step_path"] = int((~same).sum())
        arms[name]["error_vs_fp64_same_step_path"] = max([e for e, k in zip(per_run, same) if k], default=0.0)
        arms[name]["error_vs_fp64_other_step_path"] = max([e for e, k in zip(per_run, same) if not k], default=0.0)
        arms[name]["error_metric"] = ("per run: max relative L2 over the dense outputs t = 2 .. 20 vs the %s batch"
                                      % ("deterministic FP64" if base == "f64_det" else "FP64"))
    # single-run FP64 time per attempt, per mesh size
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    seq = {}
    for r, m in enumerate(mats):
        N = m.bands[0].mesh.nsplit[0]
        if N in seq:
            continue
        eng = E.Engine(m, allow_fp32=False, autotune=tune)
        s1 = torch.cuda.ExternalStream(eng.stream_ptr())
        eng.dp45_begin(states[r], 0.0, 1.0e9, DENSE, 0)
        eng.dp45_advance(3)
        eng.synchronize()
        ev0.record(s1)
        eng.dp45_advance(10)
        ev1.record(s1)
        ev1.synchronize()
        seq[N] = ev0.elapsed_time(ev1) * 1e-3 / 10
        eng.close()
    t_seq = sum(int(a) * seq[m.bands[0].mesh.nsplit[0]] for a, m in zip(attempts_f64, mats))
    return {"runs": n_runs, "t_end": T_END, "arms": arms, "deterministic_fp64_repeat_bit_identical": bool(det_equal),
            "sequential_fp64_ms_per_attempt_by_N": {N: 1e3 * v for N, v in sorted(seq.items())},
            "sequential_fp64_projected_seconds": t_seq,
            "speedup_t40_vs_sequential_fp64": t_seq / arms["t40"]["seconds"],
            "speedup_t48_vs_sequential_fp64": t_seq / arms["t48"]["seconds"],
            "speedup_f64_batch_vs_sequential_fp64": t_seq / arms["f64"]["seconds"]}


def batched(args):
    if args.to_end:
        print(json.dumps(dict({"batched_to_end": True}, **batched_to_end(args.batch, not args.no_tune))), flush=True)
        return
    d = batched_measure(args.batch, args.steps, args.warmup, args.mixed, args.layout, not args.no_tune)
    print(json.dumps(dict({"batched": True}, **d)), flush=True)


def mixed_measure(eng64, mat, f0, steps, warmup, dev):
    """The same workload with 40-bit moment storage: collision GB/s, DP45
    attempts/s and the error of its dense outputs against the FP64 path's
    (both integrated to t = 0.2 with dense step 0.05)."""
    import torch
    from tortoise_b200 import engine as E
    eng = E.Engine(mat, layout=E.LAYOUT_AUTO, allow_fp32=2, autotune=True)
    infos = [eng.channel_info(c) for c in range(len(mat.channels))]
    stream = torch.cuda.ExternalStream(eng.stream_ptr(), device=dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f = torch.tensor(f0, device=dev)
    acc = torch.zeros_like(f)
    for _ in range(3):
        eng.collision_accumulate(f.data_ptr(), acc.data_ptr())
    eng.synchronize()
    ev0.record(stream)
    for _ in range(20):
        eng.collision_accumulate(f.data_ptr(), acc.data_ptr())
    ev1.record(stream)
    ev1.synchronize()
    t_coll = ev0.elapsed_time(ev1) * 1e-3 / 20
    bytes_coll = sum(i["n_tuples"] * (moment_bytes(c.nlegs, i["layout"]) + 4 * (c.nlegs + 1))
                     for c, i in zip(mat.channels, infos)) + eng.ndofs * 8 * 3
    eng.dp45_begin(f0, 0.0, 1.0e9, DENSE, 0)
    eng.dp45_advance(warmup)
    eng.synchronize()
    ev0.record(stream)
    eng.dp45_advance(steps)
    ev1.record(stream)
    ev1.synchronize()
    t = ev0.elapsed_time(ev1) * 1e-3
    r40 = eng.dp45(f0, 0.0, 0.2, 0.05)
    r64 = eng64.dp45(f0, 0.0, 0.2, 0.05)
    err = max(float(np.linalg.norm(a - b) / np.linalg.norm(b)) for a, b in zip(r40["dense"], r64["dense"]))
    eng.close()
    hbm, _ = peaks()
    return {"layouts": [i["layout"] for i in infos], "value": steps / t, "unit": "DP45 steps/s",
            "collision_gbs": bytes_coll / t_coll / 1e9, "frac": bytes_coll / t_coll / 1e9 / hbm,
            "seconds_per_launch": t_coll,
            "error_vs_fp64": err, "error_metric": "max relative L2 over the dense outputs at t = 0.05 .. 0.2",
            "dtype": "fp64-upper-40-bit-storage/f64-accumulate"}


def adjoint(args):
    """Gradient of the band-2 (Dirac cone) energy at t = 5 of the 32x32
    two-band e-ph + drift workload with respect to every initial coefficient
    and the channel couplings: forward sweep with a checkpoint every 16
    accepted steps, reverse sweep with per-segment recomputation.  Reports the
    time of both sweeps and central differences (h = 1e-6) of the replayed
    step sequence in args.adjoint seeded directions plus the e-ph coupling."""
    from tortoise_b200 import adjoint as A
    from tortoise_b200 import engine as E
    from tortoise_b200 import workloads as W
    mat = W.two_band_eph_drift(32)
    f0 = W.initial_status(mat, kT=0.1, seed=0).vec
    layout = {"auto": E.LAYOUT_AUTO, "mc64": E.LAYOUT_MC64, "t64": E.LAYOUT_T64, "t32": E.LAYOUT_T32,
              "t40": E.LAYOUT_T40, "t48": E.LAYOUT_T48}[args.layout]
    eng = E.Engine(mat, layout=layout, allow_fp32=mixed_flag(args))
    w = A.observable_weights(mat, 1, "energy")
    amps = np.array([c.amplitude for c in mat.channels])
    tf, tb = [], []
    for _ in range(3):
        eng.synchronize()
        t0 = time.perf_counter()
        fo, st = eng.adjoint_forward(f0, 0.0, 5.0, 0.5, checkpoint_every=16, max_steps=100000)
        t1 = time.perf_counter()
        g, ga, bst = eng.adjoint_backward(w)
        t2 = time.perf_counter()
        tf.append(t1 - t0)
        tb.append(t2 - t1)
    dts, s = eng.adjoint_steps()
    J = lambda f: float(w @ eng.dp45_replay(f, dts, s))
    rng = np.random.default_rng(1234)
    h, errs = 1e-6, []
    for _ in range(args.adjoint):
        d = rng.standard_normal(eng.ndofs)
        fd = (J(f0 + h * d) - J(f0 - h * d)) / (2 * h)
        errs.append(abs(fd - float(g @ d)) / abs(float(g @ d)))
    vals = []
    for sg in (1, -1):
        A.set_amplitudes(eng, amps * (1 + sg * h))
        vals.append(J(f0))
    A.set_amplitudes(eng, amps)
    fd_c, ad_c = (vals[0] - vals[1]) / (2 * h), float(amps @ ga)
    print(json.dumps({"adjoint": True, "workload": "2-band e-ph + drift, 32x32 mesh, t 0 -> 5, dense 0.5",
                      "observable": "energy of band 2 (Dirac cone) at t = 5", "dofs": eng.ndofs,
                      "accepted_steps": bst["steps"], "attempts": bst["attempts"], "checkpoint_every": 16,
                      "checkpoints": bst["checkpoints"], "rhs_evals": bst["rhs_evals"], "vjp_evals": bst["vjp_evals"],
                      "forward_s": min(tf), "backward_s": min(tb), "backward_over_forward": min(tb) / min(tf),
                      "fd_directions": args.adjoint, "fd_max_rel_err": max(errs) if errs else None,
                      "fd_coupling_rel_err": abs(fd_c - ad_c) / abs(ad_c), "layouts": sorted(
                          {eng.channel_info(c)["layout"] for c in range(eng.channel_count())})}), flush=True)
    eng.close()


def adjoint_ee(args):
    """The adjoint configuration with its e-e channels (--adjoint-ee N): the
    two-band e-e + e-ph + drift material on an N x N mesh, e-e streamed,
    gradient of the band-2 energy at t1 (--adjoint-t1, short: every
    right-hand side walks the e-e candidates again) with respect to every
    initial coefficient and the two coupling constants (e-e: the sum over the
    e-e channels' amplitude gradients; e-ph likewise), against central
    differences (h = 1e-6) of the replayed step sequence in a few seeded
    directions and in each coupling."""
    from tortoise_b200 import adjoint as A
    from tortoise_b200 import engine as E
    from tortoise_b200 import workloads as W
    N = args.adjoint_ee
    mat = W.two_band_eph_drift(N, ee=True)
    f0 = W.initial_status(mat, kT=0.1, seed=0).vec
    eng = E.Engine(mat, stream_legs=4, autotune=not args.no_tune)
    w = A.observable_weights(mat, 1, "energy")
    amps = np.array([c.amplitude for c in mat.channels])
    is_ee = np.array([c.nlegs == 4 for c in mat.channels])
    t1 = args.adjoint_t1
    eng.synchronize()
    w0 = time.perf_counter()
    fo, st = eng.adjoint_forward(f0, 0.0, t1, t1 / 2, checkpoint_every=4, max_steps=10000)
    w1 = time.perf_counter()
    g, ga, bst = eng.adjoint_backward(w)
    w2 = time.perf_counter()
    dts, sfrac = eng.adjoint_steps()
    J = lambda f: float(w @ eng.dp45_replay(f, dts, sfrac))
    h = 1e-6
    rng = np.random.default_rng(1234)
    errs = []
    for _ in range(args.adjoint):
        d = rng.standard_normal(eng.ndofs)
        fd = (J(f0 + h * d) - J(f0 - h * d)) / (2 * h)
        errs.append(abs(fd - float(g @ d)) / abs(float(g @ d)))
    coupling = {}
    for name, sel in (("ee", is_ee), ("eph", ~is_ee)):
        vals = []
        for sg in (1, -1):
            A.set_amplitudes(eng, np.where(sel, amps * (1 + sg * h), amps))
            vals.append(J(f0))
        A.set_amplitudes(eng, amps)
        fd_c = (vals[0] - vals[1]) / (2 * h)      # dJ/d(log coupling)
        ad_c = float((amps * ga)[sel].sum())
        coupling[name] = {"adjoint": ad_c, "central_difference": fd_c, "rel_err": abs(fd_c - ad_c) / abs(ad_c)}
    print(json.dumps({"adjoint_ee": True, "workload": "2-band e-e + e-ph + drift, %dx%d mesh, t 0 -> %g, e-e streamed"
                      % (N, N, t1), "observable": "energy of band 2 (Dirac cone) at t1", "dofs": eng.ndofs,
                      "accepted_steps": bst["steps"], "attempts": bst["attempts"], "rhs_evals": bst["rhs_evals"],
                      "vjp_evals": bst["vjp_evals"], "forward_s": w1 - w0, "backward_s": w2 - w1,
                      "fd_directions": args.adjoint, "fd_max_rel_err": max(errs) if errs else None,
                      "coupling_gradients": coupling}), flush=True)
    eng.close()


def ee_streamed_measure(N):
    """One collision evaluation of every channel of the two-band workload
    with its e-e channels on an N x N mesh, the e-e channels streamed (no
    stored list), CUDA events on the library's stream; the walk's counts."""
    import torch
    from tortoise_b200 import engine as E
    from tortoise_b200 import workloads as W
    mat = W.two_band_eph_drift(N, ee=True)
    f0 = W.initial_status(mat, kT=0.1, seed=1).vec
    eng = E.Engine(mat, stream_legs=4)
    try:
        dev = torch.device("cuda", 0)
        stream = torch.cuda.ExternalStream(eng.stream_ptr(), device=dev)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f = torch.tensor(f0, device=dev)
        acc = torch.zeros_like(f)
        ms, surv, cand = [], 0, 0
        ee = [c for c in range(len(mat.channels)) if mat.channels[c].nlegs == 4]
        for c in range(len(mat.channels)):
            torch.cuda.synchronize()
            ev0.record(stream)
            eng.collision_accumulate(f.data_ptr(), acc.data_ptr(), ch=c)
            ev1.record(stream)
            ev1.synchronize()
            ms.append(ev0.elapsed_time(ev1))
            if c in ee:
                i = eng.channel_info(c)
                surv += i["n_tuples"]
                cand += i["n_prefilter"]
        ee_ms = sum(ms[c] for c in ee)
        return {"workload": "2-band e-e + e-ph + drift, %dx%d mesh, e-e streamed" % (N, N),
                "ee_channels": len(ee), "ee_collision_ms_per_rhs": ee_ms,
                "eph_collision_ms_per_rhs": sum(ms) - ee_ms, "ee_surviving_tuples": surv,
                "ee_candidates_in_energy_window": cand, "ee_surviving_tuples_per_s": surv / (1e-3 * ee_ms)}
    finally:
        eng.close()


def small_ee(args):
    """Prints small_ee_measure's line (--ee-mesh: another mesh size)."""
    print(json.dumps(small_ee_measure(args.no_cpu, args.no_tune, args.ee_mesh)), flush=True)


def small_ee_measure(no_cpu=False, no_tune=False, n_mesh=16):
    """The reference's CPU-runnable case: one parabolic band on a 16x16 mesh
    (512 triangles; n_mesh sections per side), electron-electron scattering with a constant matrix
    element, Fermi-Dirac kT 0.1 / mu 0.3 plus the seeded bump, DP45 with
    rtol 1e-6 / atol 1e-9 to t = 10 (dense output every 1.0).  The whole
    integration runs through the C ABI from host buffers (tb_dp45_integrate);
    beside it, the oracle's time for one right-hand side on all host cores,
    measured on a bounded sample of the device's tuple list and scaled to the
    whole list, times the number of right-hand sides the GPU run needed."""
    from tortoise_b200 import engine as E
    from tortoise_b200 import workloads as W
    mat = W.parabolic_ee(n_mesh)
    f0 = W.initial_status(mat, kT=0.1, seed=0).vec
    t_setup = time.perf_counter()
    eng = E.Engine(mat, autotune=not no_tune)
    t_setup = time.perf_counter() - t_setup
    info = eng.channel_info(0)
    # the collision operator alone, CUDA events on the library's stream:
    # the quadrature over the points inside the simplices only (the default)
    # and over every point of every tuple
    import torch
    dev = torch.device("cuda", 0)
    stream = torch.cuda.ExternalStream(eng.stream_ptr(), device=dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    fd = torch.tensor(f0, device=dev)
    acc = torch.zeros_like(fd)
    coll = {}
    for inside in (False, True):
        eng.set_schedule(0, 0, inside_only=inside)
        for _ in range(2):
            eng.collision_accumulate(fd.data_ptr(), acc.data_ptr())
        eng.synchronize()
        reps = 5
        ev0.record(stream)
        for _ in range(reps):
            eng.collision_accumulate(fd.data_ptr(), acc.data_ptr())
        ev1.record(stream)
        ev1.synchronize()
        coll["inside_only" if inside else "every_point"] = ev0.elapsed_time(ev1) / reps
    n_in, p_in = eng.points_inside(0)
    eng.dp45(f0, 0.0, 0.01, 0.01)   # warm-up (graph capture, first launches)
    with ClockSampler(0) as clk:
        w0 = time.perf_counter()
        r = eng.dp45(f0, 0.0, 10.0, 1.0, max_dense=11)
        w1 = time.perf_counter()
    gpu_s = w1 - w0
    line = {"workload": "%dx%d parabolic band, e-e constant matrix element (%d triangles), rtol 1e-6, t = 10"
                        % (n_mesh, n_mesh, 2 * n_mesh * n_mesh),
            "tuples": info["n_tuples"], "layout": info["layout"], "setup_s": t_setup,
            "tuples_with_points_inside": n_in, "points_inside": p_in,
            "points_evaluated_every_point": info["n_tuples"] * mat.channels[0].numMCPoints,
            "collision_ms_per_rhs": coll,
            "gpu": {"seconds": gpu_s, "status": r["status"], "attempts": r["attempts"], "accepted": r["accepted"],
                    "rejected": r["rejected"], "rhs_evals": r["rhs_evals"], "t": r["t"],
                    "attempts_per_s": r["attempts"] / gpu_s}}
    if not no_cpu:
        import oracle   # the CPU baseline of this case
        ids, umk = eng.tuples(0)
        # every tuple up to 1e8 (the 16x16 case has 5.8e7: one whole
        # right-hand side, also the parity reference); beyond, a sample
        m = len(umk) if len(umk) <= 100_000_000 else 200_000
        o = oracle.Oracle(mat, enumerate_tuples=False, nthreads=os.cpu_count())
        o.set_tuples(0, ids[:m], umk[:m])
        o.channel_propagate(0, f0, 0, min(m, 1000))   # warm-up
        samples, ref = [], None
        for _ in range(3 if m < len(umk) else 1):
            a = time.perf_counter()
            ref = o.channel_propagate(0, f0, 0, m)
            samples.append((time.perf_counter() - a) * len(umk) / m)
        t_rhs = statistics.median(samples)
        line["cpu_oracle"] = {"seconds_per_rhs": t_rhs, "cores": os.cpu_count(), "kind": "port",
                              "sample": ("one whole right-hand side (all %d tuples), measured" % len(umk))
                              if m == len(umk) else "first %d of %d tuples, scaled; median of 3" % (m, len(umk)),
                              "projected_seconds": t_rhs * r["rhs_evals"]}
        line["gpu_vs_cpu"] = line["cpu_oracle"]["projected_seconds"] / gpu_s
        if m == len(umk):
            got = eng.rhs(f0, drift=False)
            line["parity"] = {"rhs_rel_l2_vs_oracle": float(np.linalg.norm(got - ref) / np.linalg.norm(ref)),
                              "bound": 1e-12, "layout": info["layout"]}
    c = clk.summary()
    if c:
        line["clocks"] = c
    eng.close()
    return line


def to_end(args):
    """The 64x64 two-band e-ph + drift workload integrated as its
    configuration asks: DP45 at rtol 1e-8 from t = 0 to t = 20, dense output
    every 2, through tb_dp45_integrate from host buffers; with FP64 moments,
    and with 40-bit and 48-bit moments, whose dense outputs are compared with
    the FP64 run's over the whole trajectory.  Beside it, the oracle's
    time for one right-hand side on all host cores (a bounded sample of every
    channel's tuples, scaled) times the right-hand sides the FP64 run took."""
    from tortoise_b200 import engine as E
    mat, f0 = workload()
    line = {"workload": "2-band e-ph + drift, 64x64 mesh (8192 triangles/band), NMC=50, rtol 1e-8, t = 0..20",
            "arms": {}}
    dense_fp64 = None
    for name, flag in (("f64", 0), ("t40", 2), ("t48", 3)):
        t0 = time.perf_counter()
        eng = E.Engine(mat, allow_fp32=flag, autotune=not args.no_tune)
        setup = time.perf_counter() - t0
        eng.dp45(f0, 0.0, 0.01, 0.01)   # warm-up: graph capture, first launches
        with ClockSampler(0) as clk:
            w0 = time.perf_counter()
            r = eng.dp45(f0, 0.0, T_END, DENSE, max_dense=12)
            w1 = time.perf_counter()
        arm = {"seconds": w1 - w0, "setup_s": setup, "status": r["status"], "t": r["t"], "attempts": r["attempts"],
               "accepted": r["accepted"], "rejected": r["rejected"], "rhs_evals": r["rhs_evals"],
               "layouts": [eng.channel_info(c)["layout"] for c in range(len(mat.channels))]}
        c = clk.summary()
        if c:
            arm["clocks"] = c
        if dense_fp64 is None:
            dense_fp64 = r["dense"]
        else:
            k = min(len(dense_fp64), len(r["dense"]))
            arm["error_vs_fp64"] = max(float(np.linalg.norm(a - b) / np.linalg.norm(b))
                                       for a, b in zip(r["dense"][:k], dense_fp64[:k]))
            arm["error_metric"] = "max relative L2 over the dense outputs t = 2, 4, .., 20"
        line["arms"][name] = arm
        eng.close()
    if not args.no_cpu:
        import oracle   # the CPU baseline of this case
        o = oracle.Oracle(mat, nthreads=os.cpu_count())
        t_rhs = statistics.median([cpu_rhs_full(o, f0)[0] for _ in range(3)])
        n_rhs = line["arms"]["f64"]["rhs_evals"]
        line["cpu_oracle"] = {"seconds_per_rhs": t_rhs, "cores": os.cpu_count(), "kind": "port",
                              "sample": "whole right-hand sides (every tuple), median of 3",
                              "projected_seconds": t_rhs * n_rhs}
        line["gpu_vs_cpu"] = line["cpu_oracle"]["projected_seconds"] / line["arms"]["f64"]["seconds"]
    print(json.dumps(line), flush=True)


def large(args):
    """The large batched mixed-precision configuration: 16 runs of the
    three-band (parabola, Dirac cone, heavy hole), two-phonon (0.15, 0.25) e-ph
    material on a 128x128 mesh (32,768 triangles per band), rtol 1e-8, one
    structure shared by all runs, reduced-precision moments (FP32 or 40-bit),
    FP64 products, gain - loss, error norm and step control.  Times args.steps
    DP45 attempts of the whole batch after args.warmup, the collision operator
    alone, and states the error of one right-hand side of run 0 against the
    FP64 Monte-Carlo operator."""
    import torch
    from tortoise_b200 import engine as E
    from tortoise_b200 import workloads as W
    kind = args.large
    mats, states = W.large_batch(16, 128)
    f0 = np.concatenate(states)
    t0 = time.perf_counter()
    be = E.BatchEngine(mats, allow_fp32={"t32": 1, "t40": 2, "t48": 3}[kind], autotune=not args.no_tune)
    setup = time.perf_counter() - t0
    nch = be.channel_count()
    per_run = len(mats[0].channels)
    infos = [be.channel_info(c) for c in range(per_run)]
    ntup = sum(i["n_tuples"] for i in infos)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.ExternalStream(be.stream_ptr(), device=dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f = torch.tensor(f0, device=dev)
    acc = torch.zeros_like(f)
    be.collision_accumulate(f.data_ptr(), acc.data_ptr())
    be.synchronize()
    ev0.record(stream)
    for _ in range(3):
        be.collision_accumulate(f.data_ptr(), acc.data_ptr())
    ev1.record(stream)
    ev1.synchronize()
    t_coll = ev0.elapsed_time(ev1) * 1e-3 / 3
    del f, acc
    be.dp45_begin(f0, 0.0, 20.0, 2.0, 0)
    be.dp45_advance(args.warmup)
    be.synchronize()
    with ClockSampler(0) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        be.dp45_advance(args.steps)
        ev1.record(stream)
        ev1.synchronize()
    t_dev = ev0.elapsed_time(ev1) * 1e-3
    be.dp45_poll()
    st = [be.run_stats(r) for r in range(len(mats))]
    scheds = sorted({(sc["stages"], sc["runs"], sc["pair"]) for sc in (be.schedule(c) for c in range(per_run))
                     if sc["stages"]})
    # one RHS of run 0 against the FP64 Monte-Carlo operator of that run alone
    out = be.split(be.rhs(f0))[0]
    be.close()
    ref = E.Engine(mats[0], layout=E.LAYOUT_MC64).rhs(states[0])
    err = float(np.linalg.norm(out - ref) / np.linalg.norm(ref))
    bytes_mom = ntup * moment_bytes(3, kind)
    line = {"large": True, "workload": "16 runs x three-band two-phonon e-ph, 128x128 mesh (32768 triangles/band), "
                                      "rtol 1e-8, one shared structure", "dtype": kind, "runs": len(mats),
            "tuples": ntup, "channels_per_run": per_run, "dofs": int(f0.size), "setup_s": setup,
            "steps": args.steps, "warmup": args.warmup, "ms_per_attempt": 1e3 * t_dev / args.steps,
            "run_attempts_per_s": len(mats) * args.steps / t_dev,
            "collision_ms": 1e3 * t_coll, "moment_gb": bytes_mom / 1e9,
            "run_tuples_per_s": ntup * len(mats) / t_coll,
            "rhs_error_vs_fp64_mc": err,
            "schedules": scheds,
            "attempts": [s["attempts"] for s in st], "t": [s["t"] for s in st]}
    c = clk.summary()
    if c:
        line["clocks"] = c
    print(json.dumps(line), flush=True)


def ee_full(args):
    """The two-band configuration as written, e-e included: parabola + Dirac
    cone, the four-leg e-e channels (constant matrix element 1.0) and the
    e-ph channels of the optical branch (hw = 0.2, Bose kT = 0.05), drift
    field (0.1, 0), rtol 1e-8, on an N x N mesh (--ee-full N).  The e-e
    channels are streamed (their tuple lists do not fit in device memory at
    N >= 32: about 2e9 tuples per channel at 32x32, 3e10 at 64x64); the e-ph
    channels keep their moment tensors.  Times one collision evaluation of
    every channel (CUDA events on the library's stream), reports the walk's
    counts per e-e channel, then times args.steps DP45 attempts from t = 0
    after args.warmup untimed ones."""
    import torch
    from tortoise_b200 import engine as E
    from tortoise_b200 import workloads as W
    N = args.ee_full
    mat = W.two_band_eph_drift(N, ee=True)
    f0 = W.initial_status(mat, kT=0.1, seed=1).vec
    t0 = time.perf_counter()
    eng = E.Engine(mat, stream_legs=4, autotune=not args.no_tune)
    setup = time.perf_counter() - t0
    nch = len(mat.channels)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.ExternalStream(eng.stream_ptr(), device=dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f = torch.tensor(f0, device=dev)
    acc = torch.zeros_like(f)
    per_channel, infos, inside = [], [], []
    for c in range(nch):
        if args.ee_attempt_only and mat.channels[c].nlegs == 4:
            per_channel.append(0.0)   # not evaluated alone
            infos.append(eng.channel_info(c))
            inside.append((0, 0))
            continue
        # one channel alone (its streamed walk records its counts)
        torch.cuda.synchronize()
        ev0.record(stream)
        eng.collision_accumulate(f.data_ptr(), acc.data_ptr(), ch=c)
        ev1.record(stream)
        ev1.synchronize()
        per_channel.append(ev0.elapsed_time(ev1))
        infos.append(eng.channel_info(c))
        inside.append(eng.points_inside(c))
    t_rhs_host = None
    if not args.ee_once:
        w0 = time.perf_counter()
        eng.rhs(f0)   # one whole right-hand side from host buffers
        t_rhs_host = time.perf_counter() - w0
    ee_idx = [c for c in range(nch) if mat.channels[c].nlegs == 4]
    line = {"ee_full": True, "workload": "2-band e-e + e-ph + drift, %dx%d mesh (%d triangles/band), NMC=50, "
                                         "rtol 1e-8" % (N, N, 2 * N * N),
            "setup_s": setup, "channels": nch, "dofs": eng.ndofs,
            "layouts": [i["layout"] for i in infos],
            "ee_channels": {"count": len(ee_idx),
                            "candidates_in_energy_window": sum(infos[c]["n_prefilter"] for c in ee_idx),
                            "with_valid_determinant": sum(infos[c]["n_det"] for c in ee_idx),
                            "surviving_tuples": sum(infos[c]["n_tuples"] for c in ee_idx),
                            "tuples_with_points_inside": sum(inside[c][0] for c in ee_idx),
                            "points_inside": sum(inside[c][1] for c in ee_idx)},
            "collision_ms_per_channel": per_channel,
            "collision_ms_per_rhs": sum(per_channel), "collision_ms_ee": sum(per_channel[c] for c in ee_idx),
            "collision_ms_eph": sum(per_channel[c] for c in range(nch) if c not in ee_idx),
            "rhs_host_seconds": t_rhs_host}
    if args.ee_attempt_only:
        # the e-e channels were not evaluated alone: no counts, no per-channel times
        line["ee_channels"] = {"count": len(ee_idx)}
        for k in ("collision_ms_per_channel", "collision_ms_per_rhs", "collision_ms_ee"):
            line[k] = None
    elif line["collision_ms_ee"] > 0:
        line["ee_surviving_tuples_per_s"] = line["ee_channels"]["surviving_tuples"] / (1e-3 * line["collision_ms_ee"])
    if args.steps > 0:
        # the collision figures first: a long attempt that does not finish
        # leaves them behind
        print(json.dumps(dict(line, partial=True)), flush=True)
        wb = time.perf_counter()
        eng.dp45_begin(f0, 0.0, T_END, DENSE, 0)   # the first right-hand side and the graph capture
        eng.dp45_advance(args.warmup)
        eng.synchronize()
        line["begin_and_warmup_seconds"] = time.perf_counter() - wb
        with ClockSampler(0) as clk:
            ev0.record(stream)
            eng.dp45_advance(args.steps)
            ev1.record(stream)
            ev1.synchronize()
        st = eng.dp45_poll()
        line["dp45"] = {"attempts_timed": args.steps, "warmup": args.warmup,
                        "seconds_per_attempt": ev0.elapsed_time(ev1) * 1e-3 / args.steps,
                        "attempts_per_s": args.steps / (ev0.elapsed_time(ev1) * 1e-3),
                        "t": st["t"], "attempts": st["attempts"], "rejected": st["rejected"], "status": st["status"]}
        c = clk.summary()
        if c:
            line["clocks"] = c
    print(json.dumps(line), flush=True)
    eng.close()


def rhs_only(args):
    """Profiling driver: K right-hand-side evaluations (collision + drift +
    M^-1) of the workload on the device, nothing else (used for the ncu
    launch list and kernel captures summarised under profiles/)."""
    import torch
    from tortoise_b200 import engine as E
    from tortoise_b200 import workloads as W
    layout = {"auto": E.LAYOUT_AUTO, "mc64": E.LAYOUT_MC64, "t64": E.LAYOUT_T64, "t32": E.LAYOUT_T32,
              "t40": E.LAYOUT_T40, "t48": E.LAYOUT_T48}[args.layout]
    if args.ee:
        # one parabolic band with the four-leg e-e channel (Monte-Carlo
        # quadrature over the points inside the simplices)
        mat = W.parabolic_ee(args.mesh)
        f0 = W.initial_status(mat, kT=0.1, seed=0).vec
        eng = E.Engine(mat, layout=layout, autotune=not args.no_tune, stream_legs=args.stream_legs)
    elif args.batch:
        # a batch of args.batch runs of one structure (mesh args.mesh): the
        # groups shared by many runs (run-minor contraction)
        mats, states = W.ensemble_runs(args.batch, seed=3, Ns=(args.mesh,))
        eng = E.BatchEngine(mats, layout=layout, allow_fp32=mixed_flag(args), autotune=not args.no_tune)
        mat, f0 = mats[0], np.concatenate(states)
    else:
        mat, f0 = workload(args.mesh)
        eng = E.Engine(mat, layout=layout, allow_fp32=mixed_flag(args), autotune=not args.no_tune)
    f = torch.tensor(f0, device="cuda")
    out = torch.zeros_like(f)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.rhs_only):
        eng.rhs_device(f.data_ptr(), out.data_ptr())
    eng.synchronize()
    dt = time.perf_counter() - t0
    print(json.dumps({"rhs_only": args.rhs_only, "mesh": args.mesh, "runs": args.batch or 1,
                      "layouts": [eng.channel_info(c)["layout"] for c in range(len(mat.channels))],
                      "schedules": [eng.schedule(c) for c in range(len(mat.channels))], "seconds": dt}), flush=True)
    eng.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--layout", default="auto", choices=["auto", "mc64", "t64", "t32", "t40", "t48"])
    ap.add_argument("--mixed", nargs="?", const="t40", default=None, choices=["t32", "t40", "t48"],
                    help="reduced-precision moment storage: t40 (upper 40 bits of FP64, default), t48 (upper 48 "
                         "bits) or t32 (FP32)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the mixed-precision and batched measurements")
    ap.add_argument("--no-tune", action="store_true", help="fixed contraction schedule (no autotuner)")
    ap.add_argument("--rhs-only", type=int, default=0,
                    help="profiling driver: K RHS evaluations only (with --batch R: R runs of mesh --mesh)")
    ap.add_argument("--mesh", type=int, default=N_MESH, help="sections per side (profiling driver only)")
    ap.add_argument("--stream-legs", type=int, default=0,
                    help="profiling driver (--ee): stream the channels with at least this many legs")
    ap.add_argument("--ee", action="store_true",
                    help="profiling driver on the one-band e-e workload (parabolic band, --mesh sections per side)")
    ap.add_argument("--batch", type=int, default=0, help="batched ensemble of this many runs (per-run N, kT, couplings)")
    ap.add_argument("--large", nargs="?", const="t32", default=None, choices=["t32", "t40", "t48"],
                    help="16-run 128x128 three-band two-phonon batch with FP32 (default) or 40-bit moments")
    ap.add_argument("--to-end", action="store_true",
                    help="the 64x64 workload integrated to t = 20 (FP64 and 40-bit moments) vs the oracle")
    ap.add_argument("--small-ee", action="store_true",
                    help="16x16 one-band e-e integration to t = 10 (the reference's CPU-runnable case) vs the oracle")
    ap.add_argument("--ee-mesh", type=int, default=16, help="sections per side of the --small-ee workload")
    ap.add_argument("--shard", action="store_true",
                    help="one run with its tuples split over the ranks (NCCL all-reduce per RHS) instead of replicas")
    ap.add_argument("--ee-full", type=int, default=0,
                    help="the two-band workload with its e-e channels (streamed) on an N x N mesh: collision time "
                         "per RHS and --steps DP45 attempts")
    ap.add_argument("--ee-once", action="store_true",
                    help="--ee-full: one collision evaluation per channel only, no whole RHS from host buffers")
    ap.add_argument("--ee-attempt-only", action="store_true",
                    help="--ee-full: skip the per-channel evaluation of the e-e channels (time the DP45 attempts only)")
    ap.add_argument("--adjoint-ee", type=int, default=0,
                    help="adjoint of the two-band workload with its e-e channels (streamed) on an N x N mesh")
    ap.add_argument("--adjoint-t1", type=float, default=0.02, help="end time of --adjoint-ee")
    ap.add_argument("--adjoint", type=int, default=-1,
                    help="adjoint gradient of the 32x32 workload, checked in this many FD directions")
    args = ap.parse_args()
    if args.large:
        large(args)
        return
    if args.ee_full:
        ee_full(args)
        return
    if args.adjoint_ee:
        if args.adjoint < 0:
            args.adjoint = 4
        adjoint_ee(args)
        return
    if args.to_end and not args.batch:
        to_end(args)
        return
    if args.small_ee:
        small_ee(args)
        return
    if args.adjoint >= 0:
        adjoint(args)
        return
    if args.rhs_only:
        rhs_only(args)
        return
    if args.batch:
        batched(args)
        return
    world, rank, local, pg = dist_setup(args)
    try:
        if args.impl == "reference":
            reference_arm(args, world, rank)
        else:
            ours(args, world, rank, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
