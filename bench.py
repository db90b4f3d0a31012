#!/usr/bin/env python
"""Throughput of the HARM-COOL step_ch() path on B200, in zone-cycles/s.

One step = one full predictor + corrector update of every active zone of the
288x256x256 (r, theta, phi) Fishbone-Moncrief torus (a=0.9375, rin=6,
rmax=12, beta=100, gamma-law 4/3, FP64), state resident on the GPU.  The
torus comes from the library's own init (seeded, synthetic: no dataset).
The state (6 GB of FP64 planes) is far larger than the 126 MB L2, so no
flush is needed between steps.

--impl ours       the CUDA path (default)
--impl reference  the reference's own step_ch(), compiled from its C sources
                  (oracle/_ref/c2s: the same r-theta grid with 4 phi planes),
                  one process per host core, timed on the host

With --gpus N (torchrun) every rank advances its own torus (replicas: the
reference's MPI slab split is replaced by one domain per GPU, so there is no
data-path collective); the timed region is bracketed by barriers and the
slowest rank's device time is reported.
"""
import argparse
import json
import os
import shutil
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)



def kernels_per_step(n3):
    """Kernel launches of one step: per half step one flux kernel per direction,
    the corner EMFs, the conserved update and the inversion, bound_prim, the flag
    flip, the two repair kernels (list and wavefront), bound_prim; the corrector
    adds the flux diagnostics; then the mass diagnostics and the dt update."""
    nflux = 3 if n3 > 1 else 2
    return 2 * (nflux + 8) + 1 + 2
METRIC = "zone-cycles/s 288x256x256 GRMHD step_ch: FP64, mixed precision beside it"
STATE_BYTES_PER_ZONE_CYCLE = 320  # p read twice, ph written and read, p written; 8 FP64 prims


def dist_setup(backend="nccl"):
    """One process per GPU (torchrun's RANK/LOCAL_RANK/WORLD_SIZE); the process
    group only carries the barriers and the max of the device times."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=60))
    return world, rank, local


def reduce_max(x, world, local):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda:%d" % local if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.path = None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                      "--format=csv,noheader,nounits", "-lms", "100"],
                                     stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        self.proc.wait()
        rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        os.unlink(self.path)
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax = max(smax, float(r[2]))
                for n, v in zip(names, r[5:9]):
                    if v.strip() == "Active":
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": smax or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def reference_cpu_rate(seconds_per_core=20.0, cores=None, min_steps=1):
    """The reference's step_ch() on the 288x256x4 sample, one process per core:
    the -O3 timing build of the reference's own sources (oracle/_ref/c2s/
    refbench_o3), else the -O2 parity build.  The reference's MPI slab split
    would add halo exchanges; no MPI exists on the benchmark host, so each
    process advances its own 4-plane sample (generous to the CPU).

    Returns (zone-cycles/s summed over processes, cores used, sample text)."""
    exe = os.path.join(ROOT, "oracle", "_ref", "c2s", "refbench_o3")
    build = "-O3"
    if not os.path.exists(exe):
        exe = os.path.join(ROOT, "oracle", "_ref", "c2s", "refbench")
        build = "-O2 -ffp-contract=off"
    if not os.path.exists(exe):
        raise RuntimeError("reference checker build oracle/_ref/c2s is missing")
    cores = cores or os.cpu_count() or 1
    # one step of 288x256x4 is about 1 s per core; size the run to the time budget
    steps = max(min_steps, int(seconds_per_core))
    procs = [subprocess.Popen([exe, "1", str(steps)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                              cwd=os.path.dirname(exe)) for _ in range(cores)]
    rates = []
    for p in procs:
        out, _ = p.communicate()
        rates.append(json.loads(out.decode().strip().splitlines()[-1])["zone_cycles_per_s"])
    sample = ("reference step_ch() built %s on 288x256x4 (same r-theta grid, 4 phi planes), "
              "%d step(s) after 1 warm-up, %d independent process(es); the 288x256x256 rate is this "
              "rate, ms_per_step extrapolated from it" % (build, steps, cores))
    return sum(rates), cores, sample


def run_reference(args, world, rank):
    if rank != 0:
        return
    rate, cores, sample = reference_cpu_rate(seconds_per_core=max(2.0, min(20.0, 4.0 * args.steps)))
    line = {"metric": METRIC, "value": rate,
            "unit": "zone-cycles/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * args.n1 * args.n2 * args.n3 / rate, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": workload(args), "parallelism": "single",
                       "sample": "the same r-theta grid with 4 phi planes per process; ms_per_step is the "
                                 "288x256x256 step time extrapolated from the summed 4-plane rate"},
            "ms_per_step_extrapolated": True,
            "cpu_baseline": {"value": rate, "unit": "zone-cycles/s", "cores": cores, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": rate, "unit": "zone-cycles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def workload(args):
    return ("FM torus %dx%dx%d (a=0.9375, rin=6, rmax=12, beta=100), gamma-law, FP64"
            % (args.n1, args.n2, args.n3))


def alg_bytes_per_zone(kernel, n3):
    """Algorithmic DRAM bytes per zone of one launch group, FP64 state (8 B per
    primitive, 8 primitives), averaged over the predictor and the corrector:
    flux   per direction: read the zone's primitives, write its face flux;
    update k_cons reads pi (and pb in the corrector, where it differs from pi)
           and the zone's face flux in each direction (each face is shared by
           two zones) and writes U; k_invert reads U and pi and writes pf and
           pflag."""
    ndir = 3 if n3 > 1 else 2
    if kernel == "flux":
        return ndir * (64 + 64)
    pred = (64 + ndir * 64 + 64) + (64 + 64 + 64 + 1)
    corr = pred + 64
    return (pred + corr) / 2.0


def measured_traffic(kernel, zones):
    """DRAM bytes per launch group from the committed ncu capture, scaled by zones."""
    path = os.path.join(ROOT, "profiles", "dram_traffic_per_zone.json")
    if not os.path.exists(path):
        return None
    d = json.load(open(path))
    if kernel not in d:
        return None
    return d[kernel]["bytes_per_zone"] * zones


def fp64_counts():
    """FP64 pipe instructions per zone of each launch group (flux, update) and per
    zone-cycle, from the committed ncu capture of the step kernels."""
    path = os.path.join(ROOT, "profiles", "fp64_inst_per_zone.json")
    if not os.path.exists(path):
        return None
    return json.load(open(path))


def fp64_roofline(hc, local, kms, zones, dom, ms_step):
    """The FP64-pipe roofline of the dominant launch group and of the whole step:
    FP64 thread instructions (DADD, DMUL, DFMA; the step is built without FMA
    contraction, so its arithmetic issues as separate DADD and DMUL) per second
    against the device's measured FP64 instruction rate, and the step's
    zone-cycles/s ceiling at that rate."""
    counts = fp64_counts()
    peaks = hc.fp64_peak(local)
    peak = min(peaks["dfma_inst_per_s"], peaks["dadd_inst_per_s"], peaks["dmul_inst_per_s"])
    out = {"peak_inst_per_s": peak, "peak_dfma_flop_per_s": 2 * peaks["dfma_inst_per_s"],
           "measured_rates": peaks, "peak_source": "measured live (harm_fp64_peak)"}
    if counts is None:
        return out
    g = counts["groups"][dom]
    inst = g["fp64_inst_per_zone"] * zones
    flop = g["fp64_flop_per_zone"] * zones
    t = kms[dom] / 1e3
    per_cycle = counts["step"]["fp64_inst_per_zone_cycle"]
    out.update({"kernel": dom, "achieved_inst_per_s": inst / t, "fp64_frac": inst / t / peak,
                "achieved_flop_per_s": flop / t,
                "step_frac": per_cycle * zones / (ms_step / 1e3) / peak,
                "fp64_inst_per_zone_cycle": per_cycle,
                "fp64_ceiling_zcps": peak / per_cycle,
                "counts_source": counts["source"]})
    return out


def l1_errors(pa, pb):
    """L1 of (pb - pa) over the active zones relative to the L1 of pa: for rho and
    u, and for the velocity (u1..u3) and field (B1..B3) vectors as wholes, since a
    single component (u2, B3) can be near zero in the whole torus early on."""
    import numpy as np
    groups = {"rho": [0], "u": [1], "v": [2, 3, 4], "B": [5, 6, 7]}
    out = {}
    for n, ks in groups.items():
        s = float(np.sum(np.abs(pa[..., ks])))
        out[n] = float(np.sum(np.abs(pb[..., ks] - pa[..., ks])) / s) if s > 0 else 0.0
    return out


def timed_run(hc, pr, local, world, steps, warmup, mixed):
    ctx = hc.Context(pr, device=local)
    ctx.init_torus()
    if mixed:
        ctx.set_precision(hc.Context.MIXED)
    ctx.run(warmup)
    sampler = ClockSampler(local)
    barrier(world)
    sampler.start()
    ms = ctx.run_timed(steps)
    clocks = sampler.stop()
    barrier(world)
    return ctx, reduce_max(ms, world, local), clocks


def mixed_l1_leg(hc, pr, local, nsteps, act):
    """The mixed path's accuracy contract on the benchmark torus: both paths
    advance nsteps from the same initial state; L1 of the mixed state against
    the FP64 state, with the device time of each run (dt ramp included)."""
    out = {}
    states = {}
    for name, mixed in (("fp64", False), ("mixed", True)):
        c = hc.Context(pr, device=local)
        c.init_torus()
        if mixed:
            c.set_precision(hc.Context.MIXED)
        ms = c.run_timed(nsteps)
        states[name] = c.get_prims()[act]
        out["ms_per_step_%s_%d_steps" % (name, nsteps)] = ms / nsteps
        out["fail_code_%s_%d_steps" % (name, nsteps)] = c.diag()["fail_code"]
        c.close()
    out["l1_vs_fp64"] = l1_errors(states["fp64"], states["mixed"])
    out["l1_after_steps"] = nsteps
    out["l1_bound_rho"] = 1e-4
    return out


def run_ours(args, world, rank, local):
    import numpy as np
    import harm_cool_b200 as hc
    pr = hc.torus_problem(args.n1, args.n2, args.n3)
    zones = pr.zones
    ctx, ms, clocks = timed_run(hc, pr, local, world, args.steps, args.warmup, mixed=False)
    value = zones * args.steps * world / (ms / 1e3)
    # the state after warmup + steps, for the mixed run's L1 at the same step
    pa = ctx.get_prims() if not args.no_mixed else None
    d = ctx.diag()
    # end to end through the host-array call: upload p, step, download p every step
    import torch
    pinned = torch.empty(pr.shape + (8,), dtype=torch.float64, pin_memory=True).numpy()
    pinned[...] = ctx.get_prims()
    ms_e2e = ctx.step_ch_host_timed(pinned, args.e2e_steps)
    ms_e2e = reduce_max(ms_e2e, world, local)
    e2e = zones * args.e2e_steps * world / (ms_e2e / 1e3)
    bytes_host = int(np.prod(pr.shape)) * 8 * 8
    del pinned
    # dominant kernel, timed launch by launch inside ordinary steps on the context's stream
    kms = ctx.time_kernels(reps=3)
    dom = max(("flux", "update"), key=lambda k: kms[k])
    peak, peak_kind = measured_peaks()
    alg = alg_bytes_per_zone(dom, args.n3) * zones
    achieved = alg / (kms[dom] / 1e3) / 1e9
    traffic = measured_traffic(dom, zones)
    line = {"metric": METRIC,
            "value": value, "unit": "zone-cycles/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload(args),
                       "parallelism": "replicas" if world > 1 else "single",
                       "l2": "state (%.1f GB) > L2, no flush" % (zones * 64 * 2 / 1e9)},
            "e2e": {"value": e2e, "unit": "zone-cycles/s", "h2d_bytes_per_step": bytes_host,
                    "d2h_bytes_per_step": bytes_host, "steps": args.e2e_steps,
                    "path": "harm_run_host: per step upload, step, download, each upload overlapped with the "
                            "previous step's download"},
            "gpu_launches": kernels_per_step(args.n3) * args.steps,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "algorithmic_bytes": alg, "peak_source": peak_kind,
                         "step_frac": zones * STATE_BYTES_PER_ZONE_CYCLE / (ms / args.steps / 1e3) / 1e9 / peak},
            "kernel_ms": kms, "clocks": clocks, "sim_time": ctx.time(), "fail_code": d["fail_code"]}
    line["roofline"]["fp64"] = f64 = fp64_roofline(hc, local, kms, zones, dom, ms / args.steps)
    # the roofline that binds this FP64 path: the FP64 pipe (HBM is far from busy)
    line["roofline"]["fp64_frac"] = f64.get("fp64_frac")
    line["roofline"]["fp64_ceiling_zcps"] = f64.get("fp64_ceiling_zcps")
    act = (slice(1, -1) if args.n3 > 1 else slice(None), slice(2, -2), slice(2, -2))
    if not args.no_mixed:
        ctx.close()
        ctxm, msm, clocksm = timed_run(hc, pr, local, world, args.steps, args.warmup, mixed=True)
        pb = ctxm.get_prims()
        line["mixed"] = {"value": zones * args.steps * world / (msm / 1e3), "ms_per_step": msm / args.steps,
                         "speedup_vs_fp64": ms / msm, "clocks": clocksm,
                         "l1_vs_fp64_timed_run": l1_errors(pa[act], pb[act]),
                         "timed_run_steps": args.warmup + args.steps,
                         "kernel_ms": ctxm.time_kernels(reps=3), "fail_code": ctxm.diag()["fail_code"]}
        ctxm.close()
        del pa, pb
        if args.l1_steps > 0:
            line["mixed"].update(mixed_l1_leg(hc, pr, local, args.l1_steps, act))
    else:
        ctx.close()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, cores, sample = reference_cpu_rate(seconds_per_core=10.0, cores=1)
        line["cpu_baseline"] = {"value": rate, "unit": "zone-cycles/s", "cores": cores, "kind": "reference",
                                "sample": sample}
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_ensemble(args):
    """64 seeded 2D tori (N1, N2 from {96,128,192,256}, a, Rmax, beta drawn) advanced
    as one ensemble -- one CUDA graph launch per step, mixed precision, tiles chosen
    by the autotuner per resolution -- against the same 64 tori run one after the
    other on the plain FP64 path.  Aggregate zone-cycles/s over all members.  Some
    draws fail the inversion in most zones every step and run far slower than the
    rest; the same comparison is also reported without them."""
    import harm_cool_b200 as hc
    drawn = hc.ensemble_problems(args.members, seed=args.seed)
    probs = [p for p, _ in drawn]
    # sequential plain runs: each torus alone, FP64, default tile
    solo_ms = []
    for pr in probs:
        c = hc.Context(pr)
        c.init_torus()
        c.run(args.warmup)
        solo_ms.append(c.run_timed(args.steps) / args.steps)
        c.close()
    med = sorted(solo_ms)[len(solo_ms) // 2]
    heavy = [k for k, m in enumerate(solo_ms) if m > 20 * med]
    subsets = {"all": list(range(len(probs))), "without_failure_heavy": [k for k in range(len(probs)) if k not in heavy]}

    def ensemble(members, mixed):
        ctxs, tiles = [], {}
        for k in members:
            pr = probs[k]
            c = hc.Context(pr)
            c.init_torus()
            if mixed:
                c.set_precision(hc.Context.MIXED)
            key = (pr.params.n1, pr.params.n2)
            if key not in tiles:
                tiles[key] = c.autotune_tile(steps=3)
            c.set_tile(*tiles[key])
            ctxs.append(c)
        ens = hc.Ensemble(ctxs)
        ens.run(args.warmup)
        sampler = ClockSampler(0)
        sampler.start()
        ms = ens.run_timed(args.steps) / args.steps
        clocks = sampler.stop()
        fails = sorted({c.diag()["fail_code"] for c in ctxs})
        ens.close()
        for c in ctxs:
            c.close()
        zones = sum(probs[k].zones for k in members)
        return {"value": zones / (ms / 1e3), "ms_per_step": ms, "zones": zones,
                "tiles": {"%dx%d" % k: list(v) for k, v in tiles.items()}, "clocks": clocks, "fail_codes": fails}

    out = {}
    for name, members in subsets.items():
        zones = sum(probs[k].zones for k in members)
        seq_ms = sum(solo_ms[k] for k in members)
        r = {"members": len(members), "zones": zones,
             "sequential_fp64": {"value": zones / (seq_ms / 1e3), "ms_per_step": seq_ms},
             "ensemble_mixed": ensemble(members, True)}
        if name == "all":
            r["ensemble_fp64"] = ensemble(members, False)
        r["speedup_vs_sequential"] = r["ensemble_mixed"]["value"] / r["sequential_fp64"]["value"]
        out[name] = r
    line = {"metric": "aggregate zone-cycles/s, %d seeded 2D tori" % args.members,
            "value": out["all"]["ensemble_mixed"]["value"], "unit": "zone-cycles/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "dtype": "f64/f32 mixed",
            "data": "synthetic", "config": {"workload": "ensemble of %d 2D tori, N1,N2 in {96,128,192,256}, "
                                                        "a in [0,0.98], Rmax in [9,14], beta in [30,300], seed %d"
                                                        % (args.members, args.seed)},
            "failure_heavy_members": heavy, "solo_ms_per_step": solo_ms,
            "members": [d for _, d in drawn], **out}
    print(json.dumps(line), flush=True)


def run_adjoint(args):
    """The discrete adjoint on a 2D gamma-law torus (192x192, K = 50 steps,
    checkpoint every 10): J = the mass that crosses the inner boundary over the K
    steps (mass_in, diag.c:578), dJ/d(rmax, beta, A_1..A_16) -- A the amplitudes
    of 16 seeded density modes -- through one adjoint sweep, against central
    differences of the step (h = 1e-9, which resolves the branches the step takes;
    h = 1e-6 straddles the density floor that the atmosphere sits within ~1e-7
    of).  Cost: the adjoint's device time (forward with checkpoints, reverse sweep
    with its recomputation) over the plain forward's (graph replay of K steps)."""
    import numpy as np
    import harm_cool_b200 as hc
    from harm_cool_b200 import adjoint as ad
    n, K, every = args.adj_n, args.adj_steps, args.adj_every
    ctx = hc.Context(hc.torus_problem(n, n, 1))
    modes = ad.Modes(n, n, m=16, seed=args.seed)
    amps = np.zeros(16)
    theta = np.concatenate([[12.0, 100.0], amps])
    sampler = ClockSampler(0)
    sampler.start()
    fwd = []
    for r in range(args.warmup + 5):
        ad.initial_state(ctx, modes, 12.0, 100.0, amps)
        fwd.append(ctx.run_timed(K))
    fwd_ms = sorted(fwd[args.warmup:])[2]
    runs = []
    for r in range(args.warmup + 5):
        ad.initial_state(ctx, modes, 12.0, 100.0, amps)
        J, lam, ms = ctx.adjoint_mass_in(K, every)
        runs.append(ms)
    clocks = sampler.stop()
    runs = sorted(runs[args.warmup:], key=lambda m: m[0] + m[1])
    ms = runs[2]
    J, g, info = ad.mass_in_gradient(ctx, modes, 12.0, 100.0, amps, K, every, rel_step=1e-9)
    fd = {}
    for hr in (1e-9, 1e-6):
        d = np.zeros(len(theta))
        for k in range(len(theta)):
            h = hr * max(abs(theta[k]), 1.0)
            tp, tm = theta.copy(), theta.copy()
            tp[k] += h
            tm[k] -= h
            d[k] = (ad.mass_in(ctx, modes, tp[0], tp[1], tp[2:], K) - ad.mass_in(ctx, modes, tm[0], tm[1], tm[2:], K)) / (2 * h)
        fd[hr] = d
    scale = float(np.abs(fd[1e-9]).max())
    err = {("h=%g" % hr): float(np.abs(g - d).max() / scale) for hr, d in fd.items()}
    line = {"metric": "adjoint / forward device time, 2D %dx%d torus, K=%d" % (n, n, K), "value": (ms[0] + ms[1]) / fwd_ms,
            "unit": "x", "n_gpus": 1, "steps": K, "warmup": args.warmup, "higher_is_better": False, "dtype": "f64",
            "data": "synthetic", "config": {"workload": "adjoint of %d steps of the 2D gamma-law step, %dx%d torus "
                                                        "a=0.9375 rin=6 rmax=12 beta=100, checkpoint every %d, 16 density "
                                                        "modes seed %d" % (K, n, n, every, args.seed)},
            "forward_ms": fwd_ms, "adjoint_ms": {"forward_with_checkpoints": ms[0], "reverse_sweep": ms[1]},
            "J": J, "parameters": ["rmax", "beta"] + ["A%d" % (m + 1) for m in range(16)],
            "gradient": g.tolist(), "central_difference": {("h=%g" % hr): d.tolist() for hr, d in fd.items()},
            "max_abs_error_over_max_gradient": err, "clocks": clocks}
    print(json.dumps(line), flush=True)


def tracers_by_density(np, pr, p, n, seed):
    """n tracer particles at zone centres drawn with probability proportional to
    the zone's rest mass rho sqrt(-g) dV (seeded); labels (i, j, h) of the zone."""
    g = pr.geometry["gdet"][:, :, 3]
    sn1, sn2 = g.shape
    rho = np.zeros((sn1, sn2))
    rho[2:-2, 2:-2] = np.maximum(p[0, 2:-2, 2:-2, 0], 0.0)
    w = (rho * g).ravel()
    rng = np.random.default_rng(seed)
    pick = rng.choice(w.size, size=n, p=w / w.sum())
    i, j = pick // sn2, pick % sn2
    prm = pr.params
    X = np.zeros((n, 3))
    X[:, 0] = prm.startx[1] + ((i - 2) + 0.5) * prm.dx[1]
    X[:, 1] = prm.startx[2] + ((j - 2) + 0.5) * prm.dx[2]
    ids = np.stack([i, j, np.zeros(n, dtype=np.int64)], axis=1)
    return ids, X


def generator_cpu_rate(np, hc, xa, ya, hd, mask, seed, nodes=96):
    """abundance() on the host's cores over a random sample of the computed
    nodes (mask): the CPU rate beside the device's (the reference's own
    generator is Fortran, which this box cannot compile)."""
    rng = np.random.default_rng(seed)
    t, i, j = np.nonzero(mask)
    pick = rng.choice(len(t), size=min(nodes, len(t)), replace=False)
    t0 = time.perf_counter()
    hc.nu_abundance(xa[i[pick]], ya[j[pick]], hd[t[pick]])
    s = time.perf_counter() - t0
    return {"cpu_nodes_per_s": len(pick) / s, "cpu_cores": os.cpu_count(),
            "cpu_sample": "%d random nodes of the computed ones, all cores" % len(pick)}


def run_cool(args):
    """The COOL_EOS step on the 256x256 torus of the reference's init.c literals
    (a=0.6, rin=4, rmax=11.8, beta=50; cooleos.c's 3 Msun hole and units), FP64,
    with per-radius tables, and 1e5 tracer particles seeded in proportion to the
    rest mass.  Tables: the reference's 72x72 grid or a 200x200 grid over rho
    1e4-1e14 g/cm^3 and T 1e8-1e12 K from the synthetic ideal-gas-plus-radiation generator of
    harm_cool_b200.eos_tables, or ("physics") the 200x200 grid from the
    library's abundance() on the GPU, its nodes computed as the run reads them
    (eos_tables.on_demand: the whole run is repeated until it reads no node that
    is not computed, and that last run is the one reported).  The first step
    seeds the per-zone temperature guesses row by row and runs outside the
    timed region."""
    import numpy as np
    import harm_cool_b200 as hc
    from harm_cool_b200 import eos_tables
    n = args.cool_n
    pr = hc.torus_problem(n, n, 1, a=0.6, rin=4.0, rmax=11.8, beta=50.0)
    args.steps = max(args.steps, 200)  # a few ms per step: enough for the clock sampler to see the run
    gen = None
    if args.cool_tables == "reference":
        # cooleos.c:924-940: 72 x 72 over rho 1e2..1e15 g/cm^3, T 1e4..1e18 K
        xa, ya, val, consts = eos_tables.build_tables(eos_tables.zone_radii(pr), gam=pr.params.gam)
        tables = "72x72 per-radius tables (rho 1e2-1e15, T 1e4-1e18)"
    else:
        # 200 x 200 over rho 1e4..1e14 g/cm^3, T 1e8..1e12 K, and a density unit that
        # puts the torus maximum (rho = 1 in code units) at 1e11 g/cm^3
        if args.cool_tables == "physics":
            xa, ya = eos_tables.log_axis(200, 1.e4, 1.e14), eos_tables.log_axis(200, 1.e8, 1.e12)
            consts = eos_tables.constants(pr.params.gam, (1.e4, 1.e14), (1.e8, 1.e12))
            consts["hdfac"] = np.array([eos_tables.hdfac(r) for r in eos_tables.zone_radii(pr)])
            val = None
        else:
            xa, ya, val, consts = eos_tables.build_tables(eos_tables.zone_radii(pr), nx=200, ny=200,
                                                          rho=(1.e4, 1.e14), T=(1.e8, 1.e12), gam=pr.params.gam)
        consts["rho_unit"] = 1.e11
        consts["u_unit"] = consts["p_unit"] = 1.e11 * eos_tables.CL * eos_tables.CL
        tables = "200x200 per-radius tables (rho 1e4-1e14, T 1e8-1e12), torus maximum at 1e11 g/cm^3"
    zones = pr.zones
    tracer_seed = {}

    def fp64_run(eos):
        """seeding step, warm-up, timed steps, kernel timings and the host-array run"""
        ctx = hc.Context(pr)
        ctx.init_torus()
        ctx.set_eos(eos)
        if "ids" not in tracer_seed:
            tracer_seed["ids"], tracer_seed["X"] = tracers_by_density(np, pr, ctx.get_prims(), args.cool_tracers,
                                                                      args.seed)
        ctx.tracers_put(tracer_seed["ids"], tracer_seed["X"])
        t0 = time.perf_counter()
        ctx.run(1)                       # the seeding step
        r = {"seed_s": time.perf_counter() - t0}
        ctx.run(args.warmup - 1)
        sampler = ClockSampler(0)
        sampler.start()
        r["ms"] = ctx.run_timed(args.steps)
        r["clocks"] = sampler.stop()
        r["pa"] = ctx.get_prims()        # after warmup + steps, for the mixed run's L1
        r["lastT"] = ctx.eos_guess()
        r["kms"] = ctx.time_kernels(reps=2)
        import torch
        pinned = torch.empty(pr.shape + (8,), dtype=torch.float64, pin_memory=True).numpy()
        pinned[...] = ctx.get_prims()
        r["ms_e2e"] = ctx.step_ch_host_timed(pinned, args.e2e_steps)
        r["diag"], r["time"] = ctx.diag(), ctx.time()
        ctx.close()
        return r

    def mixed_run(eos):
        """the face physics' EOS calls in FP32, the same steps as the FP64 run"""
        cm = hc.Context(pr)
        cm.init_torus()
        cm.set_precision(hc.Context.MIXED)
        cm.set_eos(eos)
        cm.tracers_put(tracer_seed["ids"], tracer_seed["X"])
        cm.run(args.warmup)
        sampler = ClockSampler(0)
        sampler.start()
        r = {"ms": cm.run_timed(args.steps)}
        r["clocks"] = sampler.stop()
        r["pb"] = cm.get_prims()
        r["kms"] = cm.time_kernels(reps=2)
        r["fail_code"] = cm.diag()["fail_code"]
        cm.close()
        return r

    mixed = None
    if args.cool_tables == "physics":
        def both(eos):
            return fp64_run(eos), (None if args.no_mixed else mixed_run(eos))
        (res, mixed), how, have = eos_tables.on_demand(both, xa, ya, consts)
        seen = res["lastT"][res["lastT"] > 0]
        gen = dict(how, zone_T_range_K=[float(seen.min()), float(seen.max())] if seen.size else None)
        gen["nodes_per_s"] = gen["nodes"] / gen["generation_s"] if gen["generation_s"] > 0 else None
        gen.update(generator_cpu_rate(np, hc, xa, ya, consts["hdfac"], have, args.seed))
        eos = None
    else:
        eos = hc.Eos(xa, ya, val, consts)
        res = fp64_run(eos)
    ms, kms, pa = res["ms"], res["kms"], res["pa"]
    value = zones * args.steps / (ms / 1e3)
    bytes_host = int(np.prod(pr.shape)) * 8 * 8
    dom = max(("flux", "update"), key=lambda k: kms[k])
    peak, peak_kind = measured_peaks()
    alg = alg_bytes_per_zone(dom, 1) * zones
    achieved = alg / (kms[dom] / 1e3) / 1e9
    tbytes = len(consts["hdfac"]) * len(xa) * len(ya) * 5 * 8
    line = {"metric": "zone-cycles/s %dx%d GRMHD step_ch with COOL_EOS" % (n, n), "value": value,
            "unit": "zone-cycles/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": "FM torus %dx%d (a=0.6, rin=4, rmax=11.8, beta=50), COOL_EOS, %s, "
                                   "%s, %d tracers seeded by rest mass"
                                   % (n, n, tables, "generator tables (abundance() on the GPU, nodes computed as "
                                      "the run reads them)" if args.cool_tables == "physics"
                                      else "synthetic generator", args.cool_tracers),
                       "l2": ("tables (%.0f MB) %s; state per step is small"
                              % (tbytes / 1e6, "fit in L2" if tbytes < 126e6 else "exceed L2 (126 MB)"))},
            "seeding_step_s": res["seed_s"],
            "e2e": {"value": zones * args.e2e_steps / (res["ms_e2e"] / 1e3), "unit": "zone-cycles/s",
                    "h2d_bytes_per_step": bytes_host, "d2h_bytes_per_step": bytes_host,
                    "steps": args.e2e_steps,
                    "path": "harm_run_host: per step upload, step, download, each upload overlapped with the "
                            "previous step's download"},
            "gpu_launches": kernels_per_step(1) * args.steps,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "algorithmic_bytes": alg,
                         "peak_source": peak_kind,
                         "note": "the T solves make these kernels FP64-latency bound, not HBM bound"},
            "kernel_ms": kms, "clocks": res["clocks"], "sim_time": res["time"], "fail_code": res["diag"]["fail_code"]}
    if gen is not None:
        line["tables"] = gen
    if not args.no_mixed:
        if mixed is None:
            mixed = mixed_run(eos)
        pb = mixed["pb"]
        act = (slice(None), slice(2, -2), slice(2, -2))
        if args.dump_cool:
            np.savez_compressed(args.dump_cool, fp64=pa, mixed=pb)
        line["mixed"] = {"value": zones * args.steps / (mixed["ms"] / 1e3), "ms_per_step": mixed["ms"] / args.steps,
                         "speedup_vs_fp64": ms / mixed["ms"], "clocks": mixed["clocks"], "kernel_ms": mixed["kms"],
                         "l1_vs_fp64": l1_errors(pa[act], pb[act]), "l1_after_steps": args.warmup + args.steps,
                         "fail_code": mixed["fail_code"]}
    if eos is not None:
        eos.close()
    if not args.no_cpu_baseline and args.cool_tables == "reference":
        exe = os.path.join(ROOT, "oracle", "_ref", "ce%d" % n, "refbench")
        if os.path.exists(exe):
            out = subprocess.run([exe, "1", "1"], capture_output=True, text=True, cwd=os.path.dirname(exe)).stdout
            r = json.loads(out.strip().splitlines()[-1])
            line["cpu_baseline"] = {"value": r["zone_cycles_per_s"], "unit": "zone-cycles/s", "cores": 1,
                                    "kind": "reference", "sample": "reference COOL_EOS step_ch() on %dx%d, "
                                    "1 step after 1 warm-up, oracle/eos_standin.c tables" % (n, n)}
    print(json.dumps(line), flush=True)


def run_profile(args):
    """A case for ncu: the torus at the given size and precision, --warmup steps,
    then --steps more; the step kernels of the last steps are the ones to capture
    (each step launches 5 flux/update kernels per half step in 3D: -s 10*warmup)."""
    import harm_cool_b200 as hc
    if args.member >= 0:
        # one draw of the ensemble workload (--members, --seed) alone
        pr, desc = hc.ensemble_problems(args.members, seed=args.seed)[args.member]
        name = "ensemble member %d of seed %d: %s" % (args.member, args.seed, json.dumps(desc))
    else:
        pr = hc.torus_problem(args.n1, args.n2, args.n3)
        name = "torus %dx%dx%d" % (args.n1, args.n2, args.n3)
    ctx = hc.Context(pr)
    ctx.init_torus()
    if args.precision == "mixed":
        ctx.set_precision(hc.Context.MIXED)
    ctx.run(args.warmup)
    ctx.sync()
    ms = ctx.run_timed(args.steps)
    print(json.dumps({"workload": "profile case, %s, %s" % (name, args.precision),
                      "warmup": args.warmup, "steps": args.steps, "ms_per_step": ms / args.steps,
                      "fail_code": ctx.diag()["fail_code"]}), flush=True)
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--n1", type=int, default=288)
    ap.add_argument("--n2", type=int, default=256)
    ap.add_argument("--n3", type=int, default=256)
    ap.add_argument("--e2e-steps", type=int, default=8,
                    help="steps of the host-array run (harm_run_host) that the e2e figure times")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision run")
    ap.add_argument("--l1-steps", type=int, default=1000,
                    help="steps of the FP64 and mixed runs whose L1 difference the mixed line reports (0: skip)")
    ap.add_argument("--precision", choices=("fp64", "mixed"), default="fp64",
                    help="precision of the profile workload")
    ap.add_argument("--workload", choices=("torus", "ensemble", "cool", "adjoint", "profile"), default="torus",
                    help="torus: the 288x256x256 step (default); ensemble: 64 seeded 2D tori; "
                         "cool: the 256x256 COOL_EOS step")
    ap.add_argument("--cool-n", type=int, default=256)
    ap.add_argument("--cool-tracers", type=int, default=100000)
    ap.add_argument("--cool-tables", choices=("reference", "baseline", "physics"), default="reference",
                    help="reference: cooleos.c's 72x72 tables and units; baseline: 200x200 tables over "
                         "rho 1e4-1e14, T 1e8-1e12 with the torus maximum at 1e11 g/cm^3; physics: the "
                         "baseline grid filled by the library's abundance() on the GPU as the run reads it")
    ap.add_argument("--dump-cool", default=None, help="save the FP64 and mixed COOL_EOS states (npz)")
    ap.add_argument("--adj-n", type=int, default=192, help="adjoint workload: N1 = N2")
    ap.add_argument("--adj-steps", type=int, default=50, help="adjoint workload: steps K")
    ap.add_argument("--adj-every", type=int, default=10, help="adjoint workload: checkpoint spacing")
    ap.add_argument("--members", type=int, default=64)
    ap.add_argument("--member", type=int, default=-1, help="profile workload: this ensemble draw alone")
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        # host-only: rank 0 times the reference, the other ranks have nothing to do
        run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")))
        return
    if args.workload == "ensemble":
        run_ensemble(args)
        return
    if args.workload == "cool":
        run_cool(args)
        return
    if args.workload == "adjoint":
        run_adjoint(args)
        return
    if args.workload == "profile":
        run_profile(args)
        return
    world, rank, local = dist_setup()
    try:
        run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
