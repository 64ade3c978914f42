"""Benchmark of the boundary-value solve (assembly + LU + boundary values +
radiation force) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload sphere216]

A step is one complete solve of the workload: both domains' coefficient
matrices, the global LU solve, P/dP, pv, the dpv solves and the type-0
radiation force.  Rank 0 prints one JSON line.

  value  solves/s with the problem resident on the device (bemgpu_run +
         bemgpu_force), CUDA events on the library's stream, L2 flushed
         (256 MB write) between steps, max over ranks
  e2e    the same solves through the drop-in C API with host buffers
         (solve_bieq_aqd2 uploads the element tables, solves, downloads P, dP,
         pv, dpv; force_FN_aqd2 returns F, N)
  roofline  the dominant kernel (periodic regular-pair assembly), FP64 work
         = lattice terms x a fixed FP64 operation count per term
  cpu_baseline  the reference's own assembly loop (oracle/_ref) timed on a
         bounded sample of collocation elements on the host cores,
         extrapolated linearly in elements, plus the dense solves

--impl reference runs only the CPU arm (rank 0; other ranks exit).  N > 1
runs independent replicas (the solve of one system does not shard without a
distributed LU; requests are independent), scaling "weak".
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# FP64 operations per lattice term of the Green's-function sums (real-space or
# spectral term with its Faddeeva / erfc evaluation, per-point set-up
# amortised): counted once with ncu's FP64 instruction counters on the first
# implementation of the periodic regular-pair kernel on the 216-quad sphere
# (1.88e12 flop / 6.727e9 terms); frozen, never re-tuned.
C_TERM_FLOPS = 280.0
# nominal FP64 peak of B200 (148 SMs x 64 FP64 FMA/clk x 2 x 1.965 GHz), for
# context; the roofline divides by the FP64 rate measured in the run
# (measured_fp64_peak), as the bf16 and HBM peaks of this pool are measured
FP64_NOMINAL_TFLOPS = 37.2
# The regular-pair kernels' hardware readings from one ncu capture of a
# warm-up assembly of the timed configuration on the 216-quad workload
# (profiles/k_q0_regular_far_sphere216.md, command given there): FP64 pipe busy
# fraction (sm__pipe_fp64_cycles_active over active cycles) and DRAM bytes read +
# written per launch, for k_q0_regular and each shorter-rule tier's k_q0_far<n>.
# Reported for that workload only.
NCU_WORKLOAD = "sphere216"
NCU_REGULAR = {"k_q0_regular": {"fp64_pipe": 0.4343, "dram_bytes": 434432 + 7126272},
               "k_q0_far<10>": {"fp64_pipe": 0.4598, "dram_bytes": 414720 + 20992},
               "k_q0_far<9>": {"fp64_pipe": 0.5040, "dram_bytes": 960512 + 305408},
               "k_q0_far<8>": {"fp64_pipe": 0.5010, "dram_bytes": 817152 + 1160192},
               "k_q0_far<7>": {"fp64_pipe": 0.4631, "dram_bytes": 1312000 + 1236480},
               "k_q0_far<6>": {"fp64_pipe": 0.0, "dram_bytes": 85760 + 0}}


def measured_fp64_peak():
    """FP64 rate of a dense cuBLAS DGEMM (torch float64 matmul, 8192^3,
    2 n^3 flop, best of 3 with CUDA events): the measured FP64 ceiling of this
    GPU, in TFLOP/s."""
    import torch
    n = 8192
    g = torch.Generator(device="cuda").manual_seed(0)
    a = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g)
    b = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g)
    torch.matmul(a, b)
    best = float("inf")
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        c = torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1000.0)
    del a, b, c
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="sphere216")
    ap.add_argument("--cpu-seconds", type=float, default=20.0, help="budget of the CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-budget-s", type=float, default=150.0,
                    help="reference arm: host seconds of complete reference solves (at least one is timed)")
    ap.add_argument("--profile-mixed", action="store_true",
                    help="bracket the first timed mixed-precision step with cudaProfilerStart/Stop "
                         "(for ncu --profile-from-start off)")
    ap.add_argument("--rate", type=float, default=10.0, help="stream workload: mean arrivals per second")
    ap.add_argument("--slots", type=int, default=4, help="stream workload: server slots")
    ap.add_argument("--hbm-gb", type=float, default=150.0, help="stream: device-memory budget of the server (GiB)")
    ap.add_argument("--stream-sizes", default="6,10", help="--workload stream: cube-sphere n (6 n^2 quads)")
    ap.add_argument("--sweep-freqs", type=int, default=2, help="--workload sweep: frequencies (of 8)")
    ap.add_argument("--sweep-dirs", type=int, default=8, help="--workload sweep: incidence directions (of 64)")
    ap.add_argument("--sweep-mesh-n", type=int, default=16,
                    help="--workload sweep: cube-sphere with 6 n^2 quads (16: the 1536-quad body of the sweep)")
    ap.add_argument("--stream-requests", type=int, default=STREAM_REQUESTS,
                    help="requests of the headline stream in the default line (0: leave it out)")
    ap.add_argument("--lu-sizes", default="1728,4096,12288", help="--workload lu: matrix orders")
    ap.add_argument("--lu-arith", default="z,c,t1,t3",
                    help="--workload lu: z FP64 (DMMA), c complex FP32 (CUDA cores), t1 / t3 complex FP32 with "
                         "one / three split TF32 products on the tensor cores")
    ap.add_argument("--mixed-mode", type=int, default=2,
                    help="precision of the mixed form: 1 FP32, 2 TF32 (one product on the tensor cores), 3 TF32x3 "
                         "(three split TF32 products), 4 as 2; 0: skip it")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""
    FIELDS = ["clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.hw_slowdown",
              "clocks_event_reasons.hw_thermal_slowdown", "clocks_event_reasons.sw_thermal_slowdown",
              "clocks_event_reasons.sw_power_cap"]

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + ",".join(self.FIELDS),
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        sm = [float(r[0]) for r in self.rows if len(r) >= 7 and r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if len(r) >= 7 and r[1].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) >= 7:
                for n, v in zip(names, r[3:7]):
                    if v.lower() == "active":
                        reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(files, budget_s, threads=None, seed=20241209):
    """The reference's own assembly loop (oracle/_ref) on a seeded random
    sample of collocation elements of each domain, extrapolated linearly to
    all of them, plus the dense solves: a bounded sample (about budget_s of
    host time) of one solve, labelled as extrapolated."""
    from oracle import refwrap
    if not refwrap.available():
        return None
    threads = threads or os.cpu_count()
    os.environ["OMP_NUM_THREADS"] = str(threads)
    case = refwrap.RefCase(*files)
    rng = np.random.default_rng(seed)
    ne0, ne1 = case.dom_ne[0], case.dom_ne[1]
    # as many elements per domain as host threads (the reference's OpenMP loop
    # runs over collocation elements, dynamic schedule), drawn at random
    m0, m1 = min(ne0, threads), min(ne1, threads)
    rows0 = np.sort(rng.choice(ne0, m0, replace=False)) + 1
    rows1 = np.sort(rng.choice(ne1, m1, replace=False)) + 1
    t0 = time.perf_counter(); case.assemble_list(0, rows0); s0 = time.perf_counter() - t0
    t0 = time.perf_counter(); case.assemble_list(1, rows1); s1 = time.perf_counter() - t0
    t_asm = s0 * ne0 / m0 + s1 * ne1 / m1
    # dense solves with the same OpenBLAS the reference build links (n = 2 NN; dpv: NN with 3 rhs per domain)
    n = 8 * ne0
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    b = rng.standard_normal(n) + 0j
    t0 = time.perf_counter(); np.linalg.solve(A, b); ts = time.perf_counter() - t0
    A2 = A[: n // 2, : n // 2].copy()
    B2 = rng.standard_normal((n // 2, 3)) + 0j
    t0 = time.perf_counter(); np.linalg.solve(A2, B2); np.linalg.solve(A2, B2); td = time.perf_counter() - t0
    total = t_asm + ts + td
    return {"value": 1.0 / total, "unit": "solves/s", "cores": threads, "kind": "reference",
            "sample": "extrapolated: reference create_cmatrix_domain loop on %d of %d collocation elements (domain 0) "
                      "and %d of %d (domain 1), drawn with numpy default_rng(%d), %d OpenMP threads, scaled linearly "
                      "in elements (%.1f s measured); dense solves timed at n=%d (OpenBLAS zgesv, as linked by the "
                      "reference build)" % (m0, ne0, m1, ne1, seed, threads, s0 + s1, n),
            "seconds_per_solve": total, "assembly_seconds_extrapolated": t_asm}


# Workloads whose full reference solve fits a bench run (about 3 minutes on
# 16 host threads for the 216-quad sphere): the reference arm times complete
# solves of these; larger ones are sampled and extrapolated (cpu_baseline).
FULL_REFERENCE_SOLVE = {"sphere216"}


def reference_full_solves(files, budget_s, max_steps, threads):
    """Complete solves by the reference's own solver program
    (oracle/_ref/aw_d3qd2_bv_solver: read, assemble, PARDISO stand-in, pv,
    dpv, .dat write) plus its type-0 force (force_FN_aqd2), each timed on the
    host clock; repeated while the budget lasts (at least one)."""
    from oracle import refwrap
    exe = os.path.join(ROOT, "oracle", "_ref", "aw_d3qd2_bv_solver")
    wd = os.path.dirname(files[0])
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    times = []
    t_start = time.perf_counter()
    while len(times) < max_steps:
        t0 = time.perf_counter()
        r = subprocess.run([exe] + [os.path.basename(f) for f in files] + ["ref_out.dat"], cwd=wd, env=env,
                           stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, text=True)
        if r.returncode != 0:
            raise RuntimeError("reference solver failed: " + r.stderr[-500:])
        os.environ["OMP_NUM_THREADS"] = str(threads)
        case = refwrap.RefCase.from_dat(os.path.join(wd, "ref_out.dat"))
        case.force(0)
        times.append(time.perf_counter() - t0)
        elapsed = time.perf_counter() - t_start
        if elapsed + times[-1] > budget_s:
            break
    return times


def run_reference(args, rank, world):
    if rank != 0:
        return
    from bem3_aw_qd2_b200 import meshgen
    d = tempfile.mkdtemp(prefix="bench_ref_")
    files = meshgen.write_inputs(d, **meshgen.CONFIGS[args.workload])
    from oracle import refwrap
    if not refwrap.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (the reference build) is missing"}))
        return
    threads = os.cpu_count()
    base = {"impl": "reference", "metric": "solves/s", "unit": "solves/s", "n_gpus": args.gpus,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, **workload_desc(args.workload)}, "steps_requested": args.steps,
            "warmup_requested": args.warmup}
    if args.workload in FULL_REFERENCE_SOLVE:
        # complete solves, as many as fit the budget: steps = solves timed
        times = reference_full_solves(files, args.ref_budget_s, args.steps, threads)
        v = len(times) / sum(times)
        cb = {"value": v, "unit": "solves/s", "cores": threads, "kind": "reference",
              "sample": "%d complete solve(s) of the workload by the reference's own aw_d3qd2_bv_solver "
                        "(oracle/_ref, OpenMP on %d host threads, dense LU stand-in for PARDISO on OpenBLAS) plus "
                        "force_FN_aqd2 type 0, host clock per solve; no warm-up solve (CPU code)" % (len(times),
                                                                                                 threads),
              "seconds_per_solve": [float(t) for t in times]}
        line = dict(base, value=v, steps=len(times), warmup=0, ms_per_step=1000.0 * sum(times) / len(times))
    else:
        warm = refwrap.RefCase(*files)
        for _ in range(args.warmup):  # warm-up: one interior collocation element (pages in code and data)
            warm.assemble_rows(1, 1, 2)
        vals, walls = [], []
        for step in range(args.steps):
            t0 = time.perf_counter()
            cb = cpu_baseline(files, args.cpu_seconds, threads, seed=20241209 + step)
            walls.append(time.perf_counter() - t0)
            vals.append(cb["value"])
        v = statistics.mean(vals)
        cb["value"] = v
        cb["sample"] += "; mean of %d seeded samples" % args.steps
        line = dict(base, value=v, steps=args.steps, warmup=args.warmup,
                    ms_per_step=1000.0 * sum(walls) / len(walls), extrapolated=True)
    line["cpu_baseline"] = cb
    line["e2e"] = {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    print(json.dumps(line))


STREAM_DESC = ("seeded Poisson request stream (numpy default_rng(2024)) at the given rate: cube-spheres and spheroids "
               "of {sizes} quads (sizes drawn uniformly), radius 0.2-0.35 wavelengths (spheroids 0.85/0.85/1.15 of "
               "it), square or triangular lattice of period 0.7-1.1 wavelengths (redrawn when the body's horizontal "
               "extent exceeds 0.9 of the period), k.a in [1, 2.5], theta 0-60 deg, phi 0-360 deg; 30% of requests "
               "repeat an earlier (mesh, k, in-plane wave vector) with a new amplitude or the mirrored polar angle; "
               "draws within 2% of a Rayleigh anomaly are redrawn")
# the headline request stream: its mesh sizes (6 n^2 quads) and request count
STREAM_SIZES = (6, 16, 24, 32)
STREAM_REQUESTS = 12


def stream_requests(count, rng, sizes=STREAM_SIZES, radius=(0.2, 0.35)):
    """The request stream: (meshgen arguments, reuse key) per request."""
    import math
    reqs, seen = [], []
    while len(reqs) < count:
        if seen and rng.random() < 0.3:
            base = seen[int(rng.integers(len(seen)))]
            r = dict(base[0])
            if rng.random() < 0.5:
                r["theta_deg"] = 180.0 - r["theta_deg"]
            r["amp"] = (float(rng.uniform(0.5, 1.5)), float(rng.uniform(-1, 1)))
            reqs.append((r, base[1]))
            continue
        n = int(rng.choice(list(sizes)))
        rad = float(rng.uniform(*radius))
        axes = (rad, rad, rad) if rng.random() < 0.5 else (0.85 * rad, 0.85 * rad, 1.15 * rad)
        a = float(rng.uniform(0.7, 1.1))
        if 2.0 * axes[0] > 0.9 * a:  # the body must fit its lattice cell with a gap
            continue
        lat = ((a, 0.0), (0.0, a)) if rng.random() < 0.5 else ((a, 0.0), (0.5 * a, 0.5 * math.sqrt(3.0) * a))
        k = float(rng.uniform(1.0, 2.5)) / a
        th, ph = float(rng.uniform(0.0, 60.0)), float(rng.uniform(0.0, 360.0))
        kx, ky = k * math.sin(math.radians(th)) * math.cos(math.radians(ph)), k * math.sin(math.radians(th)) * math.sin(math.radians(ph))
        # Rayleigh anomalies |k_par + g| = k: keep 2% away
        det = lat[0][0] * lat[1][1] - lat[1][0] * lat[0][1]
        g1 = (2 * math.pi * lat[1][1] / det, -2 * math.pi * lat[1][0] / det)
        g2 = (-2 * math.pi * lat[0][1] / det, 2 * math.pi * lat[0][0] / det)
        bad = any(abs(math.hypot(kx + i * g1[0] + j * g2[0], ky + i * g1[1] + j * g2[1]) - k) < 0.02 * k
                  for i in range(-6, 7) for j in range(-6, 7))
        if bad or th < 0.5:  # the reference rejects kx = ky = 0
            continue
        r = dict(n=n, semi_axes=axes, lattice=lat, theta_deg=th, phi_deg=ph, wavelength=2 * math.pi / k)
        key = hash((n, axes, lat, round(k, 14), round(kx, 12), round(ky, 12))) & 0xFFFFFFFFFFFFFFFF
        seen.append((r, key))
        reqs.append((r, key))
    return reqs


def stream_compare(count, rate, slots, hbm_gb, mixed_mode, sizes=STREAM_SIZES, seed=2024, device=0):
    """The headline comparison on one GPU: a seeded request stream served by
    the native server in mixed precision (continuous batching, factorisation
    and interior reuse, admission by device memory) against the plain FP64
    drop-in path, one solve_bieq_aqd2 + force_FN_aqd2 per request in arrival
    order with no reuse.  Both see the same arrival times; latency is arrival
    to result.  Returns the sub-record of the bench line."""
    from bem3_aw_qd2_b200 import api, meshgen
    h, g = api.libs()
    h.aqd2_set_verbose(0)
    rng = np.random.default_rng(seed)
    reqs = stream_requests(count, rng, sizes)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, count))
    files = [meshgen.write_inputs(tempfile.mkdtemp(prefix="stream_"), **r) for r, _ in reqs]
    # plain FP64 drop-in path: requests in arrival order, one context each
    # (read + initialisation from the input files happen before the clock)
    cases = [api.Case.from_files(*f) for f in files]
    F_plain, lat_plain = [], []
    t0 = time.perf_counter()
    for i, c in enumerate(cases):
        while time.perf_counter() - t0 < arrivals[i]:
            time.sleep(0.0005)
        c.solve()
        F_plain.append(c.force(0)[0])
        c.close()
        lat_plain.append((time.perf_counter() - t0 - arrivals[i]) * 1000.0)
    el_plain = time.perf_counter() - t0
    # served, mixed precision
    cases = [api.Case.from_files(*f) for f in files]
    probs = [c.problem() for c in cases]
    srv = api.Server(device=device, hbm_budget=int(hbm_gb * (1 << 30)), slots=slots)
    done, t_sub = {}, {}
    t0 = time.perf_counter()
    for i in range(count):
        while time.perf_counter() - t0 < arrivals[i]:
            for r in srv.poll(timeout_ms=1):
                done[r.id] = (r, time.perf_counter())
        t_sub[i] = time.perf_counter()
        srv.submit(probs[i], reqs[i][1], i, precision=mixed_mode)
    while len(done) < count:
        for r in srv.poll(timeout_ms=100):
            done[r.id] = (r, time.perf_counter())
    el_served = max(t for _, t in done.values()) - t0
    st = srv.stats()
    srv.close()
    lat_served = [(done[i][1] - t0 - arrivals[i]) * 1000.0 for i in range(count)]
    bad = [done[i][0].error.decode() for i in range(count) if done[i][0].status != 0]
    fp64_run = sum(1 for i in range(count) if done[i][0].precision == 0)
    errs = [float(np.linalg.norm(np.array(done[i][0].F[:]) - F_plain[i]) / np.linalg.norm(F_plain[i]))
            for i in range(count) if done[i][0].status == 0]
    for c, p in zip(cases, probs):
        c.free_problem(p)
        c.close()
    sizes_drawn = [6 * r["n"] ** 2 for r, _ in reqs]
    return {"requests": count, "rate_per_s": rate, "mesh_quads": sizes_drawn,
            "repeats": int(count - len({k for _, k in reqs})),
            "plain_fp64": {"value": count / el_plain, "unit": "solves/s", "path": "solve_bieq_aqd2 + force_FN_aqd2 "
                           "per request (C ABI, host buffers), arrival order, no reuse",
                           "latency_ms": {"p50": float(np.percentile(lat_plain, 50)),
                                          "p99": float(np.percentile(lat_plain, 99))}},
            "served_mixed": {"value": count / el_served, "unit": "solves/s",
                             "mode": {1: "FP32", 2: "TF32", 3: "TF32x3", 4: "TF32"}.get(mixed_mode, "?") +
                                     " LU updates + FP64 refinement",
                             "slots": slots, "hbm_budget_gb": hbm_gb,
                             "latency_ms": {"p50": float(np.percentile(lat_served, 50)),
                                            "p99": float(np.percentile(lat_served, 99))},
                             "reused": int(st["reused"]), "evictions": int(st["evictions"]),
                             "ran_fp64_for_memory": fp64_run,
                             "bytes_peak": st["bytes_peak"], "failed": len(bad), "errors": bad[:3]},
            "served_over_plain": (count / el_served) / (count / el_plain),
            "target": ">= 3x served mixed over plain FP64 at force rel. err <= 1e-8",
            "force_rel_err_vs_plain_fp64": {"max": max(errs) if errs else None,
                                            "median": float(np.median(errs)) if errs else None},
            "stream": STREAM_DESC.format(sizes="/".join(str(6 * n * n) for n in sizes))}


def run_stream(args, rank, world):
    """Serving: the request stream through the native server (continuous
    batching, factorisation reuse, HBM admission), plain FP64 and mixed."""
    from bem3_aw_qd2_b200 import api, meshgen, replicas
    h, g = api.libs()
    h.aqd2_set_verbose(0)
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        # replicas: one stream of world x count requests at world x rate, each
        # rank serving its round-robin share (count requests at the given rate)
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    rng = np.random.default_rng(2024)
    per_rank = max(args.steps, 8) * 8
    total = per_rank * world
    all_reqs = stream_requests(total, rng, sizes=tuple(int(x) for x in args.stream_sizes.split(",")))
    all_arrivals = np.cumsum(rng.exponential(1.0 / (args.rate * world), total))
    mine = replicas.shard(total, rank, world)
    reqs = [all_reqs[i] for i in mine]
    arrivals = all_arrivals[mine]
    count = len(reqs)
    # requests are built (mesh, element tables, incident field) before the clock starts
    cases, probs = [], []
    for i, (r, key) in enumerate(reqs):
        d = tempfile.mkdtemp(prefix="stream_")
        c = api.Case.from_files(*meshgen.write_inputs(d, **r))
        cases.append(c)
        probs.append(c.problem())
    out = {}
    for tag, prec in (("fp64", 0), ("mixed", args.mixed_mode or 2)):
        srv = api.Server(device=local, hbm_budget=int(args.hbm_gb * (1 << 30)), slots=args.slots)
        # warm-up: one request per mesh size
        for i, n in enumerate(sorted({r["n"] for r, _ in reqs})):
            j = next(k for k, (r, _) in enumerate(reqs) if r["n"] == n)
            srv.submit(probs[j], 0xFFFF0000 + i, -1 - i, precision=prec)
        got = 0
        while got < len({r["n"] for r, _ in reqs}):
            got += len(srv.poll(timeout_ms=1000))
        done, t_sub = {}, {}
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        for i in range(count):
            while time.perf_counter() - t0 < arrivals[i]:
                for r in srv.poll(timeout_ms=1):
                    done[r.id] = (r, time.perf_counter())
            t_sub[i] = time.perf_counter()
            srv.submit(probs[i], reqs[i][1], i, precision=prec)
        while len(done) < count:
            for r in srv.poll(timeout_ms=100):
                done[r.id] = (r, time.perf_counter())
        t1 = max(t for _, t in done.values())
        st = srv.stats()
        srv.close()
        lat = [(done[i][1] - t_sub[i]) * 1000.0 for i in range(count)]
        bad = [done[i][0].error.decode() for i in range(count) if done[i][0].status != 0]
        # slowest rank's wall time and latency percentiles, all ranks' requests
        (el, p50, p99), (n_all, n_bad, n_reused) = replicas.reduce_timing(
            [t1 - t0, np.percentile(lat, 50), np.percentile(lat, 99)], [count, len(bad), st["reused"]],
            device="cuda" if world > 1 else "cpu")
        out[tag] = {"value": n_all / el, "latency_ms": {"p50": p50, "p99": p99},
                    "reused": int(n_reused), "evictions": int(st["evictions"]),
                    "bytes_peak": st["bytes_peak"], "failed": int(n_bad),
                    "F": {i: list(done[i][0].F[:]) for i in range(count)}}
    errs = []
    for i in range(count):
        a, b = np.array(out["fp64"]["F"][i]), np.array(out["mixed"]["F"][i])
        errs.append(float(np.linalg.norm(a - b) / np.linalg.norm(a)))
    for tag in out:
        del out[tag]["F"]
    for c, p in zip(cases, probs):
        c.free_problem(p)
        c.close()
    mixed = out["mixed"]
    (emax,), _ = replicas.reduce_timing([max(errs)], [], device="cuda" if world > 1 else "cpu")
    line = {"metric": "solves/s", "value": mixed["value"], "unit": "solves/s", "n_gpus": world, "steps": total,
            "warmup": 3, "ms_per_step": 1000.0 / mixed["value"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 assembly, complex-FP32 LU + FP64 refinement", "data": "synthetic",
            "config": {"workload": "stream", "requests": total, "rate_per_s": args.rate * world,
                       "requests_per_gpu": per_rank, "slots": args.slots,
                       "hbm_budget_gb": args.hbm_gb,
                       "stream": STREAM_DESC.format(sizes="/".join(str(6 * int(x) ** 2)
                                                                  for x in args.stream_sizes.split(",")))},
            "latency_ms": mixed["latency_ms"], "fp64": out["fp64"], "mixed": mixed,
            "force_rel_err_mixed_vs_fp64": {"max": emax, "median": float(np.median(errs))}}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


def roofline_record(achieved, fp64_peak, terms_reg, cnt, workload, out_bytes):
    """The dominant kernels' roofline: periodic regular-pair assembly
    (k_q0_regular on the reference's rule, k_q0_far<n> on the shorter rules'
    tiers, one phase), FP64
    work = lattice terms counted by the kernels x the frozen per-term count,
    over the phase's CUDA-event time; beside it the FP64 pipe fraction and DRAM
    traffic ncu read on the same kernels."""
    traffic, pipe = None, {k: None for k in NCU_REGULAR}
    if workload == NCU_WORKLOAD:
        traffic = sum(v["dram_bytes"] for v in NCU_REGULAR.values())
        pipe = {k: v["fp64_pipe"] for k, v in NCU_REGULAR.items()}
    return {"bound": "fp64", "kernel": "k_q0_regular + k_q0_far<10..6> (regular pairs)", "achieved": achieved,
            "peak": fp64_peak, "unit": "TFLOP/s", "frac": (achieved / fp64_peak) if achieved else None,
            "traffic": traffic, "traffic_unit": "bytes per assembly over the phase's 6 launches (ncu dram__bytes_read.sum + write.sum)",
            "algorithmic_bytes": out_bytes,
            "algorithmic_bytes_what": "G and H of the periodic domain written (the kernels' only DRAM output; "
                                      "inputs are L2-resident)",
            "peak_source": "of measured: cuBLAS DGEMM 8192^3 in this run (nominal %.1f TFLOP/s)" % FP64_NOMINAL_TFLOPS,
            "fp64_pipe_frac_ncu": pipe,
            "work": "%.3e lattice terms x %.0f FP64 ops per launch" % (terms_reg, C_TERM_FLOPS),
            "mean_terms_per_point": cnt[0] / max(cnt[3], 1)}


def sweep_instances(freqs, dirs, n=16, a=0.8):
    """Config-2 style sweep: the 1536-quad (n = 16) sphere of radius 0.3 in the
    square lattice of period a, k a in [1.2, 2.4] (freqs values), theta uniform
    in [0, 60] deg (dirs values; 0 becomes the reference's tiny tilt), phi = 0
    (the reference rejects ky = 0: phi = 1e-6 deg); an instance within 2% of a
    Rayleigh anomaly is left out.  Returns [(frequency index, meshgen args)]."""
    import math
    out = []
    for fi, ka in enumerate(np.linspace(1.2, 2.4, freqs)):
        k = ka / a
        g = 2 * math.pi / a
        for th in np.linspace(0.0, 60.0, dirs):
            th = max(float(th), 1e-6)
            kx = k * math.sin(math.radians(th))
            if any(abs(math.hypot(kx + i * g, j * g) - k) < 0.02 * k for i in range(-6, 7) for j in range(-6, 7)):
                continue
            out.append((fi, dict(n=n, semi_axes=(0.3, 0.3, 0.3), lattice=((a, 0.0), (0.0, a)), theta_deg=th,
                                 phi_deg=1e-6, wavelength=2 * math.pi / k)))
    return out


def run_sweep(args, rank, world):
    """Batched sweep (config 2, reduced to --sweep-freqs x --sweep-dirs
    instances): one context solves the instances in frequency order, so that
    instances at the same frequency keep the free-space domain's matrices and
    dpv factors (bemgpu_interior_reuses); FP64, then the mixed form, with the
    mixed form's force error against FP64 per instance; then the mixed form
    with one batch per frequency (bemgpu_batch_load / _assemble / _select),
    its forces against the unbatched ones."""
    import ctypes
    from bem3_aw_qd2_b200 import api, meshgen
    h, g = api.libs()
    h.aqd2_set_verbose(0)
    g.bemgpu_load.argtypes = [ctypes.c_void_p, ctypes.POINTER(api.Problem)]
    g.bemgpu_interior_reuses.argtypes = [ctypes.c_void_p]
    g.bemgpu_interior_reuses.restype = ctypes.c_longlong
    inst = sweep_instances(args.sweep_freqs, args.sweep_dirs, n=args.sweep_mesh_n)
    cases = [api.Case.from_files(*meshgen.write_inputs(tempfile.mkdtemp(prefix="sweep_"), **r)) for _, r in inst]
    probs = [c.problem() for c in cases]
    ctx = ctypes.c_void_p()
    if g.bemgpu_create(0, None, ctypes.byref(ctx)) != 0:
        raise RuntimeError("bemgpu_create failed")
    rc3 = np.zeros(3)
    res = {}
    for tag, prec in (("fp64", 0), ("mixed", args.mixed_mode or 2)):
        g.bemgpu_set_precision(ctx, prec)
        # warm-up: the first instance (kernels loaded, graphs captured)
        g.bemgpu_load(ctx, ctypes.byref(probs[0]))
        g.bemgpu_run(ctx)
        g.bemgpu_sync(ctx)
        r0 = g.bemgpu_interior_reuses(ctx)
        F = []
        t0 = time.perf_counter()
        for p in probs:
            if g.bemgpu_load(ctx, ctypes.byref(p)) or g.bemgpu_run(ctx):
                raise RuntimeError(g.bemgpu_error(ctx).decode())
            Fv, Nv = np.zeros(3), np.zeros(3)
            g.bemgpu_force(ctx, 0, api._p(rc3), api._p(Fv), api._p(Nv))
            F.append(Fv)
        g.bemgpu_sync(ctx)
        el = time.perf_counter() - t0
        res[tag] = {"value": len(probs) / el, "unit": "solves/s", "seconds": el,
                    "interior_reuses": int(g.bemgpu_interior_reuses(ctx) - r0), "F": F}
        if prec:
            res[tag]["mode"] = {1: "FP32", 2: "TF32", 3: "TF32x3", 4: "TF32"}.get(g.bemgpu_get_precision(ctx), "?")
    errs = [float(np.linalg.norm(a - b) / np.linalg.norm(b)) for a, b in zip(res["mixed"]["F"], res["fp64"]["F"])]
    # the mixed form again, one batch per frequency (bemgpu_batch_*): the
    # interior domains once, the periodic domain of all the frequency's
    # directions with each kernel launched once, then a solve per instance
    PP = ctypes.POINTER(api.Problem)
    g.bemgpu_batch_load.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(PP)]
    g.bemgpu_batch_assemble.argtypes = [ctypes.c_void_p]
    g.bemgpu_batch_select.argtypes = [ctypes.c_void_p, ctypes.c_int]
    groups = {}
    for i, (fi, _) in enumerate(inst):
        groups.setdefault(fi, []).append(i)

    def batch_pass(sel):
        Fb = {}
        for fi, idx in sel.items():
            arr = (PP * len(idx))(*[ctypes.pointer(probs[i]) for i in idx])
            if g.bemgpu_batch_load(ctx, len(idx), arr) or g.bemgpu_batch_assemble(ctx):
                raise RuntimeError(g.bemgpu_error(ctx).decode())
            for j, i in enumerate(idx):
                if g.bemgpu_batch_select(ctx, j) or g.bemgpu_solve(ctx):
                    raise RuntimeError(g.bemgpu_error(ctx).decode())
                Fv, Nv = np.zeros(3), np.zeros(3)
                g.bemgpu_force(ctx, 0, api._p(rc3), api._p(Fv), api._p(Nv))
                Fb[i] = Fv
        g.bemgpu_sync(ctx)
        return Fb
    g.bemgpu_set_precision(ctx, args.mixed_mode or 2)
    batch_pass({0: [0]})  # warm-up: the batched kernels' first launch
    t0 = time.perf_counter()
    Fb = batch_pass(groups)
    el = time.perf_counter() - t0
    res["mixed_batched"] = {"value": len(probs) / el, "unit": "solves/s", "seconds": el,
                            "batches": len(groups), "instances_per_batch": [len(v) for v in groups.values()],
                            "force_rel_diff_vs_unbatched": max(float(np.linalg.norm(Fb[i] - res["mixed"]["F"][i])
                                                                     / np.linalg.norm(res["mixed"]["F"][i]))
                                                               for i in range(len(probs)))}
    for tag in ("fp64", "mixed"):
        del res[tag]["F"]
    g.bemgpu_destroy(ctx)
    for c, p in zip(cases, probs):
        c.free_problem(p)
        c.close()
    v = res["mixed"]["value"]
    line = {"metric": "solves/s", "value": v, "unit": "solves/s", "n_gpus": 1, "steps": len(probs), "warmup": 1,
            "ms_per_step": 1000.0 / v, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 assembly, complex-FP32 LU + FP64 refinement", "data": "synthetic",
            "config": {"workload": "sweep", "instances": len(probs), "frequencies": args.sweep_freqs,
                       "directions": args.sweep_dirs, "full_sweep": "64 directions x 8 frequencies (reduced here)",
                       "mesh": "%d-quad cube-sphere r = 0.3, square lattice 0.8" % (6 * args.sweep_mesh_n ** 2),
                       "order": "frequency-major: instances at one frequency share the interior domain"},
            "fp64": res["fp64"], "mixed": res["mixed"], "mixed_batched": res["mixed_batched"],
            "force_rel_err_mixed_vs_fp64": {"max": max(errs), "median": float(np.median(errs))}}
    if rank == 0:
        print(json.dumps(line))


def run_lu(args, rank, world):
    """The device LU alone (bem_lu.cu): factorisation and one-right-hand-side
    solve of a seeded random complex matrix (diagonally heavy, rows permuted
    so that every panel moves rows), by order and arithmetic, CUDA events on
    the factorisation's stream, best of --steps after --warmup; the relative
    residual ||A x - b|| / (||A|| ||x||) checks each result."""
    import ctypes
    import torch
    from bem3_aw_qd2_b200 import api
    _, g = api.libs()
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    vp = ctypes.c_void_p
    g.bem_lu_init.argtypes = [vp, ctypes.c_int]
    g.bem_lu_free.argtypes = [vp]
    for p in ("z", "c"):
        getattr(g, "bem_lu_factor_" + p).argtypes = [vp, vp, ctypes.c_int, vp]
        getattr(g, "bem_lu_solve_" + p).argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, vp, vp]
    g.bem_lu_status.argtypes = [vp, vp]
    g.bem_lu_status.restype = ctypes.c_uint
    g.bem_lu_attach_tc.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    g.bem_lu_detach_tc.argtypes = [vp]
    st = torch.cuda.Stream()
    out = []
    for arith in args.lu_arith.split(","):
        for n in [int(x) for x in args.lu_sizes.split(",")]:
            w = ctypes.create_string_buffer(4096)
            wp = ctypes.addressof(w)
            if g.bem_lu_init(wp, 0) != 0:
                raise RuntimeError("bem_lu_init failed")
            if arith.startswith("t") and g.bem_lu_attach_tc(wp, n, int(arith[1])) != 0:
                raise RuntimeError("tensor-core update buffers")
            dt = torch.complex128 if arith == "z" else torch.complex64
            gen = torch.Generator(device="cuda").manual_seed(n)
            A0 = torch.randn(n, n, dtype=dt, device="cuda", generator=gen) / n ** 0.5
            A0 += (1.5 + 0.5j) * torch.eye(n, dtype=dt, device="cuda")
            A0 = A0[torch.randperm(n, generator=gen, device="cuda")]
            B0 = torch.randn(1, n, dtype=dt, device="cuda", generator=gen)
            A = A0.clone()
            torch.cuda.synchronize()  # the inputs (default stream) before st copies them
            p = "z" if arith == "z" else "c"
            fac, sol = getattr(g, "bem_lu_factor_" + p), getattr(g, "bem_lu_solve_" + p)
            tf, ts = [], []
            with torch.cuda.stream(st):
                for r in range(args.warmup + args.steps):
                    A.copy_(A0)
                    B = B0.clone()
                    e0, e1, e2 = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
                    e0.record(st)
                    if fac(wp, A.data_ptr(), n, st.cuda_stream) != 0:
                        raise RuntimeError("factorisation failed")
                    e1.record(st)
                    if sol(wp, A.data_ptr(), n, 1, B.data_ptr(), st.cuda_stream) != 0:
                        raise RuntimeError("solve failed")
                    e2.record(st)
                    e2.synchronize()
                    if r >= args.warmup:
                        tf.append(e0.elapsed_time(e1))
                        ts.append(e1.elapsed_time(e2))
            status = g.bem_lu_status(wp, st.cuda_stream)
            x = B[0].to(torch.complex128)
            Ad, bd = A0.to(torch.complex128), B0[0].to(torch.complex128)
            res = float(torch.linalg.vector_norm(Ad @ x - bd) /
                        (torch.linalg.matrix_norm(Ad) * torch.linalg.vector_norm(x)))
            g.bem_lu_detach_tc(wp)
            g.bem_lu_free(wp)
            del A, A0, Ad
            torch.cuda.empty_cache()
            out.append({"n": n, "arith": arith, "factor_ms": min(tf), "solve_ms": min(ts),
                        "tflops": 8.0 / 3.0 * n ** 3 / (min(tf) / 1e3) / 1e12, "rel_residual": res,
                        "status": int(status)})
    if rank == 0:
        print(json.dumps({"metric": "complex LU factorisation time", "unit": "ms", "workload": "lu",
                          "higher_is_better": False, "steps": args.steps, "warmup": args.warmup,
                          "data": "synthetic: seeded random complex matrices, (1.5 + 0.5i) I + N(0, 1/n), rows "
                                  "permuted", "tflops_count": "8/3 n^3 real flop per complex LU",
                          "results": out}))


def workload_desc(name):
    from bem3_aw_qd2_b200 import meshgen
    return {**meshgen.describe(name), "media": "host rho 1000 c 1500 (wavelength 1); body rho 1200 c 2250",
            "l2": "256 MB flush between timed steps"}


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference" and args.workload != "stream":
        return run_reference(args, rank, world)
    if args.workload == "lu":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference's dense solves are timed inside "
                                                                  "its full-solve line (sphere216)"}))
            return
        return run_lu(args, rank, world)
    if args.workload == "sweep":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the sweep's reference time is the sphere1536 "
                                                                  "reference line times the instance count"}))
            return
        return run_sweep(args, rank, world)
    if args.workload == "stream":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no request server; its per-solve "
                                                                  "time is the sphere216 reference line"}))
            return
        return run_stream(args, rank, world)
    from bem3_aw_qd2_b200 import api
    api.libs()
    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    from bem3_aw_qd2_b200 import api, meshgen, replicas
    h, g = api.libs()
    h.aqd2_set_device(local)
    h.aqd2_set_verbose(0)
    d = tempfile.mkdtemp(prefix="bench_")
    files = meshgen.write_inputs(d, **meshgen.CONFIGS[args.workload])
    # the mixed form's FP32 factors beside the FP64 matrices: when that does
    # not fit the device, the interior derivative rows are recomputed in
    # blocks instead of kept (bemgpu_set_interior_derivatives), for both forms
    desc = meshgen.describe(args.workload)
    n_glob, n_dom = desc["unknowns"], 4 * desc["elements"]
    need = 16 * n_glob ** 2 + 2 * 48 * n_dom ** 2 + 64 * n_dom ** 2
    if args.mixed_mode:
        need += 8 * n_glob ** 2 + 16 * n_dom ** 2
    keep_dgh = 0 if need > 0.85 * torch.cuda.get_device_properties(local).total_memory else 1
    h.aqd2_set_interior_derivatives(keep_dgh)
    case = api.Case.from_files(*files)
    case.solve()  # creates the device context, uploads, first solve
    ctx = case.ctx
    # every step assembles and factors every domain, as the reference does
    # (no interior-domain reuse across the repeated solves of one problem)
    g.bemgpu_set_interior_reuse(ctx, 0)
    stream = torch.cuda.ExternalStream(int(g.bemgpu_stream(ctx)))
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    ewald_scale = case.autotune()  # Ewald parameter for this problem (kept for every later solve)
    fp64_peak = measured_fp64_peak()
    g.bemgpu_set_profiling(ctx, 1)
    rc = np.zeros(3)
    F = np.zeros(3)
    N = np.zeros(3)
    _d = api._d

    def device_step():
        if g.bemgpu_run(ctx) != 0:
            raise RuntimeError(g.bemgpu_error(ctx).decode())
        if g.bemgpu_force(ctx, 0, api._p(rc), api._p(F), api._p(N)) != 0:
            raise RuntimeError(g.bemgpu_error(ctx).decode())

    for _ in range(args.warmup):
        with torch.cuda.stream(stream):
            flush.zero_()
        device_step()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    times, phases = [], []
    g.bemgpu_work_counters(ctx, (api.ctypes.c_ulonglong * 6)(), 1)
    launches0 = g.bemgpu_kernel_launches()
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        device_step()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
        ph = (api.ctypes.c_double * 16)()
        n = g.bemgpu_phase_times(ctx, ph, 16)
        phases.append([ph[i] for i in range(n)])
    torch.cuda.synchronize()
    launches = g.bemgpu_kernel_launches() - launches0
    cnt = (api.ctypes.c_ulonglong * 6)()
    g.bemgpu_work_counters(ctx, cnt, 1)
    total_ms = sum(times)
    F_fp64, N_fp64 = F.copy(), N.copy()
    ne = meshgen.describe(args.workload)["elements"]
    sol_fp64 = [case.solution(dd, ne) for dd in (0, 1)]
    mixed = None
    if args.mixed_mode:
        # the mixed-precision form on the same workload: FP32 LU (tensor-core
        # trailing updates) + FP64 refinement, force checked against FP64
        case.set_precision(args.mixed_mode)
        for _ in range(args.warmup):
            with torch.cuda.stream(stream):
                flush.zero_()
            device_step()
        torch.cuda.synchronize()
        mt, mph = [], []
        for step in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            if args.profile_mixed and step == 0:
                torch.cuda.cudart().cudaProfilerStart()
            device_step()
            e1.record(stream)
            e1.synchronize()
            if args.profile_mixed and step == 0:
                torch.cuda.cudart().cudaProfilerStop()
            mt.append(e0.elapsed_time(e1))
            ph = (api.ctypes.c_double * 16)()
            k = g.bemgpu_phase_times(ctx, ph, 16)
            mph.append([ph[i] for i in range(k)])
        it, rcorr, fb = case.solve_stats()
        eff_mode = case.precision()
        # surface coefficients P, dP, pv, dpv of both domains against the FP64 path
        sol_m = [case.solution(dd, ne) for dd in (0, 1)]
        coef_err = max(float(np.max(np.abs(a - b)) / np.max(np.abs(b)))
                       for sm, s6 in zip(sol_m, sol_fp64) for a, b in zip(sm, s6))
        F1m, N1m = case.force(1)
        case.set_precision(0)
        case.run_device()
        F1d, N1d = case.force(1)
        mp = np.array(mph).mean(axis=0)
        mixed = {"value": args.steps / (sum(mt) / 1000.0), "unit": "solves/s",
                 "mode": {1: "FP32", 2: "TF32", 3: "TF32x3", 4: "TF32"}[eff_mode] + " LU updates + FP64 refinement",
                 "latency_ms": {"p50": float(np.percentile(mt, 50)), "p99": float(np.percentile(mt, 99))},
                 "force_rel_err_vs_fp64": {"type0": float(np.linalg.norm(F - F_fp64) / np.linalg.norm(F_fp64)),
                                           "type1": float(np.linalg.norm(F1m - F1d) / np.linalg.norm(F1d))},
                 "surface_coef_rel_err_vs_fp64": coef_err,
                 "refine_iters": [int(x) for x in it], "refine_rel_corr": [float(x) for x in rcorr],
                 "fp64_fallbacks": int(np.sum(fb)),
                 "lu_solve_ms": float(mp[11]) if len(mp) > 11 else None,
                 "dpv_solves_ms": float(mp[13]) if len(mp) > 13 else None}
    # e2e: the public drop-in API with host buffers
    e2e_times = []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        case.solve()
        Fh, Nh = case.force(0)
        e2e_times.append(time.perf_counter() - t0)
    clk = clocks.stop()
    (total_ms, e2e_total), _ = replicas.reduce_timing([total_ms, sum(e2e_times)], [],
                                                      device="cuda" if world > 1 else "cpu")
    ms_per_step = total_ms / args.steps
    value = world * args.steps / (total_ms / 1000.0)
    e2e_value = world * args.steps / e2e_total
    ph = np.array(phases).mean(axis=0)
    names = ["d0_classify", "d0_regular", "d0_near", "d0_self", "d0_diag", "d1_classify", "d1_regular", "d1_near",
             "d1_self", "d1_diag", "gather", "lu_solve", "boundary_values", "dpv_solves"]
    phase_ms = {names[i]: float(ph[i]) for i in range(min(len(names), len(ph)))}
    terms_reg = cnt[0] / args.steps
    t_reg = phase_ms.get("d0_regular", float("nan")) / 1000.0
    achieved = terms_reg * C_TERM_FLOPS / t_reg / 1e12 if t_reg > 0 else None
    h2d = ne * (12 + 9 + 12 + 12 + 8 + 8 + 8 + 24 + 2) * 8 + ne * (1 + 4 + 1 + 2 + 8) * 4 + ne
    d2h = 2 * (4 * ne) * (2 + 2 + 6 + 6) * 8 + 48 + 4
    lat = sorted(times)
    out = {
        "metric": "solves/s", "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "precision": "plain FP64 (assembly and LU)",
                   "ewald_scale": ewald_scale, "interior_derivative_rows": "kept" if keep_dgh else "recomputed in blocks",
                   "regular_pairs_by_rule": dict(zip(["12x12 (reference)", "10x10", "9x9", "8x8", "7x7", "6x6"],
                                                     case.rule_pairs() or [])),
                   **workload_desc(args.workload)},
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
        "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "path": "solve_bieq_aqd2 + force_FN_aqd2 (C ABI, host buffers)"},
        "phase_ms": phase_ms,
        "roofline": roofline_record(achieved, fp64_peak, terms_reg, cnt, args.workload, 2 * 16 * n_dom ** 2),
        "clocks": clk,
        "mixed": mixed,
        "gpu_launches": int(launches),
    }
    if rank == 0 and world == 1 and args.stream_requests > 0 and args.workload == "sphere216":
        # the headline metric on one GPU: the config-4 request stream, served
        # mixed precision against the plain FP64 drop-in path
        case.close()
        torch.cuda.empty_cache()
        out["stream"] = stream_compare(args.stream_requests, 200.0, args.slots, args.hbm_gb, args.mixed_mode or 2,
                                       device=local)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(files, args.cpu_seconds)
    if rank == 0:
        print(json.dumps(out))
    case.close()
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
