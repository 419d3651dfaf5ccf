"""ALS benchmark: sec/iteration and GFLOP/s at f=100 on the Netflix-shaped
synthetic matrix (480,189 x 17,770, ~99.1M training ratings, 1.4M test).

One step = one full ALS iteration (user half-step, then item half-step) over
the resident matrix. GFLOP/s uses the solver-independent formula
    FLOP_iter = sum_sides nnz*f*(f+1) + 2*nnz*f + rows*(f^3/3 + 2 f^2).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

Engine arm: inputs resident in HBM, CUDA events on the model's stream, max
over ranks; e2e through the Spark JNI entry's host-buffer half-step
(als_half_step_host: CSR upload, theta upload and X download inside the timed
region, the uploads overlapped range by range with the solve).
Reference arm: the reference has no CPU ALS (its CPU path is Spark's JVM ALS,
absent here), so it times the CPU port of the same half-step (oracle FP32) on
bounded seeded row samples with all host threads, scaled by the formula.
With N > 1 ranks, rows are sharded by nnz and each half-step ends with an
all-gather of the updated factor rows: the engine's C++ shard driver
(als_shard_*, NCCL), its communicator id handed out over torch.distributed.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [ROOT, os.path.join(ROOT, "cuda-mllib_b200")]

METRIC = "ALS sec/iter & GFLOP/s at f=100, test RMSE within 0.1% of FP64 oracle"
WORKLOAD = "netflix-shape synthetic 480189x17770, ~100.5M ratings (1.4M test), f=100, lambda=0.05"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="engine", choices=["engine", "reference"])
    p.add_argument("--config", default="netflix")
    p.add_argument("--scale", type=float, default=1.0, help="shrink m, n (nnz by scale^2)")
    p.add_argument("--row-scale", type=float, default=1.0, help="shrink m and nnz, keep n")
    p.add_argument("--precision", default="bf16", choices=["fp32", "bf16", "fp16"])
    p.add_argument("--solver", default="cg", choices=["cholesky", "cg"])
    p.add_argument("--warm", default="previous", choices=["zero", "previous", "mlp"],
                   help="CG starting point")
    p.add_argument("--jacobi", action="store_true", help="diagonal-preconditioned CG")
    p.add_argument("--graph", action="store_true",
                   help="time the iteration as one CUDA graph replay (users + items launches)")
    p.add_argument("--seed", type=int, default=1)
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-forms", action="store_true",
                   help="skip timing the FP32 Cholesky and learned-start forms beside the default")
    p.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU sample time")
    return p.parse_args()


def cfg_of(args, A=None):
    if A is None:
        import als_data as A
    if args.row_scale != 1.0:
        return A.row_scaled_config(args.config, args.row_scale)
    return A.scaled_config(args.config, args.scale) if args.scale != 1.0 else dict(A.CONFIGS[args.config])


def workload_name(args):
    if args.config == "netflix" and args.scale == 1.0 and args.row_scale == 1.0:
        return WORKLOAD
    if args.row_scale != 1.0:
        return f"{args.config} rows x{args.row_scale}"
    return f"{args.config} x{args.scale}" if args.scale != 1.0 else args.config


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return d["hbm_gbs"], d["bf16_tflops"], d.get("bf16_tflops_sustained", d["bf16_tflops"]), "measured"
    except Exception:
        return 6650.0, 1590.0, 1400.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=self.tmp, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        # wait until the sampler is live; lines written before the timed
        # region starts are left out of the summary
        self.skip = 0
        t0 = time.time()
        while self.proc and time.time() - t0 < 15:
            try:
                n = len(open(self.tmp.name).read().strip().splitlines())
            except OSError:
                n = 0
            if n:
                self.skip = n
                break
            time.sleep(0.05)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        try:
            lines = open(self.tmp.name).read().strip().splitlines()
            os.unlink(self.tmp.name)
        except Exception:
            return None
        in_region = len(lines) - self.skip
        rows = [l.split(",") for l in (lines[self.skip:] if in_region > 0 else lines[-1:])]
        rows = [[x.strip() for x in r] for r in rows if len(r) >= 9]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        load = sorted(sm)[len(sm) // 2:] if sm else []
        return {"sm_mhz": float(np.median(load)) if load else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows),
                "samples_in_timed_region": max(0, in_region)}


def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return world, rank, local


# ---------------------------------------------------------------------------
# CPU port on bounded samples (reference arm and cpu_baseline leg)
# ---------------------------------------------------------------------------

def _sample_rows(ptr, idx, val, rows):
    sub_ptr = np.zeros(len(rows) + 1, np.int64)
    sub_ptr[1:] = np.cumsum(ptr[rows + 1] - ptr[rows])
    take = np.concatenate([np.arange(ptr[u], ptr[u + 1]) for u in rows]) if len(rows) else np.zeros(0, np.int64)
    return sub_ptr, idx[take], val[take]


def cpu_port_step(r, f, lam, users, items, X, T):
    """One sampled CPU iteration: the sampled users from T, the sampled items
    from X. Returns (seconds, algorithmic FLOPs of the sampled rows)."""
    import oracle as O
    up, uc, uv = _sample_rows(r.csr_ptr, r.csr_col, r.csr_val, users)
    ip, ir, iv = _sample_rows(r.csc_ptr, r.csc_row, r.csc_val, items)
    t0 = time.perf_counter()
    O.half_step_f32(up, uc, uv, T, lam)
    O.half_step_f32(ip, ir, iv, X, lam)
    dt = time.perf_counter() - t0
    nnz = up[-1] + ip[-1]
    flops = nnz * f * (f + 1) + 2 * nnz * f + (len(users) + len(items)) * (f ** 3 / 3 + 2 * f * f)
    return dt, flops


def cpu_sample_plan(r, f, lam, seconds, seed):
    """Seeded user/item samples sized so one sampled iteration takes about
    `seconds` on this host (the two sides in their full-matrix proportion)."""
    rng = np.random.default_rng(seed)
    X = np.random.default_rng(seed + 1).standard_normal((r.m, f)).astype(np.float32) * f ** -0.5
    T = np.random.default_rng(seed + 2).standard_normal((r.n, f)).astype(np.float32) * f ** -0.5
    frac = min(1.0, 2000.0 / r.m)
    while True:
        users = np.sort(rng.choice(r.m, max(1, int(r.m * frac)), replace=False))
        items = np.sort(rng.choice(r.n, max(1, int(r.n * frac)), replace=False))
        dt, _ = cpu_port_step(r, f, lam, users, items, X, T)
        if dt >= 0.25 * seconds or frac >= 1.0:
            break
        frac = min(1.0, frac * min(8.0, max(1.5, seconds / max(dt, 1e-3))))
    if dt < seconds and frac < 1.0:
        frac = min(1.0, frac * seconds / max(dt, 1e-3))
        users = np.sort(rng.choice(r.m, max(1, int(r.m * frac)), replace=False))
        items = np.sort(rng.choice(r.n, max(1, int(r.n * frac)), replace=False))
    return users, items, X, T, frac


def run_reference(args):
    world, rank = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import als_data as D  # host-only data generator: no GPU library is loaded on this arm
    cfg = cfg_of(args, D)
    f, lam = cfg["f"], cfg["lam"]
    r = D.synth(cfg, seed=args.seed)
    per_step = max(2.0, min(args.cpu_seconds, 150.0 / max(1, args.steps + args.warmup)))
    users, items, X, T, frac = cpu_sample_plan(r, f, lam, per_step, args.seed)
    for _ in range(args.warmup):
        cpu_port_step(r, f, lam, users, items, X, T)
    secs, flops = [], 0.0
    for _ in range(args.steps):
        dt, fl = cpu_port_step(r, f, lam, users, items, X, T)
        secs.append(dt)
        flops = fl
    gflops = flops / np.median(secs) / 1e9
    full = D.flop_per_iteration(r, f)
    cores = os.cpu_count()
    sample = (f"seeded {len(users)} of {r.m} user rows + {len(items)} of {r.n} item rows per step "
              f"({frac:.2%} of rows), FP32 port of the half-step, {cores} threads")
    line = {"metric": METRIC, "value": round(gflops, 3), "unit": "GFLOP/s", "impl": "reference",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(full / (gflops * 1e9) * 1e3, 3),
            "sec_per_iter": round(full / (gflops * 1e9), 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
            "config": {"workload": workload_name(args),
                       "f": f, "lambda": lam, "m": r.m, "n": r.n, "nnz_train": r.nnz},
            "cpu_baseline": {"value": round(gflops, 3), "unit": "GFLOP/s", "cores": cores,
                             "kind": "port", "sample": sample},
            "e2e": {"value": round(gflops, 3), "unit": "GFLOP/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "note": "the reference's CPU ALS is Spark's JVM implementation (not in the reference, "
                    "no JVM here); timed instead: the C restatement of the same half-step"}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# engine arm
# ---------------------------------------------------------------------------

# Per-launch DRAM traffic of the rows kernel at the default workload (the
# Netflix shape, BF16 CG, previous iterate), from one ncu capture of the same
# command at full size (dram__bytes_read.sum + dram__bytes_write.sum, one pass;
# profiles/rows_tc_ws_netflix_dram.txt): the mean of the users launch (1.468 GB)
# and the items launch (3.349 GB). None for other workloads.
DRAM_PER_LAUNCH = 2.408e9
DRAM_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum, full-size workload, 4th iteration: "
               "users 1.468e9, items 3.349e9 bytes")

FIXTURE = os.path.join(ROOT, "tests", "golden", "netflix_f100_fp64.npz")
RESTART = 10  # iterations of one training run (the workload's iteration count)


def fp64_reference_rmse(args, iters):
    """Test RMSE of FP64 ALS (the oracle) after `iters` iterations from the same
    seeded theta0, from the committed fixture; None when the workload is not
    the one the fixture holds."""
    if not (args.config == "netflix" and args.scale == 1.0 and args.row_scale == 1.0 and
            args.seed == 1 and os.path.exists(FIXTURE)):
        return None
    z = np.load(FIXTURE)
    if iters < 1 or iters > len(z["rmse_fp64"]):
        return None
    return float(z["rmse_fp64"][iters - 1])


def run_engine(args):
    import torch
    import als_b200 as A

    world, rank, local = dist_init(args)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    cfg = cfg_of(args)
    f, lam = cfg["f"], cfg["lam"]
    t0 = time.perf_counter()
    r = A.synth(cfg, seed=args.seed)
    gen_s = time.perf_counter() - t0
    prec = {"fp32": A.PREC_FP32, "bf16": A.PREC_BF16, "fp16": A.PREC_FP16}[args.precision]
    solver = {"cholesky": A.SOLVER_CHOLESKY, "cg": A.SOLVER_CG}[args.solver]
    warm = {"zero": A.WARM_ZERO, "previous": A.WARM_PREVIOUS, "mlp": A.WARM_MLP}[args.warm]
    opts = A.options(precision=prec, solver=solver, warm_start=warm,
                     cg_jacobi=1 if args.jacobi else 0, use_graph=1 if args.graph else 0)
    graph = args.graph and args.warm != "mlp" and world == 1
    stream = torch.cuda.Stream(device=dev)
    th0 = A.init_factors(r.n, f, args.seed + 100)
    th0_dev = torch.from_numpy(th0).to(dev)
    x_zero = torch.zeros((r.m, f), dtype=torch.float32, device=dev)
    with torch.cuda.stream(stream):
        model = A.Model(r, f, opts, stream=stream, theta0=th0)
    shard = None
    if world > 1:
        import torch.distributed as dist
        nid = torch.zeros(128, dtype=torch.uint8, device=dev)
        if rank == 0:
            nid.copy_(torch.frombuffer(bytearray(A.shard_unique_id()), dtype=torch.uint8))
        dist.broadcast(nid, 0)
        shard = A.Shard(model, r, world, rank, bytes(nid.cpu().tolist()))

    def restart(M):
        # a fresh training run: theta0 and X = 0, as a newly created model has
        M.set_theta(th0_dev)
        M.set_x(x_zero)

    def iteration(M, ev=None):
        # one launch of the fused rows kernel per half-step
        if ev is not None:
            ev[0].record(stream)
        if graph and M is model and ev is not None:
            M.iterate(lam, 1)  # replay of the captured users + items launches
            ev[1].record(stream)
            ev[2].record(stream)
            return
        M.half_step(A.SIDE_USERS, lam)
        if shard and M is model:
            shard.exchange(A.SIDE_USERS)
        if ev is not None:
            ev[1].record(stream)
        M.half_step(A.SIDE_ITEMS, lam)
        if shard and M is model:
            shard.exchange(A.SIDE_ITEMS)
        if ev is not None:
            ev[2].record(stream)

    # Step k runs iteration (k mod 10) + 1 of a training run restarted every 10
    # steps (theta0, X = 0), so the timed steps are the iterations of full
    # 10-iteration runs, the first (CG from zero) included, rather than ever
    # later iterations whose warm starts keep improving.
    restarts_timed = 0
    for k in range(args.warmup):
        if k % RESTART == 0:
            restart(model)
        iteration(model)
    if graph:
        model.iterate(lam, 1)  # capture (after the warm-up has tuned both sides) and replay once
        restart(model)
    torch.cuda.synchronize(dev)
    model.stats(reset=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    with Clocks(local) as ck:
        torch.cuda.synchronize(dev)
        for k in range(args.steps):
            if (args.warmup + k) % RESTART == 0:
                restart(model)  # outside the step's events
                restarts_timed += 1
            iteration(model, evs[k])
        torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    users_ms = np.array([e[0].elapsed_time(e[1]) for e in evs])
    items_ms = np.array([e[1].elapsed_time(e[2]) for e in evs])
    if graph:
        # one graph replay per step: the two launches are not timed apart
        users_ms = items_ms = (users_ms + items_ms) / 2
    print("per-step users ms", np.round(users_ms, 2).tolist(), "items ms",
          np.round(items_ms, 2).tolist(), file=sys.stderr)
    step_ms = users_ms + items_ms
    total_ms = float(step_ms.sum())
    if world > 1:
        t = torch.tensor([total_ms, float(np.median(step_ms))], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms, med_ms = float(t[0]), float(t[1])
    else:
        med_ms = float(np.median(step_ms))
    stats = model.stats()
    flop_iter = A.flop_per_iteration(r, f)
    gflops = flop_iter * args.steps / (total_ms / 1e3) / 1e9
    # launches of this library's kernels in the timed region: one rows kernel
    # per half-step, two factor conversions per restart; with the learned warm
    # start also the features pass and three MLP GEMMs per inference chunk of
    # 32,768 rows
    launches_per_step = 2
    if args.warm == "mlp":
        launches_per_step += 2 + 3 * (-(-r.m // 32768) + -(-r.n // 32768))
    launches = launches_per_step * args.steps + 2 * restarts_timed

    # Roofline of the dominant kernel, the fused rows kernel (one launch per
    # half-step): its hermitian is a tensor-core SYRK, nnz * f * (f + 1) FLOPs
    # per launch (the unique half, 2 FLOPs per multiply-add), over the measured
    # dense bf16 peak for a kernel timed alone (the burst figure: each launch
    # lasts milliseconds). achieved = that work / the mean launch time.
    hbm, tf_burst, tf_sust, src = peaks()
    s_el = 4 if args.precision == "fp32" else 2
    syrk = r.nnz * f * (f + 1)
    mean_launch_s = float(np.concatenate([users_ms, items_ms]).mean()) / 1e3
    tflops = syrk / mean_launch_s / 1e12
    u_tf = syrk / (float(users_ms.mean()) / 1e3) / 1e12
    i_tf = syrk / (float(items_ms.mean()) / 1e3) / 1e12
    # beside it: the bytes the gather moves from L2 into shared memory (the
    # factor rows are L2-resident: DRAM carries the CSR stream and the writes)
    gather_bytes = lambda nnz, rows: nnz * (8 + f * s_el) + rows * (8 + 8 * f + f * s_el)
    workload_default = (args.config == "netflix" and args.scale == 1.0 and args.row_scale == 1.0 and
                        args.precision == "bf16" and args.solver == "cg" and args.warm == "previous")
    traffic = DRAM_PER_LAUNCH if workload_default else None
    roof = {"bound": "tensor", "achieved": round(tflops, 2), "peak": tf_burst, "unit": "TFLOP/s",
            "frac": round(tflops / tf_burst, 4), "traffic": traffic,
            "traffic_source": DRAM_SOURCE if traffic else None,
            "peak_kind": f"{src} dense bf16 (burst; sustained {tf_sust})",
            "kernel": "rows kernel (gather + tensor-core hermitian + solve), mean of the two launches",
            "flops_per_launch": syrk, "flops_formula": "nnz*f*(f+1) (SYRK, unique half)",
            "users_launch": {"ms": round(float(users_ms.mean()), 3), "achieved": round(u_tf, 2),
                             "frac": round(u_tf / tf_burst, 4)},
            "items_launch": {"ms": round(float(items_ms.mean()), 3), "achieved": round(i_tf, 2),
                             "frac": round(i_tf / tf_burst, 4)},
            "l2_gather": {"bytes_per_launch": round((gather_bytes(r.nnz, r.m) + gather_bytes(r.nnz, r.n)) / 2),
                          "formula": "nnz*(8+f*s) + rows*(8+8f+f*s)",
                          "gbs": round((gather_bytes(r.nnz, r.m) + gather_bytes(r.nnz, r.n)) / 2
                                       / mean_launch_s / 1e9, 1),
                          "note": "factor rows come from L2 (Netflix X in BF16 is 96 MB), so this is "
                                  "an L2-to-SM figure, not an HBM one"},
            "hbm_peak_gbs": hbm}

    line = None
    if rank == 0:
        ck_sum = ck.summary()
        line = {"metric": METRIC, "value": round(gflops, 2), "unit": "GFLOP/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 3),
                "sec_per_iter": round(med_ms / 1e3, 5), "higher_is_better": True,
                "scaling": "strong" if world > 1 else "weak", "vs_baseline": None,
                "dtype": args.precision, "data": "synthetic",
                "config": {"workload": workload_name(args),
                           "f": f, "lambda": lam, "m": r.m, "n": r.n, "nnz_train": r.nnz,
                           "n_test": int(len(r.test_r)), "precision": args.precision,
                           "solver": args.solver, "warm_start": args.warm,
                           "cg_jacobi": args.jacobi, "seed": args.seed,
                           "cuda_graph": bool(graph),
                           "steps_are": f"iterations of {RESTART}-iteration runs: step k runs iteration "
                                        f"(k mod {RESTART}) + 1 of a run restarted from theta0, X = 0",
                           "l2": "inputs larger than L2 (CSR+CSC %.2f GB per iteration)" % (
                               (r.nnz * 16 + (r.m + r.n) * 8) / 1e9),
                           "parallelism": f"rows sharded x{world}" if world > 1 else "1 GPU",
                           "generation_s": round(gen_s, 2)},
                "roofline": roof, "gpu_launches": launches, "clocks": ck_sum,
                "solver_stats": stats,
                "cg_steps_per_row": round(stats["cg_steps"] / max(1, stats["rows_solved"]), 3)}

    # A fresh 10-iteration run (theta0, X = 0) timed per iteration: the median
    # of iterations 2..10, and its test RMSE after the last iteration against
    # FP64 ALS (the oracle) from the same theta0.
    if rank == 0 and world == 1:
        restart(model)
        fev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(RESTART)]
        for k in range(RESTART):
            iteration(model, fev[k])
        torch.cuda.synchronize(dev)
        it_ms = [e[0].elapsed_time(e[2]) for e in fev]
        rmse10 = model.rmse()
        ref = fp64_reference_rmse(args, RESTART)
        line["fresh_run"] = {"iterations": RESTART, "ms_per_iteration": [round(x, 3) for x in it_ms],
                             "median_2_to_10_s": round(float(np.median(it_ms[1:])) / 1e3, 5),
                             "rmse": round(rmse10, 6)}
        line["rmse"] = round(rmse10, 6)
        if ref is not None:
            line["rmse_fp64_oracle"] = round(ref, 6)
            line["rmse_rel_gap"] = float("%.3g" % ((rmse10 - ref) / ref))

    # The other forms of the north-star comparison on the same GPU and matrix:
    # the plain FP32 Cholesky form and the learned warm start (its net trains
    # during iterations 1-3, which are its warm-up here).
    if rank == 0 and world == 1 and args.precision != "fp32" and not args.graph and not args.no_forms:
        forms = {}
        for name, o2, warmup_it, timed_it in (
                ("fp32_cholesky", A.options(precision=A.PREC_FP32, solver=A.SOLVER_CHOLESKY), 1, 3),
                ("mixed_mlp_warm_start", A.options(precision=prec, solver=A.SOLVER_CG,
                                                   warm_start=A.WARM_MLP), 3, 3)):
            if name == "mixed_mlp_warm_start" and f > 128:
                continue
            with torch.cuda.stream(stream):
                M2 = A.Model(r, f, o2, stream=stream, theta0=th0)
            for _ in range(warmup_it):
                iteration(M2)
            M2.stats(reset=True)
            ev2 = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(timed_it)]
            for k in range(timed_it):
                iteration(M2, ev2[k])
            torch.cuda.synchronize(dev)
            ms = [e[0].elapsed_time(e[2]) for e in ev2]
            st2 = M2.stats()
            forms[name] = {"sec_per_iter": round(float(np.median(ms)) / 1e3, 5),
                           "timed_iterations": f"{warmup_it + 1}..{warmup_it + timed_it}",
                           "users_ms": round(float(np.median([e[0].elapsed_time(e[1]) for e in ev2])), 3),
                           "items_ms": round(float(np.median([e[1].elapsed_time(e[2]) for e in ev2])), 3),
                           "cg_steps_per_row": round(st2["cg_steps"] / max(1, st2["rows_solved"]), 3),
                           "kernel_errors": st2["kernel_errors"]}
            M2.close()
            del M2
        forms["mixed_previous_iterate"] = {"sec_per_iter": line["sec_per_iter"], "timed_iterations": "all"}
        if "fp32_cholesky" in forms:
            base = forms["fp32_cholesky"]["sec_per_iter"]
            for k2 in ("mixed_mlp_warm_start", "mixed_previous_iterate"):
                if k2 in forms:
                    forms[k2]["speedup_vs_fp32_cholesky"] = round(base / forms[k2]["sec_per_iter"], 2)
        line["forms"] = forms

    # e2e through the reference-facing host-buffer path: the half-step the
    # Spark JNI entry runs (als_half_step_host: the CSR arrays uploaded in row
    # ranges, each range solved while the next one crosses PCIe, X downloaded
    # range by range), rank 0 on the 1-GPU path, in the same precision and
    # solver (the drop-in call has no previous X: CG starts from zero there).
    # Theta and X live in pinned host memory, as the reference's JNI caller
    # allocates them (cudaMallocHost, CuMFJNIInterface.cpp:53-57), and so do
    # the CSR arrays.
    if rank == 0 and not args.no_e2e:
        sg = model.stats()["solver_groups"]
        A.set_dropin_options(A.options(precision=prec, solver=solver, warm_start=A.WARM_ZERO,
                                       cg_jacobi=1 if args.jacobi else 0,
                                       solver_groups=int(sg[0]) if sg[0] == sg[1] else 0))
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
        T = pin(model.factors()[1].cpu().numpy())
        Xh = pin(np.zeros((r.m, f), np.float32))
        Th = pin(np.zeros((r.n, f), np.float32))
        ptr32 = r.csr_ptr.astype(np.int32)
        cptr32 = r.csc_ptr.astype(np.int32)
        host = [pin(a) for a in (ptr32, r.csr_col, r.csr_val, cptr32, r.csc_row, r.csc_val)]
        e2e_steps = max(1, min(args.steps, 5))
        torch.cuda.synchronize(dev)
        times = []
        src_t = T
        for _ in range(e2e_steps + 1):
            t1 = time.perf_counter()
            A.half_step_host(host[0], host[1], host[2], src_t, r.m, r.n, f, lam, out=Xh)
            A.half_step_host(host[3], host[4], host[5], Xh, r.n, r.m, f, lam, out=Th)
            times.append(time.perf_counter() - t1)
            src_t = Th
        e2e_s = float(np.median(times[1:]))
        h2d = sum(a.nbytes for a in host) + 4 * (r.m + r.n) * f
        d2h = 4 * (r.m + r.n) * f
        # the host link's rate for pinned host-to-device copies (three 512 MB
        # copies after one untimed), the floor the e2e number is bound by
        hb = torch.empty(1 << 29, dtype=torch.uint8).pin_memory()
        db = torch.empty(1 << 29, dtype=torch.uint8, device=dev)
        db.copy_(hb, non_blocking=True)
        torch.cuda.synchronize(dev)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record()
        for _ in range(3):
            db.copy_(hb, non_blocking=True)
        ev[1].record()
        torch.cuda.synchronize(dev)
        h2d_gbs = 3 * hb.numel() / (ev[0].elapsed_time(ev[1]) * 1e-3) / 1e9
        del hb, db
        line["e2e"] = {"value": round(flop_iter / e2e_s / 1e9, 2), "unit": "GFLOP/s",
                       "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                       "sec_per_iter": round(e2e_s, 4),
                       "ranks": 1,  # the host-buffer call runs on rank 0's GPU alone
                       "h2d_gbs_measured": round(h2d_gbs, 1),
                       "h2d_floor_s": round(h2d / (h2d_gbs * 1e9), 4),
                       "h2d_floor_frac": round(h2d / (h2d_gbs * 1e9) / e2e_s, 3),
                       "path": "als_half_step_host x2 (users, items), the Spark JNI entry's "
                               "half-step: CSR, theta and X in pinned host memory, the ratings "
                               "uploaded in row ranges overlapped with the solve of the previous "
                               "range, X downloaded range by range; wall clock; same form (CG "
                               "from zero)"}

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        users, items, Xs, Ts, frac = cpu_sample_plan(r, f, lam, args.cpu_seconds, args.seed)
        dt, fl = cpu_port_step(r, f, lam, users, items, Xs, Ts)
        line["cpu_baseline"] = {"value": round(fl / dt / 1e9, 3), "unit": "GFLOP/s",
                                "cores": os.cpu_count(), "kind": "port",
                                "sample": f"seeded {len(users)} user + {len(items)} item rows "
                                          f"({frac:.2%}) of the same matrix, FP32 port, one pass"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if shard:
        shard.close()  # collective: every rank destroys the communicator
    model.close()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_engine(args)


if __name__ == "__main__":
    main()
