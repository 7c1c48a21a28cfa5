"""Benchmark of the TLR Cholesky (seconds per factorization) on B200.

Default workload: 2D squared-exponential covariance, N = 270,000, tile 2700
(100 x 100 tiles), accuracy e = 1e-8, maxrank 150, band 1, FP64 throughout,
nugget 1e-4, points on a jittered 520 x 520 grid in Morton order (seeded).
The compressed matrix is generated once (untimed) and kept resident in HBM;
one step = restore the pristine compressed matrix (device-to-device copy, the
factorization is in place) + the full TLR factorization.

Printed JSON line (rank 0): metric/value (s/factor, lower is better), the
end-to-end number through the C ABI with host buffers (pinned host copy of
the compressed matrix in, factor out), the roofline of the dominant kernel
class (measured with CUDA events on the library's stream), the CPU
restatement timed on whole factorizations (the workload's N = 27,000 twin,
scaled by op counts, and the reference's own 2700 case), and the SM clocks
seen during the timed region.

``--impl reference`` times the CPU restatement of the reference algorithm
(the oracle port run as a task graph on the host cores; the reference itself
cannot be built here): every step is one whole factorization of the
workload's N = 27,000 twin, extrapolated to seconds per factorization of the
workload by op counts.
Multi-GPU (torchrun): independent replicas, no collectives.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    # name: (kind, N, NB, maxrank, acc, nugget, band, autoband)
    "c2": dict(kind=2, n=270000, nb=2700, maxrank=150, acc=1e-8, noise=1e-4, band=1, autoband=False,
               workload="2D sqexp N=270000 NB=2700 (100x100 tiles) e=1e-8 maxrank=150 band=1 FP64"),
    "c1": dict(kind=2, n=2700, nb=270, maxrank=130, acc=1e-8, noise=1e-4, band=1, autoband=False,
               workload="2D sqexp N=2700 NB=270 e=1e-8 maxrank=130 band=1 FP64"),
    "c2s": dict(kind=2, n=27000, nb=2700, maxrank=150, acc=1e-8, noise=1e-4, band=1, autoband=False,
                workload="2D sqexp N=27000 NB=2700 e=1e-8 maxrank=150 band=1 FP64 (scaled twin of N=270000)"),
    # the leading 10 x 10 tiles of the N=270,000 workload (its first 27,000 Morton-ordered points)
    "c2t": dict(kind=2, n=27000, n_full=270000, nb=2700, maxrank=150, acc=1e-8, noise=1e-4, band=1,
                autoband=False,
                workload="2D sqexp leading 10x10 tiles of the N=270000 matrix, NB=2700 e=1e-8 maxrank=150 band=1 FP64"),
    # the leading 30 x 30 tiles: launches of hundreds of tasks with the full size's ranks (for profiles)
    "c2m": dict(kind=2, n=81000, n_full=270000, nb=2700, maxrank=150, acc=1e-8, noise=1e-4, band=1,
                autoband=False,
                workload="2D sqexp leading 30x30 tiles of the N=270000 matrix, NB=2700 e=1e-8 maxrank=150 band=1 FP64"),
    "c3": dict(kind=4, n=108000, nb=2700, maxrank=1350, acc=1e-8, noise=1e-4, band=1, autoband=True,
               workload="3D exp N=108000 NB=2700 e=1e-8 maxrank=1350 band auto FP64"),
    "c3s": dict(kind=4, n=27000, nb=2700, maxrank=1350, acc=1e-8, noise=1e-4, band=1, autoband=True,
                workload="3D exp N=27000 NB=2700 e=1e-8 maxrank=1350 band auto FP64 (scaled twin of N=108000)"),
    "c4": dict(kind=3, n=216000, nb=2700, maxrank=500, acc=1e-8, noise=1e-4, band=1, autoband=True,
               workload="3D sqexp N=216000 NB=2700 e=1e-8 maxrank=500 band auto FP64"),
    # the other STARS-H problem kinds of the reference driver (-D 0, -D 1)
    "rt": dict(kind=0, n=270000, nb=2700, maxrank=150, acc=1e-8, noise=0.0, band=1, autoband=False,
               workload="randtlr (-D 0) N=270000 NB=2700 decay 0.5 e=1e-8 maxrank=150 band=1 FP64"),
    "ed2s": dict(kind=1, n=27000, nb=2700, maxrank=1350, acc=1e-8, noise=0.0, band=1, autoband=True,
                 workload="electrodynamics 2D sin(kr)/r k=50 (-D 1) N=27000 NB=2700 e=1e-8 maxrank=1350 "
                          "band auto FP64"),
}
METRIC = "TLR Cholesky s/factor at e=1e-8"
UNIT = "s/factor"
WORK_FIXTURE = os.path.join(ROOT, "oracle", "workload_ops.json")


# ------------------------------------------------------------------ clocks --
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        with open(self.path) as f:
            lines = f.readlines()
        os.unlink(self.path)
        return self.parse(lines)

    @staticmethod
    def parse(lines) -> dict:
        """Summary of nvidia-smi samples (FIELDS, csv, no header, no units):
        median SM clock over the samples under load (above half the maximum),
        the maximum clock, and the throttle reasons seen active."""
        rows = []
        for line in lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [v for v in (num(r[1]) for r in rows) if v is not None]
        mxs = [v for v in (num(r[2]) for r in rows) if v is not None]
        mx = max(mxs) if mxs else None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        load = ([s for s in sm if s > 0.5 * mx] if mx else []) or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows)}


# ------------------------------------------------------------- CPU runs ----
TWIN_N = 27000            # full CPU runs: the workload's scaled twin (10 x 10 tiles of 2700)


def workload_points(tlr, prob, cfg):
    """Points of a workload: its own (None: the library generates them), or
    the first n of the n_full-point set for a leading-tiles twin."""
    if "n_full" not in cfg:
        return None
    return np.ascontiguousarray(tlr.points(prob, cfg["n_full"])[:, :cfg["n"]])


def cpu_twin_matrix(cfg, threads: int):
    """The twin of a workload: its leading 10 x 10 tiles (the first 27,000 of
    its Morton-ordered points, so the tiles are the workload's own; the
    workload itself when smaller), generated on the host cores by the oracle's
    randomized compression (one BLAS thread per tile, tiles in parallel).
    Returns (matrix, seconds)."""
    from concurrent.futures import ThreadPoolExecutor
    from threadpoolctl import threadpool_limits
    from oracle import tlr_oracle as O
    nb, mr, acc = cfg["nb"], cfg["maxrank"], cfg["acc"]
    n = min(cfg["n"], TWIN_N)
    prob = O.Problem(kind=cfg["kind"], noise=cfg["noise"])
    pts = np.ascontiguousarray(O.problem_points(prob, cfg.get("n_full", cfg["n"]), nb)[:n])
    nt = n // nb
    T = O.TLRMatrix(n, nb, 1, mr)

    def gen(mc):
        m, c = mc
        with threadpool_limits(limits=1):
            A = O.cov_block(prob, pts, m * nb, nb, c * nb, nb)
            if m == c:
                return mc, A
            U, V, r = O.compress_tile_rsvd(A, acc, mr)
            if r < 0:
                raise SystemExit(f"CPU twin: generation rejected tile {mc}")
            return mc, (U, V)

    t0 = time.perf_counter()
    with ThreadPoolExecutor(threads) as ex:
        for (m, c), v in ex.map(gen, [(m, c) for m in range(nt) for c in range(m + 1)]):
            if m == c:
                T.dense[(m, c)] = v
            else:
                T.U[(m, c)], T.V[(m, c)] = v
    return T, time.perf_counter() - t0


def cpu_full_run(T, acc: float, threads: int):
    """One whole TLR factorization of T (a copy) by the oracle's task-graph
    run on the host cores.  Returns (seconds, op_counts flops)."""
    from oracle import tlr_oracle as O
    W = T.copy()
    t0 = time.perf_counter()
    st = O.tlr_potrf_dag(W, acc, threads)
    secs = time.perf_counter() - t0
    if st.info != 0:
        raise SystemExit(f"CPU twin factorization failed, info={st.info}")
    return secs, float(st.total)


def cpu_twin_supported(cfg) -> bool:
    """Full CPU runs are bounded to a few seconds for the 2D workloads; the
    3D twins (stacked ranks up to a few thousand, dense SVDs of that size per
    update) would take minutes per run."""
    return cfg["kind"] == 2


def max_over_ranks(x: float, device=None) -> float:
    """Job time of N replicas: the maximum over ranks of each rank's device
    time (all ranks call it; one process or no process group: x itself).
    NCCL needs a device tensor, gloo a host one (device=None)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() < 2:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def class_rates(prof: dict, fp64_peak: float, hbm_peak: float) -> dict:
    """Achieved rates of every profiled kernel class: algorithmic TFLOP/s and
    its fraction of the FP64 peak, algorithmic GB/s and its fraction of the HBM
    peak (classes with no recorded time are left out; a class whose work is
    counted on the device reports what was counted)."""
    out = {}
    for name, r in prof.items():
        secs = float(r.get("seconds", 0.0) or 0.0)
        if secs <= 0.0:
            continue
        tf = float(r.get("flops", 0.0) or 0.0) / secs / 1e12
        gb = float(r.get("bytes", 0.0) or 0.0) / secs / 1e9
        out[name] = {"tflops": tf, "fp64_frac": tf / fp64_peak if fp64_peak > 0 else None,
                     "gbs": gb, "hbm_frac": gb / hbm_peak if hbm_peak > 0 else None}
    return out


def load_traffic_ratios() -> dict:
    """Measured DRAM bytes per algorithmic unit (flop, or byte for copy-like
    kernels) of each kernel, from an ncu capture summarised under profiles/:
    lines '<kernel> <ratio>' after a '# ratios' marker."""
    path = os.path.join(ROOT, "profiles", "traffic_per_unit.txt")
    out = {}
    try:
        lines = open(path).read().split("# ratios", 1)[1].splitlines()
    except (OSError, IndexError):
        return out
    for line in lines:
        parts = line.split()
        if len(parts) == 2 and not line.startswith("#"):
            try:
                out[parts[0]] = float(parts[1])
            except ValueError:
                pass
    return out


def load_work_fixture(cfg_name: str):
    try:
        with open(WORK_FIXTURE) as f:
            return json.load(f).get(cfg_name)
    except Exception:
        return None


# ------------------------------------------------------------------ arms ----
def run_reference(args, cfg):
    """The CPU restatement of the reference algorithm (the oracle's task-graph
    run; the reference itself cannot be built here) on the host cores, rank 0
    only: every step is one whole factorization of the workload's scaled twin,
    extrapolated to the workload by op_counts flops."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    if not cpu_twin_supported(cfg):
        print(json.dumps({"impl": "reference", "unavailable": "no bounded CPU run for this workload "
                          "(3D twins take minutes per factorization on the host)"}), flush=True)
        return
    T, t_gen = cpu_twin_matrix(cfg, threads)
    fx = load_work_fixture(args.config)
    times = []
    ops = 0.0
    for i in range(args.warmup + args.steps):
        secs, ops = cpu_full_run(T, cfg["acc"], threads)
        if i >= args.warmup:
            times.append(secs)
    t = statistics.median(times)
    n_twin = T.n
    if n_twin == cfg["n"]:
        value, how = t, f"whole factorization of the workload itself ({ops:.3e} op_counts flops)"
    elif fx and fx.get("total_ops"):
        value = t * fx["total_ops"] / ops
        how = (f"whole factorization of the N={n_twin} twin ({ops:.3e} op_counts flops, median {t:.2f} s); "
               f"scaled by the workload's {fx['total_ops']:.3e} op_counts flops")
    else:
        value, how = None, "twin run; workload op total unknown (no fixture)"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": cfg["workload"], "sample": how, "twin_generation_s": t_gen},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": how,
                             "full_run_s": t, "full_run_ops": ops, "full_run_n": n_twin},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def measure_dgemm_peak(torch, dev) -> float:
    """FP64 DGEMM TF/s (cuBLAS via torch.matmul), best of 5."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    best = 1e9
    for _ in range(6):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) * 1e-3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def run_profile(args, cfg):
    """One generation and one factorization with per-kernel-class event timing,
    no warm-up and no timed region: the command that ncu captures for the
    profiles (its launch list has only the work being summarised).  Prints the
    class totals (launches, seconds, algorithmic flops and bytes) as JSON."""
    from hicma_parsec_b200 import tlr
    ctx = tlr.Context(0, int(args.workspace_gb * (1 << 30)))
    prob = tlr.Problem(kind=cfg["kind"], noise=cfg["noise"], beta=0.1, sigma=1.0, seed=0)
    n, nb, mr, acc = cfg["n"], cfg["nb"], cfg["maxrank"], cfg["acc"]
    A = tlr.TLRMatrix(ctx, n, nb, mr, cfg["band"])
    ctx.prof_enable(True)
    if A.generate(prob, acc, mr, pts=workload_points(tlr, prob, cfg)) != 0:
        raise SystemExit("generation rejected a tile")
    if cfg["autoband"]:
        band = tlr.parsec_band_size_auto_tuning(A.rank_map(), n // nb, nb)
        if band != 1:
            A.band_regenerate(prob, band)
    gen = ctx.prof_read()
    ctx.prof_enable(True)
    info = A.potrf(acc, mr)
    fac = ctx.prof_read()
    ctx.prof_enable(False)
    st = A.stats()
    print(json.dumps({"config": cfg["workload"], "info": int(info), "factor_s": float(st[0]),
                      "launches": int(st[3]), "generation": gen, "factorization": fac}), flush=True)
    A.close()
    ctx.close()


def run_ours(args, cfg):
    import torch
    import torch.distributed as dist
    from hicma_parsec_b200 import tlr

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=1800))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    meas = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    fp64_peak = measure_dgemm_peak(torch, dev)

    ctx = tlr.Context(local, int(args.workspace_gb * (1 << 30)))
    ctx.set_precision(tlr.PREC_MIXED if args.precision == "mixed" else tlr.PREC_FP64)
    prob = tlr.Problem(kind=cfg["kind"], noise=cfg["noise"], beta=0.1, sigma=1.0, seed=0)
    n, nb, mr, acc = cfg["n"], cfg["nb"], cfg["maxrank"], cfg["acc"]
    tuned = ctx.autotune(nb, mr) if getattr(args, "autotune", False) else None
    A0 = tlr.TLRMatrix(ctx, n, nb, mr, cfg["band"])
    t0 = time.perf_counter()
    pts_w = workload_points(tlr, prob, cfg)
    info = A0.generate(prob, acc, mr, pts=pts_w)
    t_gen = time.perf_counter() - t0
    if info != 0:
        raise SystemExit(f"generation rejected a tile (info={info})")
    G0 = A0.rank_map()
    band = cfg["band"]
    t0 = time.perf_counter()
    if cfg["autoband"]:
        band = tlr.parsec_band_size_auto_tuning(G0, n // nb, nb)
        if band != 1:
            A0.band_regenerate(prob, band)
    t_band = time.perf_counter() - t0
    rmin, rmax, ravg = tlr.HICMA_get_stat2(A0.rank_map(), n // nb, A0.band_size)

    cpu = None

    # the working copy gets A0's layout: created at the generation band, then widened
    W = tlr.TLRMatrix(ctx, n, nb, mr, cfg["band"])
    if A0.band_size != cfg["band"]:
        W.generate(prob, acc, mr, pts=pts_w)
        W.band_regenerate(prob, A0.band_size)
    stream = torch.cuda.ExternalStream(ctx.stream)

    def step():
        W.copy_from(A0)
        inf = W.potrf(acc, mr)
        if inf != 0:
            raise SystemExit(f"factorization failed, info={inf}")

    for _ in range(args.warmup):
        step()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop()
    secs = e0.elapsed_time(e1) * 1e-3
    if world > 1:
        secs = max_over_ranks(secs, dev)
        dist.barrier()
    s_per_factor = secs / (args.steps * world)
    st = W.stats()
    total_ops = st[1]

    # profiling pass (one extra step, not part of value): per-kernel-class event timing
    ctx.prof_enable(True)
    step()
    prof = ctx.prof_read()
    ctx.prof_enable(False)
    # dominant kernel: classes whose records are one launch each (the tile POTRF
    # record spans its persistent launch plus the upper-triangle clear); every
    # batched-GEMM call site is the same kernel, k_gemm_batched
    def agg(names):
        return {f: sum(prof[n][f] for n in names) for f in ("launches", "seconds", "flops", "bytes")}
    kernels = {"k_gemm_batched": (agg([n for n in prof if n.startswith("gemm")]), "tensor"),
               "k_qr": (prof["qr"], "fp64"), "k_qapply": (prof["qapply"], "fp64"),
               "k_core_svd": (prof["core_svd"], "fp64"), "k_bcgs2": (prof["proj"], "tensor"),
               "k_copy_batched": (prof["copy"], "hbm"), "k_gram_batched": (prof["gram"], "tensor"),
               "k_rcholqr": (prof["rcholqr"], "tensor")}
    dom = max(kernels, key=lambda k: kernels[k][0]["seconds"])
    pd, kind = kernels[dom]
    launches = int(st[3])  # kernel launches of one factorization (engine counter)
    traffic_ratio = load_traffic_ratios().get(dom)
    roof = None
    if pd["launches"]:
        t_launch = pd["seconds"] / pd["launches"]
        if kind != "hbm" and pd["flops"] > 0:
            fl = pd["flops"] / pd["launches"]
            ach = fl / t_launch / 1e12
            roof = {"kernel": dom, "bound": "tensor", "achieved": ach, "peak": fp64_peak, "unit": "TFLOP/s",
                    "frac": ach / fp64_peak,
                    "traffic": traffic_ratio * fl if traffic_ratio else None,
                    "peak_source": "FP64 cuBLAS DGEMM 8192^3 measured in this run (MEASURED_PEAKS.json has no FP64 entry)",
                    "avg_launch_ms": t_launch * 1e3, "launches": pd["launches"],
                    "algorithmic_flops_per_launch": fl,
                    "traffic_source": "profiles/traffic_per_unit.txt (ncu dram bytes per algorithmic flop)"
                    if traffic_ratio else None}
        else:
            peak = meas.get("hbm_gbs", 6650.0)
            by = pd["bytes"] / pd["launches"]
            ach = by / t_launch / 1e9
            roof = {"kernel": dom, "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                    "frac": ach / peak, "traffic": traffic_ratio * by if traffic_ratio else None,
                    "peak_source": "MEASURED_PEAKS.json hbm_gbs",
                    "avg_launch_ms": t_launch * 1e3, "launches": pd["launches"]}

    # accuracy of the factor that was timed (untimed): matrix-free residual with
    # Gaussian probes against the exact covariance; with --accuracy also the
    # log-determinant against a factorization at e/100
    accuracy = {"residual_probe": W.check_probe(prob, 16, 0), "nprobe": 16, "tolerance": 10 * acc}
    ld = W.logdet()
    accuracy["logdet"] = ld
    # the consumer of the factor: one log-likelihood (TLR forward/back solve +
    # log det), host vector in and out, timed on the host
    y = np.random.default_rng(1).standard_normal(n)
    t0 = time.perf_counter()
    W.loglik(y)
    t_loglik = time.perf_counter() - t0
    if args.accuracy:
        R = tlr.TLRMatrix(ctx, n, nb, mr, cfg["band"])
        if R.generate(prob, acc / 100, mr, pts=pts_w) != 0:
            accuracy["logdet_ref"] = None
        else:
            if A0.band_size != cfg["band"]:
                R.band_regenerate(prob, A0.band_size)
            if R.potrf(acc / 100, mr) == 0:
                ld_ref = R.logdet()
                accuracy.update({"logdet_ref_e_over_100": ld_ref,
                                 "logdet_rel_err": abs(ld - ld_ref) / abs(ld_ref),
                                 "residual_probe_e_over_100": R.check_probe(prob, 16, 0)})
        R.close()

    # end to end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        nbytes = A0.store_bytes()
        host = torch.empty(nbytes // 8, dtype=torch.float64, pin_memory=True)
        ranks = np.empty((n // nb) ** 2, dtype=np.int32)
        A0.store_get(host.data_ptr(), ranks)
        # the factor's store: W holds a factor of the same matrix, so its size (plus the
        # slack of one more panel of rank growth) bounds what the copy-out writes
        out_bytes = int(W.store_bytes() * 1.25) + (n // nb) * nb * 2 * mr * 8
        out = torch.empty(out_bytes // 8, dtype=torch.float64, pin_memory=True)
        torch.cuda.synchronize()
        ts = []
        d2h = 0
        for i in range(max(1, args.e2e_steps)):
            q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            q0.record(stream)
            W.store_set(host.data_ptr(), ranks)
            # each column of the factor is copied to the host as it becomes final,
            # overlapping the later panels; the call returns with the copy-out done
            W.store_stream(out.data_ptr(), out_bytes)
            inf = W.potrf(acc, mr)
            assert inf == 0
            d2h = int(W.stats()[15])
            if d2h <= 0:
                d2h = W.store_bytes()
                W.store_get(out.data_ptr(), None)
            q1.record(stream)
            q1.synchronize()
            ts.append(q0.elapsed_time(q1) * 1e-3)
        e2e = {"value": statistics.median(ts), "unit": UNIT, "h2d_bytes_per_step": int(nbytes),
               "d2h_bytes_per_step": int(d2h), "steps": len(ts),
               "path": "hicma_tlr_store_set (pinned host -> HBM) + hicma_tlr_store_stream + hicma_tlr_dpotrf_L "
                       "(factor columns -> pinned host while the later panels run)"}
        del host, out

    # the mixed-precision form on the same matrix (FP32 products of small-norm
    # updates, everything else FP64): s/factor, probe residual and log det
    fin_stats = list(tlr.HICMA_get_stat2(W.rank_map(), n // nb, W.band_size))
    mixed = None
    if args.precision == "fp64" and not args.no_mixed:
        ctx.set_precision(tlr.PREC_MIXED)
        step()
        m0, m1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        m0.record(stream)
        for _ in range(2):
            step()
        m1.record(stream)
        m1.synchronize()
        ms = m0.elapsed_time(m1) * 1e-3 / 2
        mst = W.stats()
        mld = W.logdet()
        mixed = {"value": ms, "unit": UNIT, "steps": 2, "speedup_vs_fp64": s_per_factor / ms,
                 "updates_fp32": int(mst[9]), "residual_probe": W.check_probe(prob, 16, 0), "logdet": mld,
                 "logdet_rel_diff_vs_fp64": abs(mld - ld) / abs(ld)}
        ctx.set_precision(tlr.PREC_FP64)

    serving_line = None
    if rank == 0 and world == 1 and args.serving_requests > 0:
        serving_line = serving_stream(args.serving_requests, args.serving_nmax_default, args.slots, args.rate,
                                      min(args.workspace_gb, 8.0))

    if rank == 0 and world == 1 and not args.no_cpu and cpu_twin_supported(cfg):
        # whole factorizations on the host cores: the N=27000 twin (scaled to this
        # run's op count) and the reference's own 2700 case
        threads = os.cpu_count() or 1
        T, t_gen_cpu = cpu_twin_matrix(cfg, threads)
        csecs, cops = cpu_full_run(T, acc, threads)
        del T
        c1 = CONFIGS["c1"]
        T1, _ = cpu_twin_matrix(c1, threads)
        c1secs, c1ops = cpu_full_run(T1, c1["acc"], threads)
        del T1
        T_n = min(n, TWIN_N)
        cpu = {"value": csecs * total_ops / cops if T_n < n else csecs, "unit": UNIT, "cores": threads,
               "kind": "port",
               "sample": (f"whole TLR factorization of the N={T_n} twin (leading tiles of the workload) on the "
                          f"host cores (oracle task graph, "
                          f"one BLAS thread per task): {csecs:.2f} s for {cops:.3e} op_counts flops"
                          + (f", scaled to this run's {total_ops:.3e} op_counts flops" if T_n < n else "")),
               "full_run_s": csecs, "full_run_ops": cops, "full_run_n": T_n,
               "c1_full_run_s": c1secs, "c1_full_run_ops": c1ops}

    if rank == 0:
        line = {"metric": METRIC, "value": s_per_factor, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": secs / args.steps * 1e3, "higher_is_better": False,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": cfg["workload"], "N": n, "NB": nb, "maxrank": mr, "acc": acc,
                           "band": int(A0.band_size), "nugget": cfg["noise"], "precision": args.precision,
                           "parallelism": "replicas" if world > 1 else "single GPU",
                           "l2": "inputs larger than L2 (compressed matrix ~%.1f GB resident)" % (A0.store_bytes() / 1e9),
                           "step": "device copy of the pristine compressed matrix + full TLR factorization",
                           "generation_s": t_gen, "autoband_s": t_band, "loglik_s": t_loglik,
                           "kernel_choices": {"gemm_narrow_n": ctx.tuning()[0], "potrf_grid": ctx.tuning()[1],
                                              "autotuned": tuned is not None},
                           "rank_min_max_avg": [rmin, rmax, ravg],
                           "final_rank_min_max_avg": fin_stats},
                "tlr_tflops": total_ops / s_per_factor / world / 1e12 if world else None,
                "op_counts_flops": total_ops,
                "dense_equiv_gflops": (n ** 3 / 3.0) / s_per_factor / 1e9,
                "phase_s": {"potrf": st[4], "trsm": st[5], "syrk": st[6], "gemm_recompress": st[7],
                            "device_idle_between_panels": st[12]},
                "cholqr_null_pivots": int(st[11]), "cholqr_repeated_passes": int(st[14]),
                "jacobi_sweeps_total": st[8],
                "kernel_classes": prof,
                "kernel_class_rates": class_rates(prof, fp64_peak, meas.get("hbm_gbs", 6650.0)),
                "gpu_launches": launches * args.steps,
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk, "accuracy": accuracy,
                "mixed_precision": mixed, "serving": serving_line}
        print(json.dumps(line), flush=True)
    W.close()
    A0.close()
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def serving_stream(requests: int, nmax: int, slots: int, rate: float, workspace_gb: float) -> dict:
    """The same seeded ML requests served sequentially on one slot and by the
    continuous-batching loop (all at t=0): solves/s, p50/p99 latency, and the
    largest relative log-likelihood difference between the two runs.  Every
    slot has the same workspace in both modes, so a request that fits one slot
    alone fits it in the mix (the slots' workspaces and the admitted matrices
    share the HBM budget).  Each
    mode serves the stream once untimed on its server (first-use costs: slot
    workspaces, kernel attributes) and is timed on the second pass."""
    import torch
    from hicma_parsec_b200 import serving
    reqs = serving.sample_requests(requests, seed=0, rate=rate, n_max=nmax)
    out = {}
    ref = None
    for mode, sl in (("sequential", 1), ("continuous", slots)):
        srv = serving.MLEServer(0, slots=sl, workspace_bytes=int(workspace_gb * (1 << 30)))
        srv.run(reqs, realtime=False)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = srv.run(reqs, realtime=False)
        mk = time.perf_counter() - t0
        srv.close()
        out[mode] = serving.summarize(res, mk)
        out[mode]["slots"] = sl
        if ref is None:
            ref = res
        else:
            d = [abs(a.loglik - b.loglik) / abs(a.loglik) for a, b in zip(ref, res) if a.status == 0 and b.status == 0]
            out[mode]["max_rel_diff_vs_sequential"] = max(d) if d else None
    seq, con = out["sequential"]["solves_per_s"], out["continuous"]["solves_per_s"]
    out["speedup_vs_sequential"] = con / seq if seq and con else None
    out["workload"] = f"{requests} ML requests (seed 0), N log-U[1e4,{nmax}], tile 1000-2700, 2D/3D sqexp or 3D exp"
    return out


def run_serving(args):
    """MLE serving stream (N log-uniform requests of uneven sizes): the same seeded requests served
    sequentially on one slot and by the continuous-batching loop."""
    import torch
    from hicma_parsec_b200 import serving
    reqs = serving.sample_requests(args.requests, seed=0, rate=args.rate, n_max=args.serving_nmax)
    out = {"metric": "MLE solves/s (p50/p99 latency)", "unit": "solves/s", "higher_is_better": True,
           "n_gpus": 1, "data": "synthetic", "dtype": "f64",
           "config": {"workload": f"{len(reqs)} Poisson ML requests, N log-U[1e4,{args.serving_nmax}], tile 1000-2700, "
                                  "2D/3D sqexp or 3D exp, e in {1e-6,1e-8,1e-9}", "rate_per_s": args.rate}}
    for mode, slots, realtime in (("sequential", 1, False), ("continuous", args.slots, False),
                                  ("continuous_poisson", args.slots, True)):
        srv = serving.MLEServer(0, slots=slots, workspace_bytes=int(args.workspace_gb * (1 << 30)))
        srv.run(reqs[:2], realtime=False)   # first-use costs, untimed
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = srv.run(reqs, realtime=realtime)
        mk = time.perf_counter() - t0
        srv.close()
        out[mode] = serving.summarize(res, mk)
        out[mode]["slots"] = slots
        if mode == "sequential":
            ref = res
        else:
            diff = max(abs(a.loglik - b.loglik) / abs(a.loglik) for a, b in zip(ref, res) if a.status == 0 and b.status == 0)
            out[mode]["max_rel_diff_vs_sequential"] = diff
    out["value"] = out["continuous"]["solves_per_s"]
    out["speedup_vs_sequential"] = out["continuous"]["solves_per_s"] / out["sequential"]["solves_per_s"]
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2", choices=sorted(CONFIGS))
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--workspace-gb", type=float, default=16.0)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision measurement")
    ap.add_argument("--serving-requests", type=int, default=8,
                    help="requests of the short serving stream in the default run (0: skip)")
    ap.add_argument("--serving-nmax-default", type=int, default=60000,
                    help="largest N of the short serving stream in the default run")
    ap.add_argument("--autotune", action="store_true",
                    help="measure the kernel choices (hicma_tlr_autotune) before generation and use them")
    ap.add_argument("--serving", action="store_true", help="run the MLE serving benchmark instead")
    ap.add_argument("--accuracy", action="store_true",
                    help="also compare the log-determinant with a factorization at e/100")
    ap.add_argument("--profile-run", action="store_true",
                    help="one generation + one factorization with per-class timing (for ncu captures)")
    ap.add_argument("--requests", type=int, default=16)
    ap.add_argument("--rate", type=float, default=1.0)
    ap.add_argument("--slots", type=int, default=4)
    ap.add_argument("--serving-nmax", type=int, default=200000)
    args = ap.parse_args()
    cfg = CONFIGS[args.config]
    if args.profile_run:
        run_profile(args, cfg)
        return
    if args.serving:
        run_serving(args)
        return
    if args.impl == "reference":
        run_reference(args, cfg)
    else:
        run_ours(args, cfg)


if __name__ == "__main__":
    main()
