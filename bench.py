#!/usr/bin/env python
"""Benchmark of the zone crossmatch on B200.

Workload (default): the 50M x 50M full-scale single pass -- A and B of 50M
sources each, 80 % uniform over the sky + 20 % in 500 Gaussian clusters
(sigma 0.1 deg), B = 70 % perturbed copies of A (sigma 0.3") + 30 % random,
wrap (ra within 1" of 0/360) and polar (|dec| > 89) sources forced in,
r = zh = 1".  Synthetic and seeded (xmatch_b200/synth.py, config1).

One step = zone build of A + zone build of B + pair kernel over all of A
against B, with the input records already resident in HBM (`value`), and
the same through the C ABI from pinned host records to host pairs (`e2e`).
The metric is candidate pairs per second: pairs passing the reference
prefilter (zone band, |ddec| < r, |dra| < alpha), counted on the GPU by the
same kernel with XM_COUNT_CAND before the timed region.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--n 50000000]

Multi-GPU: the path shards by independent jobs; N ranks run N independent
replicas (weak scaling, no collective on the data path), timed as the max
over ranks.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

ARCSEC = 1.0 / 3600.0
METRIC = "xmatch 50Mx50M r=1\" candidate pairs/s (exact pair set)"
UNIT = "cand-pairs/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="xmatch_b200", choices=["xmatch_b200", "reference"])
    ap.add_argument("--n", type=int, default=50_000_000, help="sources per catalog")
    ap.add_argument("--variant", default="filter32", choices=["filter32", "plain64"])
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--dist", "--e2e-dist", dest="dist", action="store_true",
                    help="also compute and return distances (24-byte records instead of the reference's "
                         "16-byte {idA, idB} pairs)")
    ap.add_argument("--dec-band", type=float, nargs=2, default=None, metavar=("LO", "HI"),
                    help="keep only sources with dec in [LO, HI) deg (same density, smaller case for profiling)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--out", default=None, help="also append the JSON line to this file")
    ap.add_argument("--config", default="c1", choices=["c1", "c2", "c3", "c4", "dense"],
                    help="c1: 50Mx50M crossmatch (the headline); c2: 4,096-job batch; c3: precision stress; "
                         "c4: serving; dense: FP32 filter against plain FP64 in dense clusters, by radius")
    ap.add_argument("--c2-jobs", type=int, default=4096)
    ap.add_argument("--c2-scale", type=float, default=1.0, help="scale of the c2 per-job sizes")
    ap.add_argument("--c3-n", type=int, default=10_000_000)
    ap.add_argument("--c3-planted", type=int, default=1_000_000)
    ap.add_argument("--c4-catalog", type=int, default=500_000_000, help="resident catalog size")
    ap.add_argument("--c4-queries", type=int, default=400)
    ap.add_argument("--c4-rate", type=float, default=100.0, help="Poisson arrival rate (queries/s)")
    ap.add_argument("--c4-alone", type=int, default=24, help="queries also timed alone (plain FP64 kernel)")
    return ap.parse_args()


def _load_by_path(name):
    """A module of xmatch_b200 that needs neither the package nor its CUDA
    library (synth, pairhash), loaded from its file: the reference arm must not
    load this project's library."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("xm_" + name, os.path.join(ROOT, "xmatch_b200", name + ".py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def load_workload(n, seed=1001):
    """config1 catalogs, cached per box under /tmp (generation takes ~30 s at 50M)."""
    synth = _load_by_path("synth")
    OBJ_DTYPE = synth.OBJ_DTYPE
    cache = "/tmp/xmatch_b200_cfg1_%d_%d" % (n, seed)
    fa, fb = cache + "_A.bin", cache + "_B.bin"
    if os.path.exists(fa) and os.path.exists(fb):
        return np.fromfile(fa, OBJ_DTYPE), np.fromfile(fb, OBJ_DTYPE)
    A, B = synth.config1(n=n, seed=seed)
    try:
        A.tofile(fa + ".tmp")
        B.tofile(fb + ".tmp")
        os.replace(fa + ".tmp", fa)
        os.replace(fb + ".tmp", fb)
    except OSError:
        pass
    return A, B


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, power, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
                power.append(float(f[3]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "power_w_max": max(power) if power else None, "samples": len(sm), "reasons": sorted(reasons)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


# The CPU sample of the workload, the same in both arms: A's sources in a dec
# band of the sky and B's within 2r of it (every match of those A sources),
# about 17 % of the 50M catalogs and a few seconds of work per run on 16 cores.
CPU_SAMPLE_DEC = (0.0, 10.0)


def cpu_sample(A, B, r_deg):
    lo, hi = CPU_SAMPLE_DEC
    a = A[(A["dec"] >= lo) & (A["dec"] < hi)]
    b = B[(B["dec"] >= lo - 2 * r_deg) & (B["dec"] < hi + 2 * r_deg)]
    return a, b


def cpu_baseline(A, B, r_deg, steps=1):
    """The reference algorithm (zone-pair loop, all pairs per zone pair, per-pair
    FP64 sincos; Worker.cu:82-123,330-366) restated in C (oracle/), on all
    host cores, over the fixed dec-band sample of the same catalogs."""
    import oracle
    cores = os.cpu_count() or 1
    a, b = cpu_sample(A, B, r_deg)
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        p, _, st = oracle.xmatch(a, b, r_deg, mode=oracle.MODE_ALLPAIRS_SINCOS, nthreads=cores, with_dist=True)
        times.append(time.perf_counter() - t0)
    t = min(times)
    return {"value": st.n_cand / t, "unit": UNIT, "cores": cores, "kind": "port",
            "seconds": t, "sample": "A sources with dec in [%g, %g) deg (%d) x B within +-2r (%d): %d candidate "
            "pairs, %d matches; includes the CPU zone sort" % (CPU_SAMPLE_DEC + (len(a), len(b), st.n_cand, len(p))),
            "matches": len(p)}


def max_over_ranks(v, pg, device):
    """The largest of every rank's value (the whole job ends when its slowest rank does)."""
    if not pg:
        return v
    import torch
    t = torch.tensor([float(v)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, units_per_rank, ms):
    """Units per second of the whole job: every rank processes units_per_rank (replicas)."""
    return world * units_per_rank / (ms * 1e-3)


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_reference(args):
    world, rank, local = dist_setup()
    if rank != 0:
        return 0
    A, B = load_workload(args.n)
    r = 1.0 * ARCSEC
    # the fixed sample of the GPU arm's cpu_baseline, W untimed + K timed steps
    import oracle
    a, b = cpu_sample(A, B, r)
    cores = os.cpu_count() or 1
    for _ in range(args.warmup):
        oracle.xmatch(a, b, r, mode=oracle.MODE_ALLPAIRS_SINCOS, nthreads=cores)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        p, _, st = oracle.xmatch(a, b, r, mode=oracle.MODE_ALLPAIRS_SINCOS, nthreads=cores)
    dt = (time.perf_counter() - t0) / args.steps
    v = st.n_cand / dt
    sample = ("A sources with dec in [%g, %g) deg (%d) x B within +-2r (%d): %d candidate pairs, %d matches; "
              "includes the CPU zone sort" % (CPU_SAMPLE_DEC + (len(a), len(b), st.n_cand, len(p))))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded config1 mixture)",
            "config": {"workload": "config1 50Mx50M r=zh=1\" (CPU sample: dec band)", "n_per_catalog": args.n,
                       "r_arcsec": 1.0, "zh_arcsec": 1.0, "sample": sample},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference has no CPU implementation of the path; this is the oracle's restatement of "
                    "its algorithm (zone-pair loop, all pairs per zone pair, per-pair sincos), all host threads"}
    line["reference_gpu_kernel"] = reference_gpu_kernel(A, B, r, cores)
    print(json.dumps(line), flush=True)
    return 0


def reference_gpu_kernel(A, B, r, cores):
    """The reference's own pair kernel (Worker.cu xmatch_kernel, compiled unmodified
    for sm_100a) over its zone loop on the full catalogs, timed on the device; the
    candidate count of the metric comes from the oracle on the same catalogs."""
    import oracle
    from oracle import ref_kernel
    try:
        import torch
        if not (torch.cuda.is_available() and ref_kernel.available()):
            return {"unavailable": "no GPU or the reference-kernel harness was not built"}
    except ImportError:
        return {"unavailable": "torch missing"}
    secs, launches, appended = ref_kernel.time_zone_loop(A, B, r)
    p, _, st = oracle.xmatch(A, B, r, nthreads=cores, with_dist=False)
    digest = _load_by_path("pairhash").pairset_digest(p)
    return {"value": st.n_cand / secs, "unit": UNIT, "seconds": secs, "launches": launches,
            "pairs_appended": appended, "matches_oracle": st.n_match, "candidates_oracle": st.n_cand,
            "oracle_pair_set_digest": digest,
            "what": "one launch per zone pair, 16x16 blocks, FP64 with sincos per pair (Worker.cu:66-240,330-366)"}


def run_ours(args):
    import torch
    import xmatch_b200 as xm

    world, rank, local = dist_setup()
    pg = False
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = True
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    A, B = load_workload(args.n)
    if args.dec_band:
        lo, hi = args.dec_band
        A = A[(A["dec"] >= lo) & (A["dec"] < hi)]
        B = B[(B["dec"] >= lo) & (B["dec"] < hi)]
    n, nb = len(A), len(B)
    r = 1.0 * ARCSEC
    zh = 1.0 * ARCSEC
    flags = xm.XM_PLAIN64 if args.variant == "plain64" else xm.XM_FILTER32

    ctx = xm.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    # inputs resident in HBM
    dA = torch.from_numpy(A.view(np.uint8)).to(dev)
    dB = torch.from_numpy(B.view(np.uint8)).to(dev)
    torch.cuda.synchronize(dev)
    sa = ctx.build_device(dA.data_ptr(), n, zh, 0)
    sb = ctx.build_device(dB.data_ptr(), nb, zh, 1)
    # candidate count (metric numerator) and match count, untimed
    _, _, st0 = ctx.match(sa, sb, r, flags | xm.XM_COUNT_CAND, fetch=False)
    n_cand, n_match = st0["n_cand"], st0["n_match"]

    def step(stats):
        sa.rebuild_device(dA.data_ptr(), n, stats)
        sb.rebuild_device(dB.data_ptr(), nb, stats)
        ms_ = ctx.match(sa, sb, r, flags, fetch=False, with_dist=args.dist)[2]
        for k in ("ms_match", "ms_plan", "n_tested", "n_exact", "n_border", "n_launches"):
            setattr(stats, k, getattr(stats, k) + ms_[k])

    for _ in range(args.warmup):
        step(xm.XmStats())
    stats = xm.XmStats()
    if pg:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    clk = ClockSampler(local)
    clk.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step(stats)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize(dev)
    clocks = clk.stop()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, pg, dev)
    if pg:
        torch.distributed.barrier()
    K = args.steps
    per = {
        "zb_count": stats.ms_zb_count / (2 * K), "zb_offsets": stats.ms_zb_scan / (2 * K),
        "zb_scatter": stats.ms_zb_scatter / (2 * K), "zb_zone_sort": stats.ms_zb_sort / (2 * K),
        "pair_plan": stats.ms_plan / K, "pair_kernel": stats.ms_match / K,
    }
    kept_a, kept_b = len(sa), len(sb)
    n_zones = int(np.ceil(180 / zh))
    nc = (n + nb) // 2   # mean catalog size (the zb_* stages are per catalog)
    a_radec = args.dist or args.variant == "plain64"   # kernels that stage A's FP64 ra/dec
    alg_bytes = {   # algorithmic bytes per launch (per catalog for the zb_* stages)
        "zb_count": 24 * nc,                       # records in
        "zb_offsets": 16 * n_zones,                # counts in, offsets out, cursors
        "zb_scatter": (24 + 32) * nc,              # records in, 32-byte bucket records out
        "zb_zone_sort": (32 + 40) * nc,            # bucket records in; id, radec, xyz out
        "pair_plan": 64 * int(np.ceil(len(sa) / 128)),   # one 64-byte plan per tile
        # A once (id and FP32 xyz; its FP64 ra/dec too with distances or the plain-FP64 kernel), B's FP32
        # xyz once, per match B's id and the pair out; with distances also the distance out and B's ra/dec
        # in (the FP64 vectors are recomputed)
        "pair_kernel": (40 if a_radec else 24) * kept_a + 16 * kept_b + (24 + 8 + 16 if args.dist else 24) * n_match,
    }
    peaks, peak_kind = measured_peaks()
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    stages = {}
    for k, t in per.items():
        gbs = alg_bytes[k] / (t * 1e-3) / 1e9 if t > 0 else 0.0
        stages[k] = {"ms": t, "alg_bytes": alg_bytes[k], "GB/s": gbs, "frac": gbs / hbm}
    dom = max(per, key=per.get)
    # DRAM bytes (read + write) per launch from one-kernel ncu captures of the same kernels on the config-1
    # catalogs cut to dec 30..60 deg (same objects per zone; 8,919,127 A objects), scaled by the objects a
    # launch processes
    band_a = 8_919_127
    traffic_per_obj = {"pair_kernel": (437.64e6 + 87.11e6) / band_a, "zb_scatter": (214.11e6 + 237.19e6) / band_a,
                       "zb_zone_sort": (313.78e6 + 312.82e6) / band_a, "pair_plan": 3.01e6 / 4_397_838}
    units = {"pair_kernel": kept_a, "pair_plan": kept_a, "zb_scatter": nc, "zb_zone_sort": nc}
    for k in stages:
        if k in traffic_per_obj:
            stages[k]["traffic"] = traffic_per_obj[k] * units[k]
    roofline = {"bound": "hbm", "kernel": dom, "achieved": stages[dom]["GB/s"], "peak": hbm, "unit": "GB/s",
                "frac": stages[dom]["frac"], "traffic": stages[dom].get("traffic"),
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per object on a dec-band cut of "
                                  "the same catalogs, times the objects of this launch",
                "peak_source": peak_kind}
    # per catalog: records read (24) and the sorted SoA written (40); the pair kernel: A read once (24, or
    # 40 with its FP64 ra/dec), B's FP32 vectors read once (16), per match the record out (16 or 24) and
    # B's id (8)
    pipeline_bytes = ((24 + 40) * (n + nb) + (40 if a_radec else 24) * kept_a + 16 * kept_b
                      + (32 if args.dist else 24) * n_match)
    pipeline = {"alg_bytes": pipeline_bytes, "GB/s": pipeline_bytes / (ms * 1e-3) / 1e9,
                "frac": pipeline_bytes / (ms * 1e-3) / 1e9 / hbm}
    value = whole_job_rate(world, n_cand, ms)
    # FP32 issue rate of the pair loop: 7 FP32-pipe instructions per tested pair
    # (3 FSUB, 1 FMUL, 2 FFMA, 1 compare) against 128 FP32 lanes per SM at the
    # SM clock sampled during the timed steps
    sm_count = ctx.info()["sm_count"]
    f_sm = (clocks.get("sm_mhz") or 1965.0) * 1e6
    tested = stats.n_tested / K
    fp32_ach = tested * 7 / (per["pair_kernel"] * 1e-3) if per["pair_kernel"] > 0 else 0.0
    fp32_issue = {"tested_pairs": int(tested), "instr_per_pair": 7, "achieved_lane_instr_per_s": fp32_ach,
                  "peak_lane_instr_per_s": sm_count * 128 * f_sm, "frac": fp32_ach / (sm_count * 128 * f_sm),
                  "sm_mhz": f_sm / 1e6, "kernel": "pair_kernel"}

    # ---- the headline step's pair set against the oracle's (untimed) ----
    pairhash = _load_by_path("pairhash")
    pairs_dev, _ = ctx.fetch(n_match, with_dist=False)
    pair_set = {"digest": pairhash.pairset_digest(pairs_dev)}
    del pairs_dev
    gold = os.path.join(ROOT, "tests", "golden", "config1_pairset.json")
    if os.path.exists(gold) and not args.dec_band:
        with open(gold) as f:
            g = json.load(f)
        if (g["n"] == n and pairhash.inputs_fingerprint(A) == g["inputs"]["A"]
                and pairhash.inputs_fingerprint(B) == g["inputs"]["B"]):
            pair_set.update({"oracle_digest": g["digest"], "oracle_candidates": g["candidates"],
                             "equal_to_oracle": pair_set["digest"] == g["digest"] and n_cand == g["candidates"],
                             "oracle_source": "tests/golden/config1_pairset.json (oracle on the same seeded "
                                              "catalogs, tests/golden/make_config1_pairset.py)"})

    # ---- the same step with the plain all-FP64 kernel, timed the same way ----
    plain64 = None
    if args.variant == "filter32":
        def step64(st_):
            sa.rebuild_device(dA.data_ptr(), n, st_)
            sb.rebuild_device(dB.data_ptr(), nb, st_)
            st_.ms_match += ctx.match(sa, sb, r, xm.XM_PLAIN64, fetch=False, with_dist=args.dist)[2]["ms_match"]
        for _ in range(max(1, args.warmup)):
            step64(xm.XmStats())
        st64 = xm.XmStats()
        torch.cuda.synchronize(dev)
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        for _ in range(K):
            step64(st64)
        g1.record(stream)
        g1.synchronize()
        ms64 = max_over_ranks(g0.elapsed_time(g1) / K, pg, dev)
        k64 = st64.ms_match / K
        plain64 = {"ms_per_step": ms64, "pair_kernel_ms": k64, "value": whole_job_rate(world, n_cand, ms64),
                   "step_speedup_vs_plain64": ms64 / ms,
                   "kernel_speedup_vs_plain64": k64 / per["pair_kernel"] if per["pair_kernel"] > 0 else None,
                   "what": "same step and timing, pair kernel XM_PLAIN64: FP64 cuts and both unit vectors by "
                           "sincos for every candidate, as Worker.cu:88-97"}

    # ---- e2e through the C ABI with host buffers ----
    e2e_steps = args.e2e_steps or max(1, min(args.steps, 3))
    hA = torch.empty(A.nbytes, dtype=torch.uint8, pin_memory=True)
    hB = torch.empty(B.nbytes, dtype=torch.uint8, pin_memory=True)
    hA.numpy()[:] = A.view(np.uint8)
    hB.numpy()[:] = B.view(np.uint8)
    objA = hA.numpy().view(xm.OBJ_DTYPE)
    objB = hB.numpy().view(xm.OBJ_DTYPE)
    cap = n_match + 1024
    hP = torch.empty(cap * 16, dtype=torch.uint8, pin_memory=True)
    hD = torch.empty(cap * 8, dtype=torch.uint8, pin_memory=True)
    outP = hP.numpy().view(np.int64).reshape(-1, 2)
    outD = hD.numpy().view(np.float64)

    e2e_parts = {"h2d": 0.0, "build": 0.0, "plan": 0.0, "match": 0.0, "d2h": 0.0, "wall": 0.0}

    def e2e_step():
        t0 = time.perf_counter()
        p, d, st = ctx.crossmatch(objA, objB, r, zh, flags, with_dist=args.dist,
                                  out=(outP, outD if args.dist else None))
        e2e_parts["wall"] += (time.perf_counter() - t0) * 1e3
        for k in ("h2d", "build", "plan", "match", "d2h"):
            e2e_parts[k] += st["ms_" + k]
        return len(p)

    e2e_step()
    if pg:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    for k in e2e_parts:
        e2e_parts[k] = 0.0
    f0.record(stream)
    got = 0
    for _ in range(e2e_steps):
        got = e2e_step()
    f1.record(stream)
    f1.synchronize()
    e2e_ms = max_over_ranks(f0.elapsed_time(f1) / e2e_steps, pg, dev)
    if got != n_match:
        raise RuntimeError("e2e match count %d differs from %d" % (got, n_match))
    pair_set["e2e_digest_equal"] = pairhash.pairset_digest(outP[:got]) == pair_set["digest"]

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded config1 mixture; no survey data)",
        "config": {"workload": "config1 50Mx50M full-scale single pass, r=zh=1\"" if n == nb == 50_000_000 else
                   "config1 mixture %d x %d, r=zh=1\"%s" % (n, nb, " (dec band %g..%g deg of %d)" % (
                       args.dec_band[0], args.dec_band[1], args.n) if args.dec_band else ""),
                   "n_per_catalog": n, "r_arcsec": 1.0, "zh_arcsec": 1.0, "variant": args.variant,
                   "parallelism": "replicas x%d" % world,
                   "l2": "inputs (2 x %.1f GB records) larger than L2 (126 MB); no flush" % (24 * nc / 1e9),
                   "step": "zone build A + zone build B + pair kernel (inputs resident in HBM)",
                   "output": "{idA, idB, dist} per match" if args.dist else
                             "{idA, idB} per match, the reference's output record (--dist adds distances)"},
        "seconds_per_step": ms * 1e-3, "candidates": n_cand, "matches": n_match,
        "matches_per_s": whole_job_rate(world, n_match, ms),
        "tested_pairs": stats.n_tested // K, "fp64_decisions": stats.n_exact // K,
        "border_pairs": stats.n_border // K,
        "borderline_fraction": (stats.n_border / stats.n_tested) if stats.n_tested else 0.0,
        "gpu_launches": int(stats.n_launches),
        "roofline": roofline, "fp32_issue": fp32_issue, "stages": stages, "pipeline_roofline": pipeline,
        "plain64": plain64, "pair_set": pair_set,
        "clocks": clocks,
        "e2e": {"value": whole_job_rate(world, n_cand, e2e_ms), "unit": UNIT, "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": 24 * (n + nb), "d2h_bytes_per_step": (24 if args.dist else 16) * n_match,
                "path": "xm_crossmatch from pinned host records to pinned host %s (B copied while A builds; "
                        "matches written to the host by the pair kernel)"
                        % ("{idA, idB, dist} records" if args.dist else
                           "{idA, idB} records (the reference's output record)"),
                "parts_ms": {k: v / e2e_steps for k, v in e2e_parts.items()}},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(A, B, r)
    sa.free()
    sb.free()
    ctx.close()
    if pg:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        s = json.dumps(line)
        print(s, flush=True)
        if args.out:
            with open(args.out, "a") as f:
                f.write(s + "\n")
    return 0


def emit(args, line):
    s = json.dumps(line)
    print(s, flush=True)
    if args.out:
        with open(args.out, "a") as f:
            f.write(s + "\n")


def event_ms(stream, fn, steps, warmup):
    """Device time per call of fn() (CUDA events on the library's stream)."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / steps


def run_c2(args):
    """Config 2: thousands of uneven segment-pair jobs (LogNormal sizes, own
    radius and zone height each) in one persistent launch; autotuned tuning vs
    the fixed one, graph vs direct launches, FP32 filter vs plain FP64, and the
    reference-style loop of one match per job."""
    import torch
    import xmatch_b200 as xm
    from xmatch_b200 import synth
    torch.cuda.set_device(0)
    jobs = synth.config2_jobs(n_jobs=args.c2_jobs, scale=args.c2_scale)
    ctx = xm.Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=torch.device("cuda", 0))
    t0 = time.perf_counter()
    segs = [(ctx.build(A, r * ARCSEC), ctx.build(B, r * ARCSEC), r * ARCSEC) for A, B, r in jobs]
    build_s = time.perf_counter() - t0
    n_a = sum(len(A) for A, _, _ in jobs)
    n_b = sum(len(B) for _, B, _ in jobs)
    _, cnt, st = ctx.match_batch(segs, xm.XM_COUNT_CAND, fetch=False)
    n_cand, n_match = st["n_cand"], sum(cnt)
    tuning, tune_best_ms, tune_fixed_ms = ctx.autotune(segs)
    fixed = (128, 16, 0, 16)
    K, W = args.steps, max(args.warmup, 3)
    variants = {
        "autotuned": lambda: ctx.match_batch(segs, 0, tuning=tuning, fetch=False),
        "fixed": lambda: ctx.match_batch(segs, 0, tuning=fixed, fetch=False),
        "autotuned_no_graph": lambda: ctx.match_batch(segs, xm.XM_NO_GRAPH, tuning=tuning, fetch=False),
        "plain64": lambda: ctx.match_batch(segs, xm.XM_PLAIN64, tuning=tuning, fetch=False),
    }
    wall = {k: [] for k in variants}
    kern = {k: [] for k in variants}
    for rep in range(W + K):   # variants interleaved, so that drift hits all alike
        for k, f in variants.items():
            torch.cuda.synchronize()
            t = time.perf_counter()
            st_ = f()[2]
            if rep >= W:
                wall[k].append((time.perf_counter() - t) * 1e3)
                kern[k].append(st_["ms_match"])
    ms = {k: float(np.median(v)) for k, v in wall.items()}
    kernel_ms = {k: float(np.median(v)) for k, v in kern.items()}
    t = time.perf_counter()
    for a, b, r in segs:
        ctx.match(a, b, r, 0, fetch=False)
    ms["loop_of_single_matches"] = (time.perf_counter() - t) * 1e3
    t0 = time.perf_counter()
    res, _, _ = ctx.match_batch(segs, 0, tuning=tuning)
    e2e_s = time.perf_counter() - t0
    got = sum(len(p) for p, _ in res)
    if got != n_match:
        raise RuntimeError("batch returned %d matches, expected %d" % (got, n_match))
    v = n_cand / (ms["autotuned"] * 1e-3)   # whole batch call (wall), results left on the device
    emit(args, {
        "metric": "config2 batch candidate pairs/s", "value": v, "unit": UNIT, "n_gpus": 1, "steps": K,
        "warmup": W, "ms_per_step": ms["autotuned"], "higher_is_better": True, "dtype": "f64",
        "data": "synthetic (seeded config2 jobs; no survey data)",
        "config": {"workload": "config2 %d jobs, LogNormal(20k, 1) sizes x %g, dec bands 0.5-5 deg, r = zh ~ U[0.5, 5]\""
                   % (len(jobs), args.c2_scale), "objects_a": n_a, "objects_b": n_b},
        "candidates": n_cand, "matches": n_match, "jobs_per_s": len(jobs) / (ms["autotuned"] * 1e-3),
        "tuning": {"autotuned": list(tuning), "fixed": list(fixed), "autotune_best_ms": tune_best_ms,
                   "autotune_fixed_ms": tune_fixed_ms},
        "wall_ms_per_batch": ms, "pair_kernel_ms": kernel_ms,
        "speedup_vs_loop": ms["loop_of_single_matches"] / ms["autotuned"],
        "kernel_speedup_vs_plain64": kernel_ms["plain64"] / kernel_ms["autotuned"],
        "e2e": {"seconds": e2e_s, "what": "one xm_match_batch with results copied to host and split by job"},
        "segment_build_s": build_s,
    })
    for a, b, _ in segs:
        a.free()
        b.free()
    ctx.close()
    return 0


def run_c3(args):
    """Config 3: precision stress, uniform catalogs plus planted pairs at
    r (1 +- k 1e-9): every '-' pair must be found and no '+' pair, at r = 0.1"
    and 60"; reports the fraction of tested pairs in the FP32 margin band."""
    import torch
    import xmatch_b200 as xm
    from xmatch_b200 import synth
    torch.cuda.set_device(0)
    ctx = xm.Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=torch.device("cuda", 0))
    out = {}
    K, W = args.steps, max(args.warmup, 3)
    for r_arcsec in (0.1, 60.0):
        A, B, sign, kk = synth.config3(n=args.c3_n, n_planted=args.c3_planted, r_arcsec=r_arcsec)
        res = kk * 1e-9 * np.radians(r_arcsec * ARCSEC) >= 1e-13   # offset above the FP64 spacing of coordinates
        r = r_arcsec * ARCSEC
        sa, sb = ctx.build(A, r), ctx.build(B, r)
        p, _, st = ctx.match(sa, sb, r, xm.XM_COUNT_CAND)
        n = args.c3_n
        hit = np.zeros(len(sign), bool)
        pl = (p[:, 0] >= n) & (p[:, 1] - 100_000_000_000 == p[:, 0])
        hit[p[pl, 0] - n] = True
        p64, _, st64 = ctx.match(sa, sb, r, xm.XM_PLAIN64)
        same = len(p64) == len(p) and np.array_equal(p64[np.lexsort((p64[:, 1], p64[:, 0]))],
                                                    p[np.lexsort((p[:, 1], p[:, 0]))])
        t32 = event_ms(stream, lambda: ctx.match(sa, sb, r, 0, fetch=False), K, W)
        t64 = event_ms(stream, lambda: ctx.match(sa, sb, r, xm.XM_PLAIN64, fetch=False), K, W)
        out["r=%g\"" % r_arcsec] = {
            "matches": len(p), "candidates": st["n_cand"], "tested": st["n_tested"],
            "borderline": st["n_border"], "borderline_fraction": st["n_border"] / max(st["n_tested"], 1),
            "fp64_decisions": st["n_exact"],
            "planted_minus_found": int(np.sum(hit & (sign < 0))), "planted_minus": int(np.sum(sign < 0)),
            "planted_plus_found": int(np.sum(hit & (sign > 0))), "planted_plus": int(np.sum(sign > 0)),
            "planted_resolvable": int(np.sum(res)),
            "planted_resolvable_wrong": int(np.sum(res & (hit != (sign < 0)))),
            "filter32_equals_plain64": bool(same),
            "ms_filter32": t32, "ms_plain64": t64, "speedup_filter32_vs_plain64": t64 / t32,
        }
        sa.free()
        sb.free()
    first = out["r=0.1\""]
    emit(args, {
        "metric": "config3 planted-pair exactness (r = 0.1\" and 60\")", "value": first["ms_filter32"],
        "unit": "ms per match (r = 0.1\")", "n_gpus": 1, "steps": K, "warmup": W, "higher_is_better": False,
        "dtype": "f64", "data": "synthetic (seeded config3; no survey data)",
        "config": {"workload": "config3 %d uniform + %d planted pairs per side" % (args.c3_n, args.c3_planted)},
        "results": out,
    })
    ctx.close()
    return 0


def run_dense(args):
    """Where the FP32 filter pays: the pair kernel with the FP32 chord filter against
    the plain all-FP64 kernel (FP64 cuts, sincos per pair) as the candidates per
    object grow -- catalogs of only the config-1 cluster component (500 Gaussian
    clusters, sigma 0.1 deg; B = 70 % perturbed copies + 30 % random members), zone
    height = radius, radii 1" .. 30"."""
    import torch
    import xmatch_b200 as xm
    synth = _load_by_path("synth")
    torch.cuda.set_device(0)
    ctx = xm.Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=torch.device("cuda", 0))
    rng = np.random.default_rng(1005)
    n = 10_000_000
    ra, dec, centers = synth.mixture(rng, n, frac_cluster=1.0)
    A = synth.make_objs(np.arange(n), ra, dec)
    npert = int(0.7 * n)
    src = rng.integers(0, n, npert)
    pra, pdec = synth.perturb(rng, ra[src], dec[src], 0.3 * ARCSEC)
    rra, rdec, _ = synth.mixture(rng, n - npert, frac_cluster=1.0, centers=centers)
    B = synth.make_objs(np.arange(n) + 100_000_000_000, np.concatenate([pra, rra]), np.concatenate([pdec, rdec]))
    K, W = args.steps, max(args.warmup, 3)
    rows = {}
    for r_arcsec in (1.0, 3.0, 10.0, 30.0):
        r = r_arcsec * ARCSEC
        sa, sb = ctx.build(A, r), ctx.build(B, r)
        _, _, st = ctx.match(sa, sb, r, xm.XM_COUNT_CAND, fetch=False)
        t32 = event_ms(stream, lambda: ctx.match(sa, sb, r, xm.XM_NO_DIST, fetch=False), K, W)
        t64 = event_ms(stream, lambda: ctx.match(sa, sb, r, xm.XM_PLAIN64 | xm.XM_NO_DIST, fetch=False), K, W)
        k32 = ctx.match(sa, sb, r, xm.XM_NO_DIST, fetch=False)[2]["ms_match"]
        k64 = ctx.match(sa, sb, r, xm.XM_PLAIN64 | xm.XM_NO_DIST, fetch=False)[2]["ms_match"]
        rows["r=%g\"" % r_arcsec] = {
            "candidates_per_object": st["n_cand"] / len(sa), "tested_per_object": st["n_tested"] / len(sa),
            "matches": st["n_match"], "borderline_fraction": st["n_border"] / max(st["n_tested"], 1),
            "ms_match_filter32": t32, "ms_match_plain64": t64, "pair_kernel_ms_filter32": k32,
            "pair_kernel_ms_plain64": k64, "kernel_speedup_filter32_vs_plain64": k64 / k32}
        sa.free()
        sb.free()
    emit(args, {"metric": "FP32 filter vs plain FP64 pair kernel, dense clusters", "unit": "ms",
                "higher_is_better": False, "n_gpus": 1, "steps": K, "warmup": W, "dtype": "f64",
                "data": "synthetic (500 Gaussian clusters of sigma 0.1 deg, seeded)",
                "config": {"workload": "clusters only, %d x %d, zh = r" % (n, n)}, "results": rows})
    ctx.close()
    return 0


def cap_points(rng, n, ra0, dec0, radius_deg):
    """n points uniform in the spherical cap of the given radius around (ra0, dec0)."""
    ct = rng.uniform(np.cos(np.radians(radius_deg)), 1.0, n)
    st = np.sqrt(1 - ct * ct)
    ph = rng.uniform(0, 2 * np.pi, n)
    v = np.stack([ct, st * np.cos(ph), st * np.sin(ph)], axis=-1)   # around +x
    a, d = np.radians(ra0), np.radians(dec0)
    ca, sa, cd, sd = np.cos(a), np.sin(a), np.cos(d), np.sin(d)
    # rotate +x to (a, d): R = Rz(a) Ry(-d)
    x = cd * v[:, 0] - sd * v[:, 2]
    z = sd * v[:, 0] + cd * v[:, 2]
    y = v[:, 1]
    X, Y = ca * x - sa * y, sa * x + ca * y
    ra = np.degrees(np.arctan2(Y, X)) % 360.0
    dec = np.degrees(np.arcsin(np.clip(z, -1, 1)))
    return ra, dec


def run_c4(args):
    """Config 4: serving.  A resident catalog (config 1 mixture, generated on
    the GPU), query catalogs arriving as a Poisson stream (n ~ LogUniform[100,
    1M], patch diameter U[0.1, 10] deg, r ~ U[0.5, 10]\"); p50/p99 latency from
    submit to results on the host, matches/s; a sample of the queries is then
    timed alone with the plain FP64 kernel."""
    import threading
    import torch
    import xmatch_b200 as xm
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(0)
    N = args.c4_catalog
    zh = 1.0 * ARCSEC
    g = torch.Generator(device=dev)
    g.manual_seed(1004)
    nu = int(0.8 * N)
    ra = torch.rand(N, dtype=torch.float64, device=dev, generator=g) * 360.0
    dec = torch.empty(N, dtype=torch.float64, device=dev)
    dec[:nu] = torch.rad2deg(torch.asin(torch.rand(nu, dtype=torch.float64, device=dev, generator=g) * 2 - 1))
    hr = np.random.default_rng(1004)
    cra = torch.from_numpy(hr.uniform(0, 360, 500)).to(dev)
    cdec = torch.from_numpy(np.degrees(np.arcsin(hr.uniform(-1, 1, 500)))).to(dev)
    which = torch.randint(0, 500, (N - nu,), device=dev, generator=g)
    cd = cdec[which]
    dec[nu:] = (cd + 0.1 * torch.randn(N - nu, dtype=torch.float64, device=dev, generator=g)).clamp(-90.0, 90.0)
    ra[nu:] = torch.remainder(cra[which] + 0.1 * torch.randn(N - nu, dtype=torch.float64, device=dev, generator=g)
                              / torch.cos(torch.deg2rad(cd)).clamp_min(1e-3), 360.0)
    rec = torch.stack([torch.arange(N, dtype=torch.int64, device=dev), ra.view(torch.int64), dec.view(torch.int64)],
                      dim=1).contiguous()
    del ra, dec, which, cd
    ctx = xm.Context(0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    cat = ctx.build_device(rec.data_ptr(), N, zh, 0)
    cat_build_s = time.perf_counter() - t0
    del rec
    torch.cuda.empty_cache()
    # query stream, generated before the clock starts
    qr = np.random.default_rng(2004)
    queries = []
    for k in range(args.c4_queries):
        n = int(np.exp(qr.uniform(np.log(100), np.log(1_000_000))))
        diam = qr.uniform(0.1, 10.0)
        c_ra, c_dec = qr.uniform(0, 360), np.degrees(np.arcsin(qr.uniform(-1, 1)))
        ra_q, dec_q = cap_points(qr, n, c_ra, c_dec, diam / 2)
        q = np.empty(n, xm.OBJ_DTYPE)
        q["id"], q["ra"], q["dec"] = np.arange(n) + 10_000_000_000 * (k + 1), ra_q, dec_q
        queries.append((q, qr.uniform(0.5, 10.0) * ARCSEC))
    arrivals = np.cumsum(qr.exponential(1.0 / args.c4_rate, len(queries)))
    srv = xm.Server(ctx, cat)
    # warm-up before the clock (memory pools, graph, result buffers): queries of
    # the same distribution, not part of the measured stream; 4 one at a time,
    # then 8 in a burst so that multi-query batches (matches grouped by query)
    # have run too
    wr = np.random.default_rng(3004)
    warm = []
    for k in range(12):
        n = int(np.exp(wr.uniform(np.log(100), np.log(1_000_000))))
        ra_q, dec_q = cap_points(wr, n, wr.uniform(0, 360), np.degrees(np.arcsin(wr.uniform(-1, 1))),
                                 wr.uniform(0.05, 5.0))
        q = np.empty(n, xm.OBJ_DTYPE)
        q["id"], q["ra"], q["dec"] = np.arange(n), ra_q, dec_q
        warm.append((q, wr.uniform(0.5, 10.0) * ARCSEC))
    for q, r in warm[:4]:
        srv.poll(srv.submit(q, r))
    for t in [srv.submit(q, r) for q, r in warm[4:]]:
        srv.poll(t)
    tickets = [None] * len(queries)
    ready = threading.Event()

    def submitter():
        start = time.perf_counter()
        for k, (q, r) in enumerate(queries):
            d = start + arrivals[k] - time.perf_counter()
            if d > 0:
                time.sleep(d)
            tickets[k] = srv.submit(q, r)
            if k == 0:
                ready.set()
    th = threading.Thread(target=submitter)
    th.start()
    infos, matches = [], 0
    for k in range(len(queries)):
        while tickets[k] is None:
            time.sleep(0.0005)
        p, d, info = srv.poll(tickets[k])
        infos.append(info)
        matches += len(p)
    th.join()
    srv.close()
    lat = np.array([i["t_done_ms"] - i["t_submit_ms"] for i in infos])
    span_s = (max(i["t_done_ms"] for i in infos) - min(i["t_submit_ms"] for i in infos)) * 1e-3
    batches = np.array([i["batch_size"] for i in infos])
    # where each query's latency goes: waiting for admission, its zone build, waiting
    # for a batch, the batch's match (pair kernel + grouping), results to the host
    parts = {"admit_wait": ("t_submit_ms", "t_admit_ms"), "build": ("t_admit_ms", "t_built_ms"),
             "batch_wait": ("t_built_ms", "t_batch_ms"), "match": ("t_batch_ms", "t_matched_ms"),
             "to_host": ("t_matched_ms", "t_done_ms")}
    comp = {k: np.array([i[b] - i[a] for i in infos]) for k, (a, b) in parts.items()}
    slow = np.argsort(lat)[-max(1, len(lat) // 100):]   # the slowest 1 %
    breakdown = {k: {"p50": float(np.percentile(v, 50)), "p99": float(np.percentile(v, 99)),
                     "mean_slowest_1pct": float(v[slow].mean())} for k, v in comp.items()}
    slowest = [{"ms": float(lat[k]), "n": len(queries[k][0]), "r_arcsec": queries[k][1] * 3600,
                "batch": int(infos[k]["batch"]), "batch_size": int(batches[k]),
                **{p: float(comp[p][k]) for p in parts}} for k in slow[::-1]]
    # the batches of the slowest queries: every member, and the match time of each member alone
    slow_batches = {}
    for k in slow:
        b = int(infos[k]["batch"])
        if b in slow_batches:
            continue
        members = [j for j in range(len(infos)) if int(infos[j]["batch"]) == b]
        rows = []
        for j in members:
            q, r = queries[j]
            s_ = ctx.build(q, zh)
            st_ = ctx.match(s_, cat, r, 0, fetch=False)[2]
            s_.free()
            rows.append({"n": len(q), "r_arcsec": r * 3600, "match_alone_ms": st_["ms_match"],
                         "plan_alone_ms": st_["ms_plan"], "matches": st_["n_match"]})
        slow_batches[b] = rows
    # a sample alone: build + plain FP64 match + results to host, one query at a time
    alone64, alone32 = [], []
    for k in range(min(args.c4_alone, len(queries))):
        q, r = queries[k]
        for flags, acc in ((xm.XM_PLAIN64, alone64), (0, alone32)):
            t = time.perf_counter()
            s = ctx.build(q, zh)
            ctx.match(s, cat, r, flags)
            s.free()
            acc.append((time.perf_counter() - t) * 1e3)
    m = min(args.c4_alone, len(queries))
    emit(args, {
        "metric": "config4 serving p99 latency", "value": float(np.percentile(lat, 99)), "unit": "ms",
        "n_gpus": 1, "higher_is_better": False, "dtype": "f64",
        "data": "synthetic (config1 mixture catalog generated on the GPU; seeded query stream)",
        "config": {"workload": "config4 resident %d-object catalog, %d queries, Poisson %.0f/s, n ~ LogUniform[100, 1M], "
                   "patch U[0.1, 10] deg, r ~ U[0.5, 10]\"" % (N, len(queries), args.c4_rate), "zh_arcsec": 1.0},
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p90": float(np.percentile(lat, 90)),
                       "p99": float(np.percentile(lat, 99)), "max": float(lat.max())},
        "queries_per_s": len(queries) / span_s, "matches_per_s": matches / span_s, "matches": matches,
        "objects_per_s": sum(len(q) for q, _ in queries) / span_s,
        "batch_size": {"mean": float(batches.mean()), "max": int(batches.max())},
        "latency_breakdown_ms": breakdown, "slowest_queries": slowest, "batches_of_slowest": slow_batches,
        "alone_first_%d_queries_ms" % m: {"plain64_mean": float(np.mean(alone64)),
                                          "filter32_mean": float(np.mean(alone32)),
                                          "served_latency_mean": float(np.mean(lat[:m]))},
        "catalog_build_s": cat_build_s,
    })
    cat.free()
    ctx.close()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.config == "c2":
        return run_c2(args)
    if args.config == "c3":
        return run_c3(args)
    if args.config == "c4":
        return run_c4(args)
    if args.config == "dense":
        return run_dense(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
