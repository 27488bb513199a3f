#!/usr/bin/env python
"""Benchmark: CV-grid fits/s of the batched mixed-precision double CV on B200,
plus the other four synthetic configurations of the hot path.

Headline workload (C4): synthetic omics PLS-DA, X 3000 x 20000 FP32 (log1p of
log-normal, column-centred, 50 informative features), 4 classes 40/30/20/10 %,
groups of 1..5 samples, 10 outer x 5 inner stratified folds, SIMPLS ncomp
1..30.  One step = one complete double CV: 50 inner SIMPLS paths of 30
components (= 1500 (fold, ncomp) fits, the count the reference reports) plus
the 10 outer refits, test-row predictions, inner accuracies and ncomp choice.

  value     batched + BF16x3 split, X already resident in HBM (FP32)
  e2e       the same through the public host-buffer call (H2D of X, D2H of
            predictions inside the timed region)
  plain     FP64, one fit after another (the drop-in path), X resident

The other configurations ride in the same JSON line under "configs":
  c1  SIMPLS regression 400 x 2000 (+100 test rows), ncomp 10, FP64
  c2  PLSSVD (rSVD l = 60, power 2) + LDA, 20000 x 5000, 100 classes, ncomp 50,
      5000 test rows; FP64 and BF16x3
  c3  label-aware PLSSVD + candidate kNN, 1.2M x 768 FP32, 1000 Zipf classes,
      ncomp 100 (rSVD), 50000 test rows, k 10, top 5
  c5  OPLS (north 2) + Gaussian response compression (5000 -> 100) + fast
      SIMPLS ncomp 50, X 50000 x 20000, 10000 test rows; FP64, BF16x3, BF16x6
each with value (inputs in HBM), e2e (host buffers), the roofline of its step
(algorithmic flops and bytes of the reference route over the step time), the
roofline of its dominant kernel class and a CPU baseline of the oracle.

Device time comes from CUDA events on the library's stream around each call;
multi-GPU runs (torchrun) are weak-scaled replicas and report the max over ranks.
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
sys.path.insert(0, ROOT)

FITS_PER_RUN = 10 * 5 * 30
CONFIG = dict(workload="C4 double CV SIMPLS PLS-DA 3000x20000 fp32, 10x5 folds, ncomp 1..30",
              n=3000, p=20000, n_classes=4, kfold_outer=10, kfold_inner=5, ncomp_max=30,
              l2="inputs larger than L2 (X fp32 240 MB, its BF16 planes 240 MB; no flush needed)")
OTHER_CONFIGS = ("c1", "c2", "c3", "c5")
HEADLINE_DTYPE = {
    "bf16x3": "bf16x3 split (fp32 accumulate) + int8 digit planes (exact int32) + fp64",
    "bf16x6": "bf16x6 split (fp32 accumulate) + int8 digit planes (exact int32) + fp64",
    "int8": "int8 digit planes (exact int32, Ozaki) + fp64",
    "fp64": "f64",
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--small", action="store_true", help="reduced shapes (profiling captures)")
    ap.add_argument("--configs", default="all",
                    help="comma list of c1,c2,c3,c5 run besides the C4 headline, 'none' or 'all'")
    ap.add_argument("--only", default=None, help="run just this configuration (c1..c5), no C4 headline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="headline without the autotuner (profiling captures)")
    ap.add_argument("--precision", default="bf16x3", choices=["bf16x3", "bf16x6", "int8", "fp64"],
                    help="precision of the timed headline steps")
    ap.add_argument("--mode", default="replicas", choices=["replicas", "folds"],
                    help="N > 1: independent replicas of the C4 job (weak scaling), or ONE C4 job whose "
                         "outer folds are split over the ranks (strong scaling)")
    return ap.parse_args()


def workload(small=False, seed=1):
    from fastpls_b200 import synthetic
    return synthetic.c4_double_cv(seed=seed, small=small)


class Clocks:
    """Samples SM clocks and throttle reasons during a timed region."""

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        fd, self.path = tempfile.mkstemp(prefix="fastpls_clocks_", suffix=".csv")
        os.close(fd)

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.2)
            self.proc.terminate()
            self.proc.wait()
            self.fh.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return dict(sm_mhz=None, sm_max_mhz=None, reasons=["nvidia-smi unavailable"])
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        try:
            os.remove(self.path)
        except OSError:
            pass
        return dict(sm_mhz=float(np.median(sm)) if sm else None, sm_max_mhz=smax,
                    reasons=sorted(reasons), samples=len(sm))


def measured_peaks():
    """HBM GB/s and dense BF16 TFLOP/s denominators (burst figures: the kernels
    are timed inside a step of a few milliseconds)."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    fp64 = (40.0, "nominal B200 FP64 tensor 40 TFLOP/s (no measured FP64 figure)")
    if os.path.exists(path):
        d = json.load(open(path))
        bf16 = float(d["bf16_tflops"])
        return dict(hbm=(float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"),
                    bf16=(bf16, "measured (MEASURED_PEAKS.json bf16_tflops, burst)"),
                    bf16x3=(bf16 / 3.0, "measured BF16 burst / 3 (three products per split GEMM)"),
                    fp64=fp64,
                    int8=(2.0 * bf16,
                          "2 x measured BF16 burst (dense INT8 tensor rate is twice BF16; no measured INT8 figure)"))
    return dict(hbm=(6650.0, "fallback 6.65 TB/s"), bf16=(1590.0, "fallback 1.59 PFLOP/s"),
                bf16x3=(530.0, "fallback BF16 1.59 PFLOP/s / 3"), fp64=fp64,
                int8=(3180.0, "2 x fallback BF16 1.59 PFLOP/s"))


# kernel class -> (peak key of its compute roofline or None, kernel description,
# ncu traffic file); a class is reported against the roof it comes closer to
# (its algorithmic flops over the compute peak or its bytes over HBM)
KERNEL_CLASSES = {
    "dual_step": (None, "k_dual_step<4, 512, 2, *> (per-fit SIMPLS steps in row space, 4-CTA clusters; "
                  "merged launches for 0 < a < K)", "k_dual_step_c4_traffic.json"),
    "k_products_f64": ("fp64", "gemm_f64_dmma (batched K products, FP64 DMMA)", None),
    "k_products_int8": ("int8", "ozaki_gemm_kernel<5> (batched K products on INT8 tcgen05 digit planes; "
                        "TOP/s of int8 plane products)", "ozaki_gemm_c4_traffic.json"),
    "gram_bf16x3": ("bf16", "split_gemm_kernel<2, 128> (tcgen05 BF16x3 row Gram, upper tiles)",
                    "gram_bf16x3_c4_traffic.json"),
    "gram_bf16x6": ("bf16", "split_gemm_kernel<3, 64> (tcgen05 BF16x6 row Gram, upper tiles)", None),
    "split_gemm_bf16x3": ("bf16", "split_gemm_kernel<2, 64 | 128> (tcgen05 BF16x3 split GEMM)", "split_gemm_c4_traffic.json"),
    "split_gemm_bf16x6": ("bf16", "split_gemm_kernel<3, 64 | 128> (tcgen05 BF16x6 split GEMM)", None),
    "gemm_f64_dmma": ("fp64", "gemm_f64_dmma (FP64 DMMA m8n8k4 tiles)", None),
    "gemv_f64": (None, "gemv_n / gemv_t (FP64 matrix-vector passes over X)", None),
    "cknn_tiles": ("fp64", "knn_tile_kernel_v2<1> (class-grouped 64x64 FP64 DMMA similarity tiles, contraction "
                           "staged in shared memory, two CTAs per SM, top-k epilogue)",
                   None),
    "cknn_filter": ("bf16", "knn_filter_kernel<1, 2> (class-grouped 128x128 tcgen05 BF16x3 similarity tiles: "
                            "approximate top-k pass, bar per pair, pass with exact FP64 rescoring of the rows "
                            "within the error bound; TFLOP/s of the BF16 products of both passes)", None),
}


def profile_traffic(fname):
    """Per-launch DRAM traffic of a kernel from its committed ncu summary."""
    if not fname:
        return None
    path = os.path.join(ROOT, "profiles", fname)
    if os.path.exists(path):
        try:
            return json.load(open(path)).get("traffic_bytes_per_launch_full_size")
        except (OSError, ValueError):
            return None
    return None


def kernel_rooflines(classes, peaks):
    """Achieved bandwidth and throughput of each profiled kernel class against
    both roofs; the class with the most device time is the dominant one."""
    out = []
    for c in classes:
        key, desc, tfile = KERNEL_CLASSES.get(c["name"], (None, c["name"], None))
        nl = max(c["launches"], 1)
        per_ms = c["ms"] / nl
        if per_ms <= 0:
            continue
        bw = (c["bytes"] / nl) / (per_ms / 1e3) / 1e9
        fb = bw / peaks["hbm"][0]
        ft, tf = 0.0, None
        if key is not None:
            tf = (c["flops"] / nl) / (per_ms / 1e3) / 1e12
            ft = tf / peaks[key][0]
        if key is not None and ft >= fb:
            r = dict(bound="tensor", achieved=tf, peak=peaks[key][0], unit="TFLOP/s", frac=ft,
                     peak_source=peaks[key][1], hbm_frac=fb)
        else:
            r = dict(bound="hbm", achieved=bw, peak=peaks["hbm"][0], unit="GB/s", frac=fb,
                     peak_source=peaks["hbm"][1], tensor_frac=ft if key else None)
        r.update(traffic=profile_traffic(tfile), kernel=desc, launches=c["launches"], total_ms=c["ms"],
                 avg_launch_ms=per_ms, algorithmic_bytes_per_launch=c["bytes"] / nl,
                 algorithmic_flops_per_launch=c["flops"] / nl)
        out.append(r)
    out.sort(key=lambda r: -r["total_ms"])
    return out


def step_roofline(flops, bytes_, ms, peaks, flop_key):
    """Roofline of a whole step: the larger of the algorithmic flops over the
    compute peak and the algorithmic bytes over HBM, per the reference route's
    work (flops and bytes counted once, at the precision the step reads)."""
    t = ms / 1e3
    peak_f, src_f = peaks[flop_key]
    peak_b, src_b = peaks["hbm"]
    ff = flops / t / 1e12 / peak_f
    fb = bytes_ / t / 1e9 / peak_b
    if ff >= fb:
        return dict(bound="tensor", achieved=flops / t / 1e12, peak=peak_f, unit="TFLOP/s", frac=ff,
                    traffic=None, scope="whole step", algorithmic_flops=flops, algorithmic_bytes=bytes_,
                    peak_source=src_f, other_frac=fb)
    return dict(bound="hbm", achieved=bytes_ / t / 1e9, peak=peak_b, unit="GB/s", frac=fb, traffic=None,
                scope="whole step", algorithmic_flops=flops, algorithmic_bytes=bytes_, peak_source=src_b,
                other_frac=ff)


# ------------------------------------------------------------ CPU baselines --

def _one_thread():
    from threadpoolctl import threadpool_limits
    return threadpool_limits(1)


def timed_cpu(sample, reps=3, one_thread_sample=None):
    """Median over `reps` runs of sample() -> (units, seconds) on all host threads,
    plus one run (of one_thread_sample when given, a smaller sample of the same
    work) with the BLAS pools held to one thread."""
    vals, secs, units = [], [], None
    for _ in range(reps):
        u, s = sample()
        units = u
        vals.append(u / s)
        secs.append(s)
    with _one_thread():
        u1, s1 = (one_thread_sample or sample)()
    return dict(value=float(np.median(vals)), samples=[float(v) for v in vals], seconds=float(np.median(secs)),
                units_per_sample=units, one_thread_value=u1 / s1, cores=os.cpu_count(), median_of=reps)


def cpu_baseline(d, min_seconds=4.0, reps=3):
    """The oracle (numpy/scipy, all host threads) on a bounded sample of the C4
    double CV: inner fold paths (30 fits each, with their predictions), outer
    fold after outer fold, until about min_seconds of CPU work; median of reps
    samples, plus a 1-thread sample."""
    from oracle import pls as opls
    from oracle import cv as ocv
    X = d["X"].astype(np.float64)
    y = d["y"]
    paths = []
    for o in range(int(d["outer"].max()) + 1):
        tr = np.where(d["outer"] != o)[0]
        for i in range(int(d["inner"][tr, o].max()) + 1):
            paths.append((o, i))

    def sample():
        fits = 0
        t0 = time.perf_counter()
        for o, i in paths:
            tr = np.where(d["outer"] != o)[0]
            fo = d["inner"][tr, o]
            train, test = tr[fo != i], tr[fo == i]
            model = opls.pls_model2_fast(X[train], ocv.response_rows(y, train, d["n_classes"]), d["ncomp"],
                                         seed=1 + 1000 + o + 1 + i)
            opls.pls_predict_classes_compact(model, X[test])
            fits += len(d["ncomp"])
            if time.perf_counter() - t0 > min_seconds:
                break
        return fits, time.perf_counter() - t0

    r = timed_cpu(sample, reps)
    r.update(unit="fits/s", kind="port",
             sample=f"{r['units_per_sample'] // len(d['ncomp'])} inner-fold SIMPLS paths ({len(d['ncomp'])} ncomp "
                    f"fits each) + predictions of the full C4 shape per sample, numpy/OpenBLAS restatement, "
                    f"median of {reps}; one_thread_value with BLAS held to 1 thread")
    return r


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    d = workload(args.small)
    for _ in range(args.warmup):
        cpu_baseline(d, min_seconds=1.0, reps=1)
    vals, secs = [], []
    cb = None
    for _ in range(args.steps):
        cb = cpu_baseline(d, min_seconds=5.0, reps=1)
        vals.append(cb["value"])
        secs.append(cb["seconds"])
    v = float(np.median(vals))
    cb["value"] = v
    print(json.dumps(dict(
        impl="reference", metric="CV-grid fits/s", value=v, unit="fits/s", n_gpus=args.gpus,
        steps=args.steps, warmup=args.warmup, ms_per_step=1000.0 * float(np.median(secs)), higher_is_better=True,
        scaling="weak", vs_baseline=None, dtype="f64", data="synthetic", config=CONFIG,
        cpu_baseline=cb, e2e=dict(value=v, unit="fits/s", h2d_bytes_per_step=0, d2h_bytes_per_step=0),
        note="reference arm = CPU restatement of the reference algorithm (R/Armadillo build is not "
             "available); each step is a bounded sample (inner-fold paths) of the C4 workload")))


def dist_init(args):
    from fastpls_b200 import replicas
    return replicas.init_from_env()


def reduce_max(pg, v):
    from fastpls_b200 import replicas
    return replicas.reduce_max(pg, v)


def barrier(pg):
    from fastpls_b200 import replicas
    replicas.barrier(pg)


# ------------------------------------------------------ other configurations --

def _torch_dev(local):
    import torch
    torch.cuda.set_device(local)
    return torch


def _dev(torch, a, dtype=None):
    """Column-major device copy of a host matrix (transpose of a contiguous tensor)."""
    a = np.asarray(a)
    if dtype is not None:
        a = a.astype(dtype)
    t = torch.from_numpy(np.ascontiguousarray(a.T)).cuda()
    return t.T


def _timed_calls(lib, fn, steps, warmup):
    """Runs fn() warmup + steps times; fn returns (result, device ms of its calls)."""
    for _ in range(warmup):
        fn()
    ms, wall, res = [], [], None
    for _ in range(steps):
        t0 = time.perf_counter()
        res, m = fn()
        wall.append(1e3 * (time.perf_counter() - t0))
        ms.append(m)
    return res, float(np.median(ms)), float(np.median(wall))


def _profile_step(lib, fn, peaks):
    lib.profile_begin()
    fn()
    lib.profile_end()
    return kernel_rooflines(lib.profile_classes(), peaks)


def config_c1(lib, args, peaks, local):
    """SIMPLS regression, FP64 drop-in: fast SIMPLS (ncomp 10) + prediction."""
    from fastpls_b200 import synthetic
    torch = _torch_dev(local)
    d = synthetic.c1_simpls_regression(seed=1)
    X, Y, Xt = d["Xtrain"], d["Ytrain"], d["Xtest"]
    n, p = X.shape
    m, K = Y.shape[1], 10
    Xd, Yd, Xtd = _dev(torch, X), _dev(torch, Y), _dev(torch, Xt)
    torch.cuda.synchronize()

    def step(Xa, Ya, Xta):
        def fn():
            model = lib.pls_model2_fast(Xa, Ya, [K], seed=1)
            t = lib.last_call_ms()
            pred = lib.predict_lowrank(model, Xta)["Ypred"]
            return pred, t + lib.last_call_ms()
        return fn

    steps = min(args.steps * 4, 40)
    pred_d, ms_d, _ = _timed_calls(lib, step(Xd, Yd, Xtd), steps, max(args.warmup, 3))
    pred_h, ms_h, wall_h = _timed_calls(lib, step(X, Y, Xt), steps, 2)
    kr = _profile_step(lib, step(Xd, Yd, Xtd), peaks)
    F = 2.0 * n * p * m + sum(4.0 * n * p + 2.0 * n * m + 14.0 * p * m + 4.0 * p * a for a in range(1, K + 1))
    B = 8.0 * n * p * (1 + K)
    out = dict(workload="C1 fast SIMPLS regression 400x2000 (+100 test rows), m=5, ncomp 10, seed 1, FP64",
               metric="fits/s (fit + test prediction)", unit="fits/s", value=1e3 / ms_d, ms_per_step=ms_d,
               steps=steps, dtype="f64",
               e2e=dict(value=1e3 / wall_h, unit="fits/s", ms_per_step=wall_h, device_ms_per_step=ms_h,
                        h2d_bytes_per_step=int(X.nbytes + Y.nbytes + Xt.nbytes),
                        d2h_bytes_per_step=int(8 * (p * K + m * K + p * m + Xt.shape[0] * m))),
               roofline=step_roofline(F, B, ms_d, peaks, "fp64"), kernel_rooflines=kr[:3],
               max_abs_diff_device_vs_host_inputs=float(np.max(np.abs(pred_d - pred_h))))
    if not args.no_cpu_baseline:
        from oracle import pls as opls

        def sample():
            t0 = time.perf_counter()
            k = 0
            while time.perf_counter() - t0 < 1.0:
                mod = opls.pls_model2_fast(X, Y, [K], seed=1)
                opls.pls_predict(mod, Xt)
                k += 1
            return k, time.perf_counter() - t0
        cb = timed_cpu(sample)
        cb.update(unit="fits/s", kind="port", sample="full C1 fits + predictions for ~1 s per sample, median of 3")
        out["cpu_baseline"] = cb
    return out


def config_c2(lib, args, peaks, local):
    """PLSSVD PLS-DA with the LDA classifier through the fused entry
    (fpls_pls_lda): rSVD fit, LDA on the fit's training scores, prediction of
    the held-out rows, X (FP32) sent once; FP64 and BF16x3."""
    from fastpls_b200 import synthetic
    from oracle import pls as opls
    torch = _torch_dev(local)
    d = synthetic.c2_plsda(seed=1)
    X, Xt = d["Xtrain"], d["Xtest"]          # FP32, column-major
    y, C, K = d["ytrain"], d["n_classes"], 50
    Y = np.asfortranarray(opls.transformy(y), dtype=np.float64)
    n, p = X.shape
    nt = Xt.shape[0]
    Xd, Xtd, Yd = _dev(torch, X), _dev(torch, Xt), _dev(torch, Y)
    torch.cuda.synchronize()
    kw = dict(method=1, oversample=10, power_iters=2, seed=1, store_B=False)

    def step(Xa, Xta, Ya):
        def fn():
            r = lib.pls_lda(Xa, Ya, y, Xta, [K], C, **kw)
            return r, lib.last_call_ms()
        return fn

    steps = min(args.steps, 10)
    res = {}
    for prec in ("fp64", "bf16x3"):
        lib.set_precision(prec)
        try:
            r_d, ms_d, _ = _timed_calls(lib, step(Xd, Xtd, Yd), steps, max(args.warmup, 2))
            lib.host_register(X)
            lib.host_register(Xt)
            lib.host_register(Y)
            try:
                r_h, ms_h, wall_h = _timed_calls(lib, step(X, Xt, Y), steps, 1)
            finally:
                lib.host_unregister(X)
                lib.host_unregister(Xt)
                lib.host_unregister(Y)
            kr = _profile_step(lib, step(Xd, Xtd, Yd), peaks)
        finally:
            lib.set_precision("fp64")
        res[prec] = (r_d, ms_d, ms_h, wall_h, kr)
    l = min(K + 10, p)
    F = (n * p + 2.0 * (1 + 2 * 2) * p * C * l + 2.0 * p * C * l + 4.0 * p * l * l + 2.0 * n * p * K
         + 4.0 * n * K * K + 2.0 * nt * p * K + 2.0 * nt * K * C)
    B = 4.0 * (2.0 * n * p + nt * p)
    r64, r3 = res["fp64"][0], res["bf16x3"][0]
    # LDA scores of the test rows under both fits (the labels' margins)
    Rp64, off64 = r64["R_predict"], r64["R_offset"]
    lin64, c64 = r64["lda_linear"][:, :K, 0], r64["lda_constants"][:, 0]
    s64 = (Xt.astype(np.float64) @ Rp64 - off64) @ lin64.T + c64
    gap = np.sort(s64, axis=1)
    clear = (gap[:, -1] - gap[:, -2]) > 1e-5 * np.abs(gap).max(axis=1)
    p64, p3 = r64["pred_codes"][:, 0], r3["pred_codes"][:, 0]
    s3 = (Xt.astype(np.float64) @ r3["R_predict"] - r3["R_offset"]) @ r3["lda_linear"][:, :K, 0].T + \
        r3["lda_constants"][:, 0]
    acc = dict(lda_score_rel_err_bf16x3_vs_fp64=float(np.linalg.norm(s3 - s64) / np.linalg.norm(s64)),
               labels_equal_beyond_margin_1e5=bool(np.all(p3[clear] == p64[clear])),
               rows_beyond_margin=int(clear.sum()),
               test_accuracy_fp64=float(np.mean(p64 == d["ytest"])),
               test_accuracy_bf16x3=float(np.mean(p3 == d["ytest"])))
    _, ms_d, ms_h, wall_h, kr = res["bf16x3"]
    out = dict(workload="C2 PLSSVD + LDA PLS-DA 20000x5000 fp32, 100 classes, ncomp 50, rSVD oversample 10 "
                        "power 2, 5000 test rows, one fused call (fpls_pls_lda)",
               metric="X rows/s (fit + LDA + test prediction)", unit="rows/s", value=n / (ms_d / 1e3),
               fits_per_s=1e3 / ms_d, ms_per_step=ms_d, steps=steps, precision="bf16x3",
               dtype="bf16x3 split GEMMs (fp32 accumulate) + fp64",
               e2e=dict(value=n / (wall_h / 1e3), unit="rows/s", ms_per_step=wall_h, device_ms_per_step=ms_h,
                        h2d_bytes_per_step=int(X.nbytes + Y.nbytes + Xt.nbytes + y.nbytes),
                        d2h_bytes_per_step=int(8 * (p * K * 3 + C * K * 2) + 4 * nt)),
               roofline=step_roofline(F, B, ms_d, peaks, "bf16x3"), kernel_rooflines=kr[:3],
               fp64=dict(ms_per_step=res["fp64"][1], rows_per_s=n / (res["fp64"][1] / 1e3),
                         e2e_ms_per_step=res["fp64"][3],
                         roofline=step_roofline(F, B, res["fp64"][1], peaks, "fp64"),
                         kernel_rooflines=res["fp64"][4][:3]),
               accuracy=acc)
    if not args.no_cpu_baseline:
        from oracle import pls_lda as opl
        Xh, Xth = X.astype(np.float64), Xt.astype(np.float64)

        def sample():
            t0 = time.perf_counter()
            opl.pls_lda(Xh, Y, y, Xth, [K], C, method=1, oversample=10, power_iters=2, seed=1)
            return n, time.perf_counter() - t0
        cb = timed_cpu(sample)
        cb.update(unit="rows/s", kind="port", sample="the full C2 step (fit, LDA, 5000 test rows) per sample, "
                                                     "FP64 numpy/OpenBLAS restatement, median of 3")
        out["cpu_baseline"] = cb
    return out


def config_c3(lib, args, peaks, local):
    """Label-aware PLSSVD (class-sorted segmented class sums, rSVD) + candidate
    kNN at 1000 classes, FP64 arithmetic on FP32 features."""
    from fastpls_b200 import synthetic
    d = synthetic.c3_prototypes(seed=1, n=200_000, n_test=10_000) if args.small else synthetic.c3_prototypes(seed=1)
    X, Xt, y, C = d["Xtrain"], d["Xtest"], d["ytrain"], d["n_classes"]
    n, p = X.shape
    nt = Xt.shape[0]
    kw = dict(ncomp=100, svd_method=4, oversample=10, power_iters=1, seed=1, knn_k=10, tau=0.2, alpha=0.75,
              top_m=20, top_k=5)
    htr, hte = lib.x_upload(X), lib.x_upload(Xt)
    steps = min(args.steps, 5)
    try:
        def fn_d():
            r = lib.label_aware_cknn_resident(htr, y, C, hte, nt, **kw)
            return r, lib.last_call_ms()

        def fn_h():
            r = lib.label_aware_cknn(X, y, C, Xt, **kw)
            return r, lib.last_call_ms()

        r_d, ms_d, _ = _timed_calls(lib, fn_d, steps, max(min(args.warmup, 2), 1))
        lib.host_register(X)
        lib.host_register(Xt)
        try:
            r_h, ms_h, wall_h = _timed_calls(lib, fn_h, steps, 1)
        finally:
            lib.host_unregister(X)
            lib.host_unregister(Xt)
        kr = _profile_step(lib, fn_d, peaks)
    finally:
        lib.x_free(htr)
        lib.x_free(hte)
    k = kw["ncomp"]
    knn = next((c for c in kr if c["kernel"].startswith("knn_tile")), None)
    F_knn = knn["algorithmic_flops_per_launch"] if knn else 0.0
    filt = next((c for c in kr if c["kernel"].startswith("knn_filter")), None)
    if filt:
        # FP64-equivalent work of the similarity tiles: one kdim-long dot per
        # (candidate pair, class row), a sixth of the BF16 products counted
        F_knn = filt["algorithmic_flops_per_launch"] / 6.0
    F = n * p + 2.0 * n * p * k + 2.0 * n * k * k + F_knn + 2.0 * nt * k * C + 2.0 * nt * p * k
    B = 2.0 * n * p * 4 + nt * p * 4
    out = dict(workload="C3 label-aware PLSSVD + cKNN 1.2Mx768 fp32, 1000 Zipf(1.1) classes, ncomp 100 (rSVD "
                        "l=110, power 1), 50000 test rows, k 10, tau 0.2, alpha 0.75, top_m 20, top 5",
               metric="X rows/s (fit + 50000-row cKNN prediction)", unit="rows/s", value=n / (ms_d / 1e3),
               ms_per_step=ms_d, steps=steps, dtype="f64 (fp32 features widened exactly)",
               e2e=dict(value=n / (wall_h / 1e3), unit="rows/s", ms_per_step=wall_h, device_ms_per_step=ms_h,
                        h2d_bytes_per_step=int(X.nbytes + Xt.nbytes + y.nbytes),
                        d2h_bytes_per_step=int(nt * 5 * 12)),
               roofline=step_roofline(F, B, ms_d, peaks, "fp64"), kernel_rooflines=kr[:3],
               resident_equals_host=bool(np.array_equal(r_d["top_index"], r_h["top_index"])))
    if not args.no_cpu_baseline:
        from oracle import cknn as ok
        from oracle import label_aware as ola
        ns, nts = 60000, 50
        Xs, ys = X[:ns].astype(np.float64), y[:ns]
        Xts = Xt[:nts].astype(np.float64)

        def sample():
            t0 = time.perf_counter()
            fit = ola.label_aware_plssvd(Xs, ys, C, [k], svd_method=4, oversample=10, power_iters=1, seed=1)
            Cl = fit["C_latent"][:, :, 0]
            Tn = ok.row_l2((((Xs - fit["mX"]) / fit["vX"]) @ fit["R"]) @ Cl)
            cents = ok.centroids(Tn, ys, C)
            t_fit = time.perf_counter() - t0
            Tt = ok.row_l2((((Xts - fit["mX"]) / fit["vX"]) @ fit["R"]) @ Cl)
            ok.candidate_knn_predict(Tt, Tn, ys, cents, top_k=5, top_m=20, knn_k=10, tau=0.2, alpha=0.75)
            t_knn = time.perf_counter() - t0 - t_fit
            # fit work is linear in the training rows; cKNN work in training rows x test rows
            est = t_fit * (n / ns) + t_knn * (n / ns) * (nt / nts)
            return n, est
        cb = timed_cpu(sample)
        cb.update(unit="rows/s", kind="port",
                  sample=f"oracle on {ns} training rows and {nts} test rows per sample, extrapolated linearly "
                         f"to {n} rows (fit) and {n} x {nt} rows (cKNN); median of 3")
        out["cpu_baseline"] = cb
    return out


def config_c5(lib, args, peaks, local):
    """OPLS filter (north 2, uncompressed Y) + Gaussian response compression
    (5000 -> 100, ridge decoder) + fast SIMPLS (ncomp 50) + filtered test
    prediction and decoding, X 50000 x 20000."""
    from fastpls_b200 import synthetic
    torch = _torch_dev(local)
    d = synthetic.c5_lowrank(seed=1)
    X = np.asfortranarray(d["Xtrain"], dtype=np.float64)
    Y = np.asfortranarray(d["Ytrain"], dtype=np.float64)
    Xt = np.asfortranarray(d["Xtest"], dtype=np.float64)
    del d
    n, p = X.shape
    q, dim, K, north = Y.shape[1], 100, 50, 2
    nt = Xt.shape[0]
    G = np.random.default_rng(1).standard_normal((q, dim)) / np.sqrt(dim)
    Xd, Yd, Xtd = _dev(torch, X), _dev(torch, Y), _dev(torch, Xt)
    Xfd = torch.empty((p, n), dtype=torch.float64, device="cuda").T
    Xtfd = torch.empty((p, nt), dtype=torch.float64, device="cuda").T
    torch.cuda.synchronize()

    def step(Xa, Ya, Xta, Xf_out, Xtf_out):
        def fn():
            filt = lib.opls_filter(Xa, Ya, north, out=Xf_out)
            t = lib.last_call_ms()
            enc = lib.gaussian_y_encode(Ya, G)
            t += lib.last_call_ms()
            model = lib.pls_model2_fast(Xf_out if Xf_out is not None else filt["X"], enc["Z"], [K], seed=1)
            t += lib.last_call_ms()
            Xtf = lib.opls_apply_filter(Xta, filt["mX"], filt["vX"], filt["W_orth"], filt["P_orth"], out=Xtf_out)
            t += lib.last_call_ms()
            Zp = lib.predict_lowrank(model, Xtf_out if Xtf_out is not None else Xtf)["Ypred"][:, :, 0]
            t += lib.last_call_ms()
            Yp = lib.gaussian_y_decode(Zp, enc["decoder"], enc["y_center"])
            return Yp, t + lib.last_call_ms()
        return fn

    steps = min(args.steps, 3)
    res = {}
    for prec in ("fp64", "bf16x3", "bf16x6"):
        lib.set_precision(prec)
        try:
            r_d, ms_d, _ = _timed_calls(lib, step(Xd, Yd, Xtd, Xfd, Xtfd), steps, 1)
            kr = _profile_step(lib, step(Xd, Yd, Xtd, Xfd, Xtfd), peaks)
            e2e = None
            if prec == "bf16x6":
                # host buffers through the public API: each matrix crosses PCIe
                # once (registered resident matrices, the filtered X kept in HBM)
                for a in (X, Y, Xt):
                    lib.host_register(a)
                try:
                    def e2e_step():
                        t0 = time.perf_counter()
                        rx, ry, rt = lib.x_resident(X), lib.x_resident(Y), lib.x_resident(Xt)
                        up_ms = 1e3 * (time.perf_counter() - t0)
                        rf, rtf = lib.x_alloc(n, p), lib.x_alloc(nt, p)
                        try:
                            yp, dev_ms = step(rx, ry, rt, rf, rtf)()
                        finally:
                            for r in (rx, ry, rt, rf, rtf):
                                r.free()
                        return yp, up_ms + dev_ms
                    # one untimed pass first (the first large allocations and
                    # registrations of the process), then the median of two
                    _, ms_h, wall_h = _timed_calls(lib, e2e_step, 2, 1)
                finally:
                    for a in (X, Y, Xt):
                        lib.host_unregister(a)
                e2e = (ms_h, wall_h)
        finally:
            lib.set_precision("fp64")
        res[prec] = (r_d, ms_d, kr, e2e)
    del Xd, Yd, Xtd, Xfd, Xtfd
    torch.cuda.empty_cache()
    s = 8
    F = (north * (2.0 * n * p * q + 4.0 * n * p) + 2.0 * n * q * dim + 2.0 * n * p * dim + K * 4.0 * n * p
         + 2.0 * n * dim * dim + 2.0 * n * q * dim + 2.0 * nt * p * K + 2.0 * nt * dim * q)
    B = s * n * p * (1 + K + 4 * north) + s * n * q * (1 + north)
    ref = res["fp64"][0]
    acc = {f"ypred_rel_err_{pr}_vs_fp64": float(np.linalg.norm(res[pr][0] - ref) / np.linalg.norm(ref))
           for pr in ("bf16x3", "bf16x6")}
    ms_h, wall_h = res["bf16x6"][3]
    out = dict(workload="C5 OPLS (north 2) + Gaussian Y (5000 -> 100) + fast SIMPLS ncomp 50, X 50000x20000, "
                        "Y 50000x5000, 10000 test rows (fp32 data, fp64 calls)",
               metric="X rows/s (filter, compression, fit, filtered test prediction, decode)", unit="rows/s",
               value=n / (res["bf16x6"][1] / 1e3), ms_per_step=res["bf16x6"][1], steps=steps,
               precision="bf16x6", dtype="bf16x6 split GEMMs (fp32 accumulate) + fp64",
               e2e=dict(value=n / (wall_h / 1e3), unit="rows/s", ms_per_step=wall_h, device_ms_per_step=ms_h,
                        h2d_bytes_per_step=int(X.nbytes + Y.nbytes + Xt.nbytes + G.nbytes),
                        d2h_bytes_per_step=int(nt * q * 8 + p * K * 8 * 2),
                        note="X, Y and Xtest uploaded once as resident matrices (fpls_x_upload), the filtered "
                             "matrices kept in HBM (fpls_x_alloc), the decoded test predictions returned"),
               roofline=step_roofline(F, B, res["bf16x6"][1], peaks, "bf16x3"),
               kernel_rooflines=res["bf16x6"][2][:3],
               other_precisions={pr: dict(ms_per_step=res[pr][1], rows_per_s=n / (res[pr][1] / 1e3),
                                          roofline=step_roofline(F, B, res[pr][1], peaks,
                                                                 "fp64" if pr == "fp64" else "bf16x3"),
                                          kernel_rooflines=res[pr][2][:3]) for pr in ("fp64", "bf16x3")},
               accuracy=acc)
    if not args.no_cpu_baseline:
        from oracle import gaussian_y as og
        from oracle import opls as oopls
        from oracle import pls as opls
        def work(nn, pp, qq, tt):
            return (north * (2.0 * nn * pp * qq + 4.0 * pp * qq * min(pp, qq) + 4.0 * nn * pp)
                    + 4.0 * nn * qq * dim + K * 4.0 * nn * pp + 2.0 * tt * pp * K + 2.0 * tt * dim * qq)

        def make_sample(f):
            ns, ps, qs, nts = n // f, p // f, q // f, nt // f
            Xs, Ys, Xts = X[:ns, :ps], Y[:ns, :qs], Xt[:nts, :ps]
            Gs = G[:qs]

            def sample():
                t0 = time.perf_counter()
                filt = oopls.opls_filter(Xs, Ys, north)
                enc = og.prepare_regression(Ys, Gs)
                model = opls.pls_model2_fast(filt["X"], enc["Z"], [K], seed=1)
                Xtf = oopls.opls_apply_filter(Xts, filt["mX"], filt["vX"], filt["W_orth"], filt["P_orth"])
                Zp = opls.pls_predict(model, Xtf)["Ypred"][:, :, 0]
                og.decode_regression(Zp, enc["decoder"], enc["y_center"])
                dt = time.perf_counter() - t0
                return n, dt * work(n, p, q, nt) / work(ns, ps, qs, nts)
            return sample
        cb = timed_cpu(make_sample(5), one_thread_sample=make_sample(10))
        cb.update(unit="rows/s", kind="port",
                  sample=f"oracle pipeline at 1/5 scale in rows, features, responses and test rows "
                         f"({n // 5}x{p // 5}, q {q // 5}), extrapolated to the full shape by the reference "
                         f"route's flop count (S products, full SVDs of S, SIMPLS passes); median of 3; the "
                         f"1-thread figure at 1/10 scale")
        out["cpu_baseline"] = cb
    return out


CONFIG_RUNNERS = dict(c1=config_c1, c2=config_c2, c3=config_c3, c5=config_c5)


# ----------------------------------------------------------- headline (C4) --

def accuracy_clause(lib, d, kw):
    """Class-score error of the mixed grid against the FP64 grid, with labels
    beyond margin, and FP64's own sensitivity: the FP64 grid on X perturbed by
    2^-24 relative (the rounding of the FP32 storage) against FP64 on X."""
    a = lib.double_cv(d["X"], d["y"], d["outer"], d["inner"], precision="fp64", return_scores=True, **kw)
    b = lib.double_cv(d["X"], d["y"], d["outer"], d["inner"], precision="bf16x3", return_scores=True, **kw)
    b6 = lib.double_cv(d["X"], d["y"], d["outer"], d["inner"], precision="bf16x6", return_scores=True, **kw)
    b8 = lib.double_cv(d["X"], d["y"], d["outer"], d["inner"], precision="int8", return_scores=True, **kw)
    rng = np.random.default_rng(7)
    Xp = (d["X"].astype(np.float64) * (1.0 + 2.0 ** -24 * rng.standard_normal(d["X"].shape)))
    c = lib.double_cv(np.asfortranarray(Xp), d["y"], d["outer"], d["inner"], precision="fp64",
                      return_scores=True, **kw)

    def rel_by_slice(x, y):
        L = x["inner_score"].shape[1]
        out = []
        for l in range(L):
            num = np.linalg.norm((x["inner_score"][:, l] - y["inner_score"][:, l]).reshape(-1))
            den = np.linalg.norm(y["inner_score"][:, l].reshape(-1))
            out.append(float(num / den))
        return out

    def labels(x, y, margin):
        s = np.sort(y["inner_score"], axis=-1)
        scale = np.abs(s).max(axis=-1)
        clear = (s[..., -1] - s[..., -2]) > margin * scale
        gi = np.transpose(x["inner_pred"], (2, 1, 0))
        gr = np.transpose(y["inner_pred"], (2, 1, 0))
        return int(np.sum((gi != gr) & clear)), int(np.sum(gi != gr))

    mixed = rel_by_slice(b, a)
    mixed6 = rel_by_slice(b6, a)
    mixed8 = rel_by_slice(b8, a)
    sens = rel_by_slice(c, a)
    out = dict(
        score_rel_err_int8_vs_fp64_max=max(mixed8),
        score_rel_err_int8_vs_fp64_by_ncomp=[round(v, 12) for v in mixed8],
        outer_score_rel_err_int8_vs_fp64=float(np.linalg.norm(b8["outer_score"] - a["outer_score"])
                                               / np.linalg.norm(a["outer_score"])),
        inner_labels_differing_int8=labels(b8, a, 0.0)[1],
        outer_labels_equal_int8=bool(np.array_equal(a["pred"], b8["pred"])),
        best_comp_equal_int8=bool(np.array_equal(a["best_comp"], b8["best_comp"])),
        score_rel_err_bf16x6_vs_fp64_max=max(mixed6),
        score_rel_err_bf16x6_vs_fp64_by_ncomp=[round(v, 9) for v in mixed6],
        outer_score_rel_err_bf16x6_vs_fp64=float(np.linalg.norm(b6["outer_score"] - a["outer_score"])
                                                 / np.linalg.norm(a["outer_score"])),
        inner_labels_differing_bf16x6=labels(b6, a, 0.0)[1],
        outer_labels_equal_bf16x6=bool(np.array_equal(a["pred"], b6["pred"])),
        score_rel_err_bf16x3_vs_fp64_max=max(mixed),
        score_rel_err_bf16x3_vs_fp64_by_ncomp=[round(v, 9) for v in mixed],
        outer_score_rel_err_bf16x3_vs_fp64=float(np.linalg.norm(b["outer_score"] - a["outer_score"])
                                                 / np.linalg.norm(a["outer_score"])),
        fp64_sensitivity_max=max(sens),
        fp64_sensitivity_by_ncomp=[round(v, 9) for v in sens],
        inner_labels_differing_bf16x3=labels(b, a, 0.0)[1],
        inner_labels_differing_beyond_margin_1e3=labels(b, a, 1e-3)[0],
        inner_labels_differing_beyond_margin_1e4=labels(b, a, 1e-4)[0],
        inner_labels_differing_fp64_perturbed=labels(c, a, 0.0)[1],
        inner_label_count=int(np.transpose(a["inner_pred"], (2, 1, 0)).size),
        outer_labels_equal=bool(np.array_equal(a["pred"], b["pred"])),
        best_comp_equal=bool(np.array_equal(a["best_comp"], b["best_comp"])),
        north_star_rel_err_1e5=dict(
            int8=bool(max(mixed8) <= 1e-5), bf16x6=bool(max(mixed6) <= 1e-5), bf16x3=bool(max(mixed) <= 1e-5),
            note="largest relative class-score error over the (outer fold, ncomp) slices against the FP64 grid; "
                 "FP64 itself moves by fp64_sensitivity under a 2^-24 relative change of X"))
    return out


def run_ours(args):
    world, rank, local, pg = dist_init(args)
    from fastpls_b200 import _lib as lib
    lib.load()
    if not lib.has_cuda():
        raise SystemExit("no B200 device")
    peaks = measured_peaks()
    if args.only:
        out = CONFIG_RUNNERS[args.only](lib, args, peaks, local)
        if rank == 0:
            print(json.dumps(out))
        return
    d = workload(args.small, seed=1 + rank)
    n, p = d["X"].shape
    kw = dict(ncomp=d["ncomp"], n_classes=d["n_classes"], seed=1)
    h = lib.x_upload(d["X"])

    def step_value(prec="bf16x3", batched=True):
        r = lib.double_cv_resident(h, n, d["y"], d["outer"], d["inner"], precision=prec,
                                   batched=batched, **kw)
        return r, lib.last_call_ms()

    # the first call of the shape tunes it (one-time cost, outside the timed steps)
    lib.set_autotune(not args.no_autotune)
    t_tune = time.perf_counter()
    step_value(args.precision)
    tune_s = time.perf_counter() - t_tune
    # warm-up
    for _ in range(max(args.warmup, 3)):
        step_value(args.precision)
    barrier(pg)
    launches0 = lib.launch_count()
    times = []
    with Clocks(local) as clk:
        # timed steps: no per-kernel events (an event between two kernels
        # stops the next one's early launch and costs a record per launch)
        for _ in range(args.steps):
            r_mixed, ms = step_value(args.precision)
            times.append(ms)
        launches = lib.launch_count() - launches0
        # the same number of steps again with CUDA events around every hot
        # kernel class on its stream: the per-kernel durations of the rooflines
        lib.profile_begin()
        for _ in range(args.steps):
            step_value(args.precision)
        lib.profile_end()
    kernels = kernel_rooflines(lib.profile_classes(), peaks)
    clocks = clk.summary()
    barrier(pg)
    total_ms = reduce_max(pg, float(np.sum(times)))
    value = world * FITS_PER_RUN * args.steps / (total_ms / 1e3)

    # e2e through the host-buffer call, inputs in page-locked host memory
    lib.host_register(d["X"])
    for _ in range(2):
        lib.double_cv(d["X"], d["y"], d["outer"], d["inner"], precision=args.precision, **kw)
    barrier(pg)
    e2e_times = []
    for _ in range(args.steps):
        lib.double_cv(d["X"], d["y"], d["outer"], d["inner"], precision=args.precision, **kw)
        e2e_times.append(lib.last_call_ms())
    barrier(pg)
    # the FP64 batched grid through the same host-buffer call
    fp64_e2e = []
    for _ in range(max(2, min(args.steps, 5))):
        lib.double_cv(d["X"], d["y"], d["outer"], d["inner"], precision="fp64", **kw)
        fp64_e2e.append(lib.last_call_ms())
    # the INT8 grid (the form within 1e-5 of FP64) through the same call
    lib.double_cv(d["X"], d["y"], d["outer"], d["inner"], precision="int8", **kw)
    int8_e2e = []
    for _ in range(max(3, min(args.steps, 5))):
        lib.double_cv(d["X"], d["y"], d["outer"], d["inner"], precision="int8", **kw)
        int8_e2e.append(lib.last_call_ms())
    lib.host_unregister(d["X"])
    e2e_ms = reduce_max(pg, float(np.sum(e2e_times)))
    e2e_value = world * FITS_PER_RUN * args.steps / (e2e_ms / 1e3)
    h2d = d["X"].nbytes + d["y"].nbytes + d["outer"].nbytes + d["inner"].nbytes + 4 * 30
    d2h = 4 * (10 + 10 * 30 * 2 + n + 60)  # best comps, accuracies, predictions, statuses

    # FP64 arms (same work, both batched and one fit after another)
    fp64_b = [step_value("fp64", True)[1] for _ in range(3)]
    fp64_batched_ms = float(np.median(fp64_b))
    step_value("bf16x6", True)
    b6_ms = float(np.median([step_value("bf16x6", True)[1] for _ in range(max(3, args.steps))]))
    step_value("int8", True)
    i8_ms = float(np.median([step_value("int8", True)[1] for _ in range(max(3, args.steps))]))
    r64 = lib.double_cv_resident(h, n, d["y"], d["outer"], d["inner"], precision="fp64",
                                 batched=True, **kw)
    plain_ms = None
    if not args.no_plain:
        r_plain, plain_ms = step_value("fp64", False)
    barrier(pg)
    lib.x_free(h)

    agree = float(np.mean(r_mixed["pred"] == r64["pred"]))
    rows_per_fit = np.mean([np.sum((d["outer"] != o) & (d["inner"][:, o] != i))
                            for o in range(10) for i in range(5)])
    ms_per_step = total_ms / args.steps
    fp64_e2e_ms = float(np.median(fp64_e2e))
    int8_e2e_ms = float(np.median(int8_e2e))
    out = dict(
        metric="CV-grid fits/s", value=value, unit="fits/s", n_gpus=world, steps=args.steps,
        warmup=args.warmup, ms_per_step=ms_per_step, higher_is_better=True, scaling="weak",
        vs_baseline=None, dtype=HEADLINE_DTYPE[args.precision],
        data="synthetic",
        config=dict(CONFIG, parallelism=f"{world} independent replicas" if world > 1 else "1 GPU",
                    precision=args.precision, batched=True, autotune=not args.no_autotune,
                    roofline_timing="per-kernel CUDA events over args.steps further steps run right after the "
                                    "timed ones (the timed steps carry no per-kernel events)"),
        x_rows_per_s=world * rows_per_fit * 50 * args.steps / (total_ms / 1e3),
        e2e=dict(value=e2e_value, unit="fits/s", h2d_bytes_per_step=int(h2d),
                 d2h_bytes_per_step=int(d2h), ms_per_step=e2e_ms / args.steps),
        roofline=kernels[0] if kernels else None,
        kernel_rooflines=kernels[1:],
        clocks=clocks, gpu_launches=int(launches),
        fp64_batched=dict(ms_per_step=fp64_batched_ms, fits_per_s=FITS_PER_RUN / (fp64_batched_ms / 1e3),
                          e2e=dict(value=FITS_PER_RUN / (fp64_e2e_ms / 1e3), unit="fits/s",
                                   ms_per_step=fp64_e2e_ms, h2d_bytes_per_step=int(h2d),
                                   d2h_bytes_per_step=int(d2h))),
        bf16x6_batched=dict(ms_per_step=b6_ms, fits_per_s=FITS_PER_RUN / (b6_ms / 1e3),
                            note="row Gram from three BF16 planes and six products; K products on INT8 as "
                                 "in the headline form"),
        int8_batched=dict(ms_per_step=i8_ms, fits_per_s=FITS_PER_RUN / (i8_ms / 1e3),
                          e2e=dict(value=FITS_PER_RUN / (int8_e2e_ms / 1e3), unit="fits/s",
                                   ms_per_step=int8_e2e_ms, h2d_bytes_per_step=int(h2d),
                                   d2h_bytes_per_step=int(d2h)),
                          note="row Gram and sketch product from digit planes of the centred rows on the INT8 "
                               "tensor cores (5 slices, exact int32 accumulation), K products on INT8 with 6 slices; "
                               "e2e: a host X goes up in column chunks, each split with its own row scales and "
                               "its Gram share taken while the next chunk is in flight"),
        parity=dict(outer_pred_agreement_bf16x3_vs_fp64=agree,
                    best_comp_equal=bool(np.array_equal(r_mixed["best_comp"], r64["best_comp"])),
                    inner_accuracy_max_abs_diff=float(np.nanmax(np.abs(r_mixed["inner_accuracy"] - r64["inner_accuracy"]))),
                    accuracy_bf16x3=r_mixed["accuracy"], accuracy_fp64=r64["accuracy"]),
    )
    if plain_ms is not None:
        out["plain_fp64"] = dict(ms_per_step=plain_ms, fits_per_s=FITS_PER_RUN / (plain_ms / 1e3),
                                 best_comp_equal=bool(np.array_equal(r_plain["best_comp"], r64["best_comp"])))
        out["speedup_vs_plain_fp64"] = (plain_ms / ms_per_step)
    rep = [r for r in lib.autotune_report() if r["n"] == n and r["p"] == p]
    out["autotune"] = dict(first_call_seconds=tune_s, shapes=[
        dict(precision=r["precision"], chosen=r["chosen"],
             default_ms=r["candidates"][0]["ms"],
             chosen_ms=min(c["ms"] for c in r["candidates"] if c["config"] == r["chosen"]),
             candidates=len(r["candidates"]), eligible=sum(1 for c in r["candidates"] if c["same_results"]))
        for r in rep])
    if rank == 0 and not args.small:
        out["accuracy"] = accuracy_clause(lib, d, kw)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(d)
    del d
    chosen = [] if args.configs == "none" else (list(OTHER_CONFIGS) if args.configs == "all"
                                                 else [c for c in args.configs.split(",") if c])
    if rank == 0 and world == 1 and chosen:
        out["configs"] = {}
        for c in chosen:
            try:
                out["configs"][c] = CONFIG_RUNNERS[c](lib, args, peaks, local)
            except Exception as e:  # a config that cannot run is reported, not hidden
                out["configs"][c] = dict(error=f"{type(e).__name__}: {e}")
    if rank == 0:
        print(json.dumps(out))
    if pg is not None:
        pg.destroy_process_group()


def run_folds(args):
    """One C4 double CV per step, its outer folds split over the ranks
    (fold_shards.double_cv_sharded): each rank fits the inner grids and refits
    of its folds on its own copy of X, and the outputs are merged by an
    all-reduce.  Every rank times the whole step (its call and the merge) with
    CUDA events after a device synchronisation; the job's time is the maximum
    over the ranks."""
    import torch
    from fastpls_b200 import _lib as lib
    from fastpls_b200 import fold_shards
    world, rank, local, pg = dist_init(args)
    lib.load()
    if not lib.has_cuda():
        raise SystemExit("no B200 device")
    torch.cuda.set_device(local)
    peaks = measured_peaks()
    d = workload(args.small, seed=1)
    n, p = d["X"].shape
    kw = dict(ncomp=d["ncomp"], n_classes=d["n_classes"], seed=1, precision=args.precision)
    h = lib.x_upload(d["X"])
    lib.set_autotune(not args.no_autotune)

    def step():
        return fold_shards.double_cv_sharded(None, d["y"], d["outer"], d["inner"], handle=h, n=n, pg=pg, **kw)

    for _ in range(max(args.warmup, 3) + 1):
        step()
    barrier(pg)
    launches0 = lib.launch_count()
    times = []
    with Clocks(local) as clk:
        for _ in range(args.steps):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            r = step()
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        launches = lib.launch_count() - launches0
        lib.profile_begin()
        for _ in range(args.steps):
            step()
        lib.profile_end()
    kernels = kernel_rooflines(lib.profile_classes(), peaks)
    barrier(pg)
    total_ms = reduce_max(pg, float(np.sum(times)))
    # e2e: the host-buffer call, X copied from page-locked memory on every rank
    lib.host_register(d["X"])
    for _ in range(2):
        fold_shards.double_cv_sharded(d["X"], d["y"], d["outer"], d["inner"], pg=pg, **kw)
    barrier(pg)
    e2e = []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fold_shards.double_cv_sharded(d["X"], d["y"], d["outer"], d["inner"], pg=pg, **kw)
        e1.record()
        torch.cuda.synchronize()
        e2e.append(e0.elapsed_time(e1))
    lib.host_unregister(d["X"])
    e2e_ms = reduce_max(pg, float(np.sum(e2e)))
    lib.x_free(h)
    plan = r["plan"]
    out = dict(
        metric="CV-grid fits/s", value=FITS_PER_RUN * args.steps / (total_ms / 1e3), unit="fits/s", n_gpus=world,
        steps=args.steps, warmup=args.warmup, ms_per_step=total_ms / args.steps, higher_is_better=True,
        scaling="strong", vs_baseline=None, dtype=HEADLINE_DTYPE[args.precision], data="synthetic",
        config=dict(CONFIG, parallelism=f"one job, outer folds split over {world} GPUs" if world > 1 else "1 GPU",
                    precision=args.precision, batched=True, autotune=not args.no_autotune, mode="folds",
                    folds_per_rank=[len(x) for x in plan]),
        e2e=dict(value=FITS_PER_RUN * args.steps / (e2e_ms / 1e3), unit="fits/s",
                 h2d_bytes_per_step=int(world * d["X"].nbytes), d2h_bytes_per_step=int(4 * (10 + 600 + n)),
                 ms_per_step=e2e_ms / args.steps),
        roofline=kernels[0] if kernels else None, kernel_rooflines=kernels[1:],
        clocks=clk.summary(), gpu_launches=int(launches), accuracy=r["accuracy"])
    if rank == 0:
        print(json.dumps(out))
    if pg is not None:
        pg.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.mode == "folds":
        run_folds(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
