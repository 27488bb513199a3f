#!/usr/bin/env python
"""Benchmark: CV-grid fits/s of the batched mixed-precision double CV on B200.

Workload (C4): synthetic omics PLS-DA, X 3000 x 20000 FP32 (log1p of
log-normal, column-centred, 50 informative features), 4 classes 40/30/20/10 %,
groups of 1..5 samples, 10 outer x 5 inner stratified folds, SIMPLS ncomp
1..30.  One step = one complete double CV: 50 inner SIMPLS paths of 30
components (= 1500 (fold, ncomp) fits, the count the reference reports) plus
the 10 outer refits, test-row predictions, inner accuracies and ncomp choice.

  value     batched + BF16x3 split, X already resident in HBM (FP32)
  e2e       the same through the public host-buffer call (H2D of X, D2H of
            predictions inside the timed region)
  plain     FP64, one fit after another (the drop-in path), X resident

Device time comes from CUDA events on the library's stream around each call;
multi-GPU runs (torchrun) are weak-scaled replicas and report the max over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FITS_PER_RUN = 10 * 5 * 30
CONFIG = dict(workload="C4 double CV SIMPLS PLS-DA 3000x20000 fp32, 10x5 folds, ncomp 1..30",
              n=3000, p=20000, n_classes=4, kfold_outer=10, kfold_inner=5, ncomp_max=30,
              l2="inputs larger than L2 (X fp32 240 MB, its BF16 planes 240 MB; no flush needed)")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--small", action="store_true", help="reduced shapes (profiling captures)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    return ap.parse_args()


def workload(small=False, seed=1):
    from fastpls_b200 import synthetic
    return synthetic.c4_double_cv(seed=seed, small=small)


class Clocks:
    """Samples SM clocks and throttle reasons during a timed region."""

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out" if os.path.isdir(os.path.join(ROOT, "gpurun_out")) else ".",
                                 f".clocks_{os.getpid()}.csv")

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
    if os.path.exists(path):
        d = json.load(open(path))
        return dict(hbm=(float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"),
                    bf16=(float(d["bf16_tflops"]), "measured (MEASURED_PEAKS.json bf16_tflops, burst)"),
                    fp64=(40.0, "nominal B200 FP64 tensor 40 TFLOP/s (no measured FP64 figure)"),
                    int8=(2.0 * float(d["bf16_tflops"]),
                          "2 x measured BF16 burst (dense INT8 tensor rate is twice BF16; no measured INT8 figure)"))
    return dict(hbm=(6650.0, "fallback 6.65 TB/s"), bf16=(1590.0, "fallback 1.59 PFLOP/s"),
                fp64=(40.0, "nominal B200 FP64 tensor 40 TFLOP/s (no measured FP64 figure)"),
                int8=(3180.0, "2 x fallback BF16 1.59 PFLOP/s"))


# kernel class -> (roofline bound, peak key, kernel description, ncu traffic file)
KERNEL_CLASSES = {
    "dual_step": ("hbm", "hbm", "k_dual_step<4, 512, 2, *> (per-fit SIMPLS steps in row space, 4-CTA clusters; "
                  "merged launches for 0 < a < K)", "k_dual_step_c4_traffic.json"),
    "k_products_f64": ("tensor", "fp64", "gemm_f64_dmma (batched K products, FP64 DMMA)", None),
    "k_products_int8": ("tensor", "int8", "ozaki_gemm_kernel<5> (batched K products on INT8 tcgen05 digit planes; "
                        "TOP/s of int8 plane products)", "ozaki_gemm_c4_traffic.json"),
    "gram_bf16x3": ("tensor", "bf16", "split_gemm_kernel<2, 128> (tcgen05 BF16x3 row Gram, upper tiles)",
                    "gram_bf16x3_c4_traffic.json"),
    "split_gemm_bf16x3": ("hbm", "hbm", "split_gemm_kernel (tcgen05 BF16x3 skinny GEMM)",
                          "split_gemm_c4_traffic.json"),
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
    """Achieved bandwidth or throughput of each profiled kernel class against
    its roofline; the class with the most device time is the dominant one."""
    out = []
    for c in classes:
        bound, key, desc, tfile = KERNEL_CLASSES.get(c["name"], ("hbm", "hbm", c["name"], None))
        per_ms = c["ms"] / max(c["launches"], 1)
        peak, src = peaks[key]
        if bound == "hbm":
            ach = (c["bytes"] / max(c["launches"], 1)) / (per_ms / 1e3) / 1e9 if per_ms > 0 else None
            unit = "GB/s"
        else:
            ach = (c["flops"] / max(c["launches"], 1)) / (per_ms / 1e3) / 1e12 if per_ms > 0 else None
            unit = "TFLOP/s"
        out.append(dict(bound=bound, achieved=ach, peak=peak, unit=unit, frac=(ach / peak) if ach else None,
                        traffic=profile_traffic(tfile), kernel=desc, launches=c["launches"],
                        total_ms=c["ms"], avg_launch_ms=per_ms,
                        algorithmic_bytes_per_launch=c["bytes"] / max(c["launches"], 1),
                        algorithmic_flops_per_launch=c["flops"] / max(c["launches"], 1), peak_source=src))
    out.sort(key=lambda r: -r["total_ms"])
    return out


def cpu_baseline(d, min_seconds=12.0):
    """The oracle (numpy/scipy, all host threads) on a bounded sample: inner
    fold paths (30 fits each, with their predictions), outer fold after outer
    fold, until about min_seconds of CPU work."""
    from oracle import pls as opls
    from oracle import cv as ocv
    X = d["X"].astype(np.float64)
    y = d["y"]
    fits = 0
    t0 = time.perf_counter()
    done = False
    for o in range(int(d["outer"].max()) + 1):
        tr = np.where(d["outer"] != o)[0]
        Xo, yo, fo = X[tr], y[tr], d["inner"][tr, o]
        for i in range(int(fo.max()) + 1):
            train = np.where(fo != i)[0]
            test = np.where(fo == i)[0]
            model = opls.pls_model2_fast(Xo[train], ocv.response_rows(yo, train, d["n_classes"]),
                                         d["ncomp"], seed=1 + 1000 + o + 1 + i)
            opls.pls_predict_classes_compact(model, Xo[test])
            fits += len(d["ncomp"])
            if time.perf_counter() - t0 > min_seconds:
                done = True
                break
        if done:
            break
    dt = time.perf_counter() - t0
    return dict(value=fits / dt, unit="fits/s", cores=os.cpu_count(), kind="port",
                sample=f"{fits // len(d['ncomp'])} inner-fold SIMPLS paths ({len(d['ncomp'])} ncomp fits each) "
                       f"+ predictions of the full C4 shape, numpy/OpenBLAS restatement", seconds=dt)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    d = workload(args.small)
    vals, secs = [], []
    for _ in range(args.warmup):
        cpu_baseline(d, min_seconds=1.0)
    cb = None
    for _ in range(args.steps):
        cb = cpu_baseline(d, min_seconds=5.0)
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


def run_ours(args):
    world, rank, local, pg = dist_init(args)
    from fastpls_b200 import _lib as lib
    lib.load()
    if not lib.has_cuda():
        raise SystemExit("no B200 device")
    d = workload(args.small, seed=1 + rank)
    n, p = d["X"].shape
    kw = dict(ncomp=d["ncomp"], n_classes=d["n_classes"], seed=1)
    h = lib.x_upload(d["X"])

    def step_value(prec="bf16x3", batched=True):
        r = lib.double_cv_resident(h, n, d["y"], d["outer"], d["inner"], precision=prec,
                                   batched=batched, **kw)
        return r, lib.last_call_ms()

    # warm-up
    for _ in range(max(args.warmup, 3)):
        step_value()
    barrier(pg)
    launches0 = lib.launch_count()
    times = []
    with Clocks(local) as clk:
        # timed steps: no per-kernel events (an event between two kernels
        # stops the next one's early launch and costs a record per launch)
        for _ in range(args.steps):
            r_mixed, ms = step_value()
            times.append(ms)
        launches = lib.launch_count() - launches0
        # the same number of steps again with CUDA events around every hot
        # kernel class on its stream: the per-kernel durations of the rooflines
        lib.profile_begin()
        for _ in range(args.steps):
            step_value()
        lib.profile_end()
    kernels = kernel_rooflines(lib.profile_classes(), measured_peaks())
    clocks = clk.summary()
    barrier(pg)
    total_ms = reduce_max(pg, float(np.sum(times)))
    value = world * FITS_PER_RUN * args.steps / (total_ms / 1e3)

    # e2e through the host-buffer call, inputs in page-locked host memory
    lib.host_register(d["X"])
    for _ in range(2):
        lib.double_cv(d["X"], d["y"], d["outer"], d["inner"], precision="bf16x3", **kw)
    barrier(pg)
    e2e_times = []
    for _ in range(args.steps):
        lib.double_cv(d["X"], d["y"], d["outer"], d["inner"], precision="bf16x3", **kw)
        e2e_times.append(lib.last_call_ms())
    barrier(pg)
    lib.host_unregister(d["X"])
    e2e_ms = reduce_max(pg, float(np.sum(e2e_times)))
    e2e_value = world * FITS_PER_RUN * args.steps / (e2e_ms / 1e3)
    h2d = d["X"].nbytes + d["y"].nbytes + d["outer"].nbytes + d["inner"].nbytes + 4 * 30
    d2h = 4 * (10 + 10 * 30 * 2 + n + 60)  # best comps, accuracies, predictions, statuses

    # FP64 arms (same work, both batched and one fit after another)
    _, fp64_batched_ms = step_value("fp64", True)
    r64 = lib.double_cv_resident(h, n, d["y"], d["outer"], d["inner"], precision="fp64",
                                 batched=True, **kw)
    plain_ms = None
    if not args.no_plain:
        r_plain, plain_ms = step_value("fp64", False)
    barrier(pg)

    agree = float(np.mean(r_mixed["pred"] == r64["pred"]))
    rows_per_fit = np.mean([np.sum((d["outer"] != o) & (d["inner"][:, o] != i))
                            for o in range(10) for i in range(5)])
    ms_per_step = total_ms / args.steps
    out = dict(
        metric="CV-grid fits/s", value=value, unit="fits/s", n_gpus=world, steps=args.steps,
        warmup=args.warmup, ms_per_step=ms_per_step, higher_is_better=True, scaling="weak",
        vs_baseline=None, dtype="bf16x3 split (fp32 accumulate) + int8 digit planes (exact int32) + fp64",
        data="synthetic",
        config=dict(CONFIG, parallelism=f"{world} independent replicas" if world > 1 else "1 GPU",
                    precision="bf16x3", batched=True,
                    roofline_timing="per-kernel CUDA events over args.steps further steps run right after the "
                                    "timed ones (the timed steps carry no per-kernel events)"),
        x_rows_per_s=world * rows_per_fit * 50 * args.steps / (total_ms / 1e3),
        e2e=dict(value=e2e_value, unit="fits/s", h2d_bytes_per_step=int(h2d),
                 d2h_bytes_per_step=int(d2h), ms_per_step=e2e_ms / args.steps),
        roofline=kernels[0] if kernels else None,
        kernel_rooflines=kernels[1:],
        clocks=clocks, gpu_launches=int(launches),
        fp64_batched=dict(ms_per_step=fp64_batched_ms, fits_per_s=FITS_PER_RUN / (fp64_batched_ms / 1e3)),
        parity=dict(outer_pred_agreement_bf16x3_vs_fp64=agree,
                    best_comp_equal=bool(np.array_equal(r_mixed["best_comp"], r64["best_comp"])),
                    inner_accuracy_max_abs_diff=float(np.nanmax(np.abs(r_mixed["inner_accuracy"] - r64["inner_accuracy"]))),
                    accuracy_bf16x3=r_mixed["accuracy"], accuracy_fp64=r64["accuracy"]),
    )
    if plain_ms is not None:
        out["plain_fp64"] = dict(ms_per_step=plain_ms, fits_per_s=FITS_PER_RUN / (plain_ms / 1e3),
                                 best_comp_equal=bool(np.array_equal(r_plain["best_comp"], r64["best_comp"])))
        out["speedup_vs_plain_fp64"] = (plain_ms / ms_per_step)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(d)
    lib.x_free(h)
    if rank == 0:
        print(json.dumps(out))
    if pg is not None:
        pg.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
