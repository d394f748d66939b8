#!/usr/bin/env python
"""Benchmark of the batched fitting path on B200: fits per second.

Workload (the cross-validation x permutation configuration): X 5000 x 10000
FP32 from the latent-factor generator (k = 10, noise 0.3), Y with 3
continuous responses, 10 uneven folds (480-520 rows), the ncomp path 1..20
and 200 seeded row permutations of Y -> (1 + 200) x 10 = 2010 SIMPLS fits per
step, all sharing one device-resident X. Arithmetic is FP64 on the device;
the products with the shared n x n Gram run as int8 digit-split products on
the tensor cores (6 digits: error below 2^-47 of the row/column scale, the
path within 1e-5 of FP64), or as FP64 DMMA GEMMs with --digits 0.

One JSON line on rank 0 with
  value    fits/s with X, Y, folds and permutations resident in HBM,
  e2e      fits/s through the host-pointer C ABI call (H2D of every input and
           D2H of every result inside the timed region, pinned host buffers),
  roofline the dominant kernel (the int8 split product) against the measured
           int8 tensor throughput of a library GEMM (FP64 DMMA GEMM against
           the measured FP64 FMA rate with --digits 0),
  cpu_baseline the reference's own FP64 C++ core (oracle/_ref, OpenBLAS on all
           host cores) on a bounded sample of the same workload.
`--impl reference` times that CPU reference alone (the reference arm).
"""
from __future__ import annotations

import argparse
import ctypes as C
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

METRIC = ("PLS fits/sec, p50/p99 ms: batched+served vs plain on 1 B200 at "
          "rel err≤1e-5")
N, P, Q, FOLDS, NCOMP = 5000, 10000, 3, 10, 20


def args_parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--perms", type=int, default=200)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--served-requests", type=int, default=120,
                    help="requests in the served mixed-workload leg (0 = skip)")
    ap.add_argument("--plain-perms", type=int, default=3,
                    help="permutations sampled for the one-fit-at-a-time path")
    ap.add_argument("--digits", type=int, default=6,
                    help="int8 digits per FP64 value in the products with the "
                         "shared Gram (0 = FP64 DMMA GEMMs)")
    ap.add_argument("--lanes", type=int, default=3,
                    help="stream lanes of the batched engine (1..4)")
    ap.add_argument("--fp64-steps", type=int, default=2,
                    help="timed steps with FP64 DMMA products, for comparison")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the single-fit configuration legs (plain FP64 "
                         "SIMPLS, full-size PLS-SVD + LDA, full-size BF16 SIMPLS)")
    ap.add_argument("--served-spec-requests", type=int, default=40,
                    help="requests in the served leg at the configuration's stated "
                         "sizes (n, p up to 50000; 0 = skip)")
    ap.add_argument("--latency-steps", type=int, default=60,
                    help="untimed extra steps for the step-latency distribution")
    return ap.parse_args()


def make_workload(rank: int, perms: int):
    from fastpls_b200 import workloads as W
    x, y, folds = W.config_cv_permutation(N, P, dtype=np.float32)
    pm = W.permutations(N, perms, 3 + 1000 * rank)
    prefixes = np.arange(1, NCOMP + 1, dtype=np.int32)
    return x, y, folds, pm, prefixes


def clock_sampler_start(path):
    q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    try:
        f = open(path, "w")
        p = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                              "-lms", "200"], stdout=f, stderr=subprocess.DEVNULL)
        import atexit

        def _end(proc=p):  # never leave the sampler running past this process
            if proc.poll() is None:
                proc.kill()
        atexit.register(_end)
        return p, f
    except Exception:
        return None, None


def clock_sampler_stop(handle, path, device_index, window=None):
    """Median SM clock and the throttle reasons seen; with window = (t0, t1)
    (time.time() around the timed region) only the samples taken inside it
    (the sampler runs from well before, so that its start-up does not fall
    into the timed steps)."""
    from datetime import datetime
    p, f = handle
    if p is None:
        return None
    p.terminate()
    try:
        p.wait(timeout=5)
    except Exception:
        p.kill()
    f.close()
    sm, mx, reasons = [], None, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for line in open(path):
        parts = [s.strip() for s in line.split(",")]
        if len(parts) < 10 or parts[1] != str(device_index):
            continue
        if window is not None:
            try:
                ts = datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
            except ValueError:
                continue
            if ts < window[0] or ts > window[1]:
                continue
        try:
            sm.append(float(parts[2]))
            mx = float(parts[3])
        except ValueError:
            continue
        for name, val in zip(names, parts[6:10]):
            if val.lower() == "active":
                reasons.add(name)
    if not sm:
        return None
    return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx,
            "reasons": sorted(reasons), "samples": len(sm)}


def cpu_reference_sample(x, y, folds, prefixes):
    """The reference FP64 core (oracle/_ref) on the observed-response CV
    (10 fold fits of the workload) with OpenBLAS on all host cores."""
    from oracle import ref
    if not ref.available():
        return None, None
    cores = os.cpu_count() or 1
    ref.set_threads(cores)
    x64 = np.asfortranarray(x, dtype=np.float64)
    y64 = np.asfortranarray(y, dtype=np.float64)
    t0 = time.perf_counter()
    out = ref.cv_regression(x64, y64, folds, prefixes, scaling=1, family=3)
    dt = time.perf_counter() - t0
    fits = int(folds.max())
    return ({"value": fits / dt, "unit": "fits/s", "cores": cores,
             "kind": "reference",
             "sample": f"observed-response {fits}-fold CV, ncomp path 1..{NCOMP} "
                       f"({fits} of the {fits * 201} fits), {dt:.1f} s"}, out)


def run_reference_arm(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import ref
    x, y, folds, _, prefixes = make_workload(0, 0)
    if not ref.available():
        print(json.dumps({"impl": "reference", "metric": METRIC,
                          "unavailable": "oracle/_ref/libfastpls_ref.so not built"}))
        return 0
    cores = os.cpu_count() or 1
    ref.set_threads(cores)
    x64 = np.asfortranarray(x, dtype=np.float64)
    y64 = np.asfortranarray(y, dtype=np.float64)
    test = np.nonzero(folds == 1)[0]
    train = np.nonzero(folds != 1)[0]
    xtr, ytr, xte = x64[train], y64[train], x64[test]

    def one_fit():
        # one fold fit plus its held-out prefix-path predictions = 1 fit unit
        m = ref.simpls_fit(xtr, ytr, ncomp=NCOMP, scaling=1)
        xs = (xte - m["centre"]) / m["scale"]
        t = xs @ m["R"]
        for k in range(1, NCOMP + 1):
            _ = m["ymean"] + t[:, :k] @ m["Q"][:, :k].T

    for _ in range(a.warmup):
        one_fit()
    times = []
    for _ in range(a.steps):
        t0 = time.perf_counter()
        one_fit()
        times.append(time.perf_counter() - t0)
    tot = sum(times)
    value = a.steps / tot
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "fits/s",
        "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": 1000 * tot / a.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(a.perms),
        "latency_ms": {"p50": 1000 * float(np.percentile(times, 50)),
                       "p99": 1000 * float(np.percentile(times, 99))},
        "cpu_baseline": {"value": value, "unit": "fits/s", "cores": cores,
                         "kind": "reference",
                         "sample": "one fold fit (4500 x 10000, ncomp 20) + its "
                                   "held-out prefix-path predictions per step"},
        "e2e": {"value": value, "unit": "fits/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def served_workload(count, seed=11):
    """Mixed request stream (scaled-down served configuration): n log-uniform
    in [200, 3000], p log-uniform in [500, 4000], m in 1..10, ncomp in 2..30;
    SIMPLS 50%, PLS-SVD 20%, OPLS 15%, kernel PLS (RBF) 15%; 30%
    classification (2-20 classes); 70% fits, 30% predictions against the
    models fitted so far. Inputs are seeded per request id."""
    from fastpls_b200 import workloads as W
    g = np.random.default_rng(seed)
    reqs = []
    fitted = []
    for rid in range(count):
        if fitted and g.random() < 0.3:
            src = fitted[int(g.integers(len(fitted)))]
            rows = int(g.integers(50, 500))
            xt, _ = W.latent_regression(rows, src["p"], 1, 3, 0.4, 5000 + rid)
            reqs.append(dict(kind="predict", src=src, x=xt))
            continue
        n = int(np.exp(g.uniform(np.log(200), np.log(3000))))
        p = int(np.exp(g.uniform(np.log(500), np.log(4000))))
        m = int(g.integers(1, 11))
        method = g.choice(["simpls", "plssvd", "opls", "kernelpls"], p=[0.5, 0.2, 0.15, 0.15])
        cls = g.random() < 0.3
        if cls:
            m = int(g.integers(2, 21))
            x, lab = W.latent_classification(n, p, m, 5, 0.4, rid)
            # factor levels present only (R drops empty levels)
            present, lab = np.unique(lab, return_inverse=True)
            lab = (lab + 1).astype(np.int32)
            m = int(present.size)
            if m < 2:
                continue
            y = None
        else:
            x, y = W.latent_regression(n, p, m, 5, 0.4, rid)
            lab = None
        cap = min(n - 1, p) if method != "kernelpls" else n - 1
        a = int(min(int(g.integers(2, 31)), cap))
        if method == "plssvd":
            a = max(1, min(a, m - 1 if cls else m))
            if cls and a < 1:
                continue
        r = dict(kind="fit", method=str(method), x=x, y=y, labels=lab,
                 classes=m if cls else None, ncomp=a, p=p, q=m)
        reqs.append(r)
        fitted.append(r)
    return reqs


def served_spec_workload(count, seed=12):
    """The served mixed workload at its stated sizes: n log-uniform in
    [200, 50000], p log-uniform in [500, 50000], m uniform in 1..10, ncomp
    uniform in [2, 30]; SIMPLS 50%, PLS-SVD 20%, OPLS 15%, kernel PLS (RBF,
    n <= 5000) 15%; 30% classification (2-20 classes); 70% fits and 30%
    predictions (100-2000 rows) against the models fitted so far. Inputs come
    from the latent-factor generator seeded by request id, drawn on the
    device (torch's Philox generator) and copied to host memory."""
    import torch
    dev = torch.device("cuda")
    g = np.random.default_rng(seed)
    reqs, fitted = [], []

    def latent(n, p, k, rid):
        gen = torch.Generator(device=dev).manual_seed(rid)
        t = torch.randn(n, k, generator=gen, device=dev)
        w = torch.randn(p, k, generator=gen, device=dev)
        xt = w @ t.T + 0.4 * torch.randn(p, n, generator=gen, device=dev)
        xt -= xt.mean(dim=1, keepdim=True)
        x = xt.cpu().numpy().T          # n x p, Fortran order
        return x, t, gen
    for rid in range(count):
        if fitted and g.random() < 0.3:
            src = fitted[int(g.integers(len(fitted)))]
            rows = int(g.integers(100, 2001))
            x, _, _ = latent(rows, src["p"], 5, 900000 + rid)
            reqs.append(dict(kind="predict", src=src, x=x))
            continue
        method = str(g.choice(["simpls", "plssvd", "opls", "kernelpls"], p=[0.5, 0.2, 0.15, 0.15]))
        n = int(np.exp(g.uniform(np.log(200), np.log(50000))))
        p = int(np.exp(g.uniform(np.log(500), np.log(50000))))
        if method == "kernelpls":
            n = min(n, 5000)
        m = int(g.integers(1, 11))
        cls = g.random() < 0.3
        x, t, gen = latent(n, p, 5, rid)
        if cls:
            m = int(g.integers(2, 21))
            c = torch.randn(5, m, generator=gen, device=t.device)
            lab = (torch.argmax(t @ c, dim=1)).cpu().numpy()
            present, lab = np.unique(lab, return_inverse=True)
            lab = (lab + 1).astype(np.int32)
            m = int(present.size)
            if m < 2:
                continue
            y = None
        else:
            c = torch.randn(5, m, generator=gen, device=t.device)
            y = (t @ c + 0.1 * torch.randn(n, m, generator=gen, device=t.device)).cpu().numpy()
            y = np.asfortranarray(y)
            lab = None
        cap = min(n - 1, p) if method != "kernelpls" else n - 1
        a = int(min(int(g.integers(2, 31)), cap))
        if method == "plssvd":
            a = max(1, min(a, m - 1 if cls else m))
        r = dict(kind="fit", method=method, x=x, y=y, labels=lab,
                 classes=m if cls else None, ncomp=a, p=p, q=m)
        reqs.append(r)
        fitted.append(r)
    del t
    torch.cuda.empty_cache()
    return reqs


def _kw(r):
    return dict(kernel="rbf", gamma=1.0 / r["p"]) if r["method"] == "kernelpls" else {}


def _describe(r):
    if r["kind"] != "fit":
        return f"predict rows={r['x'].shape[0]} p={r['src']['p']}"
    return (f"{r['method']} n={r['x'].shape[0]} p={r['p']} q={r['q']} a={r['ncomp']} "
            f"{'classification' if r['labels'] is not None else 'regression'}")


def run_plain(lib_api, reqs):
    """Each request through the drop-in entry points, one at a time. A
    request that fails is recorded (count, first message) and its
    predictions are skipped."""
    kw = _kw
    models = {}
    plain_lat = []
    failed = []
    t0 = time.perf_counter()
    for i, r in enumerate(reqs):
        s = time.perf_counter()
        try:
            if r["kind"] == "fit":
                models[id(r)] = lib_api.fit_resident(
                    r["x"], r["y"], labels=r["labels"], classes=r["classes"],
                    ncomp=r["ncomp"], method=r["method"], precision=32, **kw(r))
            else:
                src = r["src"]
                if id(src) in models:
                    models[id(src)].predict_path(r["x"], [src["ncomp"]])
        except Exception as exc:  # recorded in the bench line
            failed.append(f"{_describe(r)}: {exc}")
        plain_lat.append(1000 * (time.perf_counter() - s))
    plain_time = time.perf_counter() - t0
    for mdl in models.values():
        mdl.close()
    fits = sum(1 for r in reqs if r["kind"] == "fit")
    out = {"plain_fits_per_s": fits / plain_time,
           "plain_p50_ms": float(np.percentile(plain_lat, 50)),
           "plain_p99_ms": float(np.percentile(plain_lat, 99))}
    if failed:
        out["plain_failed"] = {"count": len(failed), "first": failed[0]}
    return out


def run_served(lib_api, reqs, mean_gap_ms=2.0, workers=4):
    """Served (continuous batching): Poisson arrivals into the server."""
    kw = _kw
    g = np.random.default_rng(3)
    gaps = g.exponential(mean_gap_ms / 1000.0, size=len(reqs))
    srv = lib_api.Server(budget_bytes=150 * 10**9, workers=workers)
    tickets = []
    fit_tickets = {}
    submit_t = []
    t0 = time.perf_counter()
    next_t = t0
    for i, r in enumerate(reqs):
        next_t += gaps[i]
        delay = next_t - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        if r["kind"] == "fit":
            t = srv.submit_fit(r["x"], r["y"], labels=r["labels"], classes=r["classes"],
                               ncomp=r["ncomp"], method=r["method"], precision=32, **kw(r))
            fit_tickets[id(r)] = t
        else:
            # queued behind its model's fit if that is still running
            src = r["src"]
            t = srv.submit_predict(fit_tickets[id(src)], r["x"], [src["ncomp"]])
        tickets.append(t)
        submit_t.append(time.perf_counter())
    lat = []
    failed = []
    for t in tickets:
        try:
            _, qms, sms = srv.wait(t)
            lat.append(qms + sms)
        except Exception as exc:  # recorded in the bench line
            failed.append(str(exc))
    served_time = time.perf_counter() - t0
    for t in fit_tickets.values():
        try:
            srv.release(t)
        except Exception:
            pass
    batches = srv.batch_stats()
    srv.close()
    fits = sum(1 for r in reqs if r["kind"] == "fit")
    out = {"mean_gap_ms": mean_gap_ms, "fits_per_s": fits / served_time,
           "p50_ms": float(np.percentile(lat, 50)) if lat else None,
           "p99_ms": float(np.percentile(lat, 99)) if lat else None,
           "batched_launches": batches["launches"], "batched_fits": batches["fits"]}
    if failed:
        out["failed"] = {"count": len(failed), "first": failed[0]}
    return out


def int8_peak_tops(torch, dev):
    """Dense int8 tensor-core throughput of this device, measured with the
    library GEMM torch._int_mm (cuBLAS) on 8192^3 int8 operands."""
    try:
        a = torch.randint(-127, 128, (8192, 8192), dtype=torch.int8, device=dev)
        b = torch.randint(-127, 128, (8192, 8192), dtype=torch.int8, device=dev)
        for _ in range(3):
            torch._int_mm(a, b)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        reps = 20
        e0.record()
        for _ in range(reps):
            torch._int_mm(a, b)
        e1.record()
        torch.cuda.synchronize(dev)
        return 2.0 * 8192 ** 3 * reps / (e0.elapsed_time(e1) * 1e-3) / 1e12, \
            "measured in this run (cuBLAS int8 GEMM via torch._int_mm, 8192^3)"
    except Exception as exc:  # no int8 library GEMM: nominal dense figure
        return 4500.0, f"nominal B200 dense int8 (library GEMM unavailable: {exc})"


def measured_peaks():
    """Roofline denominators: MEASURED_PEAKS.json (written per pod by the
    driver) when present, else the stated fallback of this GPU pool."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(path))
        hbm = float(d.get("hbm_gbs") or d.get("hbm_GBps") or 0) or None
        bf16 = float(d.get("bf16_tflops") or 0) or None
        if hbm:
            return {"hbm_gbs": hbm, "bf16_tflops": bf16, "source": "measured (MEASURED_PEAKS.json)"}
    except Exception:
        pass
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0,
            "source": "fallback (6.65 TB/s copy, 1.59 PFLOP/s bf16: earlier measurement on this pool)"}


def _errors_simpls(R, Q, T, ref, prefixes, pred=None, want_pred=None):
    from oracle import pls_oracle as O
    sg = np.where(np.einsum("ij,ij->j", R, ref["R"]) < 0.0, -1.0, 1.0)
    out = {"R": O.rel_err(R * sg, ref["R"]), "Q": O.rel_err(Q * sg, ref["Q"])}
    if T is not None:
        out["T"] = O.rel_err(T * sg, ref["T"])
    out["B"] = max(O.rel_err(R[:, :k] @ Q[:, :k].T, ref["R"][:, :k] @ ref["Q"][:, :k].T)
                   for k in prefixes)
    if pred is not None:
        out["Yhat"] = max(O.rel_err(pred[j], want_pred[j]) for j in range(len(prefixes)))
    return {k: float(v) for k, v in out.items()}


def _ref_predictions(ref, xp, prefixes):
    t = (xp - ref["centre"]) / ref["scale"] @ ref["R"]
    return [ref["ymean"] + t[:, :k] @ ref["Q"][:, :k].T for k in prefixes]


def leg_small_fits(fapi, with_ref, fits=100):
    """The plain FP64 SIMPLS configuration: n 500, p 2000, 3 responses, 10
    components (latent T 500 x 5, noise 0.5, seed 1): fits/s one fit at a
    time through fastpls_resident_simpls_create (host buffers), the device
    time of each fit, and errors against the reference FP64 core."""
    from fastpls_b200 import workloads as W
    n, p, m, a = 500, 2000, 3, 10
    x, y = W.latent_regression(n, p, m, 5, 0.5, 1, dtype=np.float64)
    pre = [1, 5, 10]
    for _ in range(5):
        fapi.fit_resident(x, y, ncomp=a, precision=64).close()
    dev_ms, lat = [], []
    t0 = time.perf_counter()
    for _ in range(fits):
        s = time.perf_counter()
        mdl = fapi.fit_resident(x, y, ncomp=a, precision=64)
        dev_ms.append(fapi.last_fit_times()["fit_ms"])
        mdl.close()
        lat.append(1000 * (time.perf_counter() - s))
    wall = time.perf_counter() - t0
    mdl = fapi.fit_resident(x, y, ncomp=a, precision=64)
    R, Q, T = (mdl.export(f).astype(np.float64) for f in (0, 1, 2))
    pred = mdl.predict_path(x, pre).astype(np.float64)
    mdl.close()
    out = {"workload": f"simpls_{n}x{p}_m{m}_ncomp{a}_f64", "fits": fits,
           "value": 1000.0 / float(np.mean(dev_ms)), "unit": "fits/s",
           "value_is": "inputs on the device (device time of the fit proper)",
           "e2e": {"value": fits / wall, "unit": "fits/s",
                   "p50_ms": float(np.percentile(lat, 50)),
                   "p99_ms": float(np.percentile(lat, 99)),
                   "h2d_bytes_per_fit": int(x.nbytes + y.nbytes)}}
    if with_ref:
        from oracle import ref
        cores = os.cpu_count() or 1
        ref.set_threads(cores)
        rr = ref.simpls_fit(x, y, ncomp=a)
        t0 = time.perf_counter()
        reps = 20
        for _ in range(reps):
            ref.simpls_fit(x, y, ncomp=a)
        dt = time.perf_counter() - t0
        out["errors_vs_fp64_reference"] = _errors_simpls(
            R, Q, T, rr, pre, pred, _ref_predictions(rr, x, pre))
        out["cpu_baseline"] = {"value": reps / dt, "unit": "fits/s", "cores": cores,
                               "kind": "reference", "sample": f"{reps} reference fits"}
    return out


def leg_plssvd_lda(fapi, peaks, with_ref):
    """The PLS-SVD + LDA configuration at full size: X 20000 x 50000 FP32
    (latent k = 20, scales 100 * 0.8^i, noise 0.1), 10 classes, ncomp capped
    at 9, oversample 10, power 2; LDA on the scores of 2000 rows. Device time
    of the fit against HBM (algorithmic bytes: the label cross-product pass
    and the score pass over X, 2 n p 4 bytes); labels against the reference's
    PLS-SVD + LDA (bit-exact)."""
    from fastpls_b200 import workloads as W
    n, p, classes, a = 20_000, 50_000, 10, 9
    x, lab = W.plssvd_lda_config(seed=2, n=n, p=p, k=20, classes=classes)
    pre = [1, 3, 5, 9]
    probe = np.arange(0, n, 10)
    xp = np.asfortranarray(x[probe])
    kw = dict(labels=lab, classes=classes, ncomp=a, method="plssvd", precision=32,
              oversample=10, power=2)
    fapi.fit_resident(x, **kw).close()
    fit_ms, copy_ms, walls = [], [], []
    for _ in range(3):
        t0 = time.perf_counter()
        mdl = fapi.fit_resident(x, **kw)
        t = fapi.last_fit_times()
        got = mdl.classify_path(xp, pre, lda=True)
        walls.append(time.perf_counter() - t0)
        fit_ms.append(t["fit_ms"])
        copy_ms.append(t["copy_ms"])
        mdl.close()
    fms = float(np.median(fit_ms))
    alg = 2.0 * n * p * 4
    achieved = alg / (fms * 1e-3) / 1e9
    out = {"workload": f"plssvd_lda_{n}x{p}_c{classes}_ncomp{a}_f32",
           "fit_ms": fms, "copy_ms": float(np.median(copy_ms)),
           "e2e_ms": 1000 * float(np.median(walls)),
           "e2e_is": "host buffers: H2D of X (4 GB) and labels, fit, LDA labels of 2000 rows",
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"],
                        "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
                        "algorithmic_bytes": alg, "peak_source": peaks["source"]}}
    if with_ref:
        from oracle import ref
        cores = os.cpu_count() or 1
        ref.set_threads(cores)
        x64 = np.asfortranarray(x, dtype=np.float64)
        del x
        t0 = time.perf_counter()
        rr = ref.plssvd_fit(x64, labels=lab, classes=classes, prefixes=pre, scaling=1,
                            oversample=10, power=2)
        tp = (x64[probe] - rr["centre"]) @ rr["R"]
        _, want = ref.lda(rr["T"], lab, classes, pre, tp)
        dt = time.perf_counter() - t0
        del x64
        out["labels_equal_reference"] = bool(all(
            np.array_equal(got[j][:, 0], want[:, j]) for j in range(len(pre))))
        out["label_differences"] = [int(np.sum(got[j][:, 0] != want[:, j]))
                                    for j in range(len(pre))]
        out["cpu_baseline"] = {"value": dt, "unit": "s per fit", "cores": cores,
                               "kind": "reference",
                               "sample": "one FP64 PLS-SVD fit + LDA labels of 2000 rows"}
    return out


def leg_mixed_precision(fapi, peaks, with_ref):
    """The mixed-precision configuration at full size: X 100000 x 20000 in
    BF16 (latent k = 50, column scales logN(0, 1)), 10 responses, 50
    components. Device time of the fit against HBM (algorithmic bytes:
    (1 + 2 a) n p 2, the cross-product pass and two passes per component),
    and the error of R, Q, T, B and predictions against the reference FP64
    core on the same BF16-rounded values."""
    from fastpls_b200 import workloads as W
    n, p, m, a = 100_000, 20_000, 10, 50
    bits, y = W.mixed_precision_config(seed=4, n=n, p=p, m=m, k=50)
    pre = [1, 10, 25, 50]
    rows = np.arange(0, n, 25)[:4000]
    fapi.fit_resident(bits, y, ncomp=a, precision=16).close()
    fit_ms, copy_ms, walls = [], [], []
    for _ in range(2):
        t0 = time.perf_counter()
        mdl = fapi.fit_resident(bits, y, ncomp=a, precision=16)
        walls.append(time.perf_counter() - t0)
        t = fapi.last_fit_times()
        fit_ms.append(t["fit_ms"])
        copy_ms.append(t["copy_ms"])
        if len(walls) < 2:
            mdl.close()
    pred = mdl.predict_path(bits[rows], pre).astype(np.float64)
    R, Q, T = (mdl.export(f).astype(np.float64) for f in (0, 1, 2))
    mdl.close()
    fms = float(np.median(fit_ms))
    alg = (1.0 + 2.0 * a) * n * p * 2
    achieved = alg / (fms * 1e-3) / 1e9
    out = {"workload": f"simpls_{n}x{p}_m{m}_ncomp{a}_bf16",
           "fit_ms": fms, "copy_ms": float(np.median(copy_ms)),
           "e2e_ms": 1000 * float(np.median(walls)),
           "e2e_is": "host buffers: H2D of X (4 GB BF16) and Y, the fit",
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"],
                        "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
                        "algorithmic_bytes": alg, "peak_source": peaks["source"]}}
    if with_ref:
        from oracle import ref
        cores = os.cpu_count() or 1
        ref.set_threads(cores)
        x64 = W.bf16_to_f64(bits)
        del bits
        t0 = time.perf_counter()
        rr = ref.simpls_fit(x64, y.astype(np.float64), ncomp=a, scaling=1)
        dt = time.perf_counter() - t0
        want = _ref_predictions(rr, x64[rows], pre)
        del x64
        out["errors_vs_fp64_reference"] = _errors_simpls(R, Q, T, rr, pre, pred, want)
        out["cpu_baseline"] = {"value": dt, "unit": "s per fit", "cores": cores,
                               "kind": "reference",
                               "sample": "one FP64 fit of the same BF16-rounded values"}
    return out


def workload_config(perms, digits=6, lanes=3):
    return {"workload": f"cv{FOLDS}_perm{perms}_ncomp{NCOMP}_{N}x{P}_f32",
            "n": N, "p": P, "q": Q, "folds": FOLDS, "fold_sizes": "480-520",
            "permutations": perms, "ncomp_path": f"1..{NCOMP}",
            "fits_per_step": (perms + 1) * FOLDS, "storage": "f32",
            "arithmetic": "f64", "method": "simpls", "scaling": "centering",
            "gram_products": (f"int8 split, {digits} digits per FP64 value "
                              "(tcgen05.mma kind::i8, exact int32 accumulation)"
                              if digits > 0 else "FP64 DMMA"),
            "l2": "inputs larger than L2 (X 200 MB FP32, Gram 200 MB FP64)",
            "parallelism": "replicas", "stream_lanes": lanes}


def main():
    a = args_parse()
    if a.impl == "reference":
        return run_reference_arm(a)

    import torch
    import torch.distributed as dist
    from fastpls_b200 import _lib

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    lib = _lib.load()
    dev = torch.device("cuda", local)

    # clock sampler: started now so that nvidia-smi's start-up is over before
    # the timed steps; only its samples inside the timed window are used
    clk_path = os.path.join(tempfile.gettempdir(), f"fpls_clocks_{rank}.csv")
    clk = clock_sampler_start(clk_path)
    x, y, folds, perms, prefixes = make_workload(rank, a.perms)
    Pn = perms.shape[0]
    fits_per_step = (Pn + 1) * FOLDS
    stream = torch.cuda.Stream(device=dev)
    lib.fastpls_b200_set_stream(C.c_void_p(stream.cuda_stream))

    Xd = torch.from_numpy(np.ravel(x, order="F").copy()).to(dev)
    Yd = torch.from_numpy(np.ravel(y, order="F").copy()).to(dev)
    Fd = torch.from_numpy(folds.astype(np.int32)).to(dev)
    Pd = torch.from_numpy(np.ascontiguousarray(perms, dtype=np.int32).ravel()).to(dev)
    k = len(prefixes)
    outs = [np.zeros((Pn + 1) * k) for _ in range(4)]
    status = np.zeros(FOLDS, dtype=np.int32)
    err, cap = _lib.error_buffer()

    def ptr(a_):
        return a_.ctypes.data_as(C.c_void_p)

    def step_device():
        rc = lib.fastpls_b200_simpls_cv_permutation_device(
            C.c_void_p(Xd.data_ptr()), C.c_void_p(Yd.data_ptr()),
            C.c_void_p(Fd.data_ptr()), C.c_void_p(Pd.data_ptr()), Pn, 32, N, P, Q,
            ptr(prefixes), k, 1, 3, *[ptr(o) for o in outs], ptr(status), err, cap)
        _lib.check(rc, err)

    # pinned host copies for the end-to-end (host-pointer ABI) measurement
    Xh = torch.from_numpy(np.ravel(x, order="F").copy()).pin_memory()
    Yh = torch.from_numpy(np.ravel(y, order="F").copy()).pin_memory()
    Ph = torch.from_numpy(np.ascontiguousarray(perms, dtype=np.int32).ravel()).pin_memory()
    folds32 = np.ascontiguousarray(folds, dtype=np.int32)

    def step_host():
        rc = lib.fastpls_b200_simpls_cv_permutation(
            C.c_void_p(Xh.data_ptr()), C.c_void_p(Yh.data_ptr()), ptr(folds32),
            C.c_void_p(Ph.data_ptr()), Pn, 32, N, P, Q, ptr(prefixes), k, 1, 3,
            *[ptr(o) for o in outs], ptr(status), err, cap)
        _lib.check(rc, err)

    def barrier():
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def max_over_ranks(v):
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    lib.fastpls_b200_set_product_digits(a.digits)
    digits = lib.fastpls_b200_product_digits()
    lib.fastpls_b200_set_batch_lanes(a.lanes)
    lanes = lib.fastpls_b200_batch_lanes()

    for _ in range(max(a.warmup, 3)):
        step_device()
    barrier()
    launches0 = lib.fastpls_b200_launch_count()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps + 1)]
    barrier()
    t_lo = time.time()
    ev[0].record(stream)
    for s in range(a.steps):
        step_device()
        ev[s + 1].record(stream)
    barrier()
    t_hi = time.time()
    launches = lib.fastpls_b200_launch_count() - launches0
    # at least the samples of the last 0.6 s for a very short timed region
    clocks = clock_sampler_stop(clk, clk_path, local, (min(t_lo, t_hi - 0.6), t_hi + 0.05))
    step_ms = [ev[s].elapsed_time(ev[s + 1]) for s in range(a.steps)]
    total_ms = max_over_ranks(ev[0].elapsed_time(ev[-1]))
    observed_q2 = outs[1].reshape(Pn + 1, k)[0].copy()
    all_q2 = outs[1].reshape(Pn + 1, k).copy()
    # step-latency distribution over more steps than the timed region (the
    # same step, device-timed one by one with CUDA events)
    lat_ms = list(step_ms)
    if a.latency_steps > 0:
        lev = [torch.cuda.Event(enable_timing=True) for _ in range(a.latency_steps + 1)]
        lev[0].record(stream)
        for s_ in range(a.latency_steps):
            step_device()
            lev[s_ + 1].record(stream)
        barrier()
        lat_ms += [lev[s_].elapsed_time(lev[s_ + 1]) for s_ in range(a.latency_steps)]
    sched = {}
    try:
        from fastpls_b200 import api as _fapi
        sched = _fapi.batched_stats()
    except Exception:
        pass

    # roofline of the dominant kernel: one more step with a single lane (the
    # products run alone, not overlapped with the other lane's kernels), each
    # product bracketed by CUDA events on its stream
    lib.fastpls_b200_set_batch_lanes(1)
    lib.fastpls_b200_profile_gemm(1)
    lib.fastpls_b200_profile_int8(1)
    r0 = torch.cuda.Event(enable_timing=True)
    r1 = torch.cuda.Event(enable_timing=True)
    r0.record(stream)
    step_device()
    r1.record(stream)
    barrier()
    lib.fastpls_b200_profile_gemm(0)
    lib.fastpls_b200_profile_int8(0)
    lib.fastpls_b200_set_batch_lanes(lanes)
    roof_step_ms = r0.elapsed_time(r1)
    gms, gfl, gl = C.c_double(0), C.c_double(0), C.c_ulonglong(0)
    lib.fastpls_b200_profile_gemm_read(C.byref(gms), C.byref(gfl), C.byref(gl))
    ims, iops, il = C.c_double(0), C.c_double(0), C.c_ulonglong(0)
    lib.fastpls_b200_profile_int8_read(C.byref(ims), C.byref(iops), C.byref(il))

    # the same step with FP64 DMMA products, for comparison (and the distance
    # of the int8 split path to it over every instance)
    fp64_leg = None
    if digits > 0 and a.fp64_steps > 0:
        lib.fastpls_b200_set_product_digits(0)
        step_device()
        barrier()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(a.fp64_steps):
            step_device()
        f1.record(stream)
        barrier()
        fms = max_over_ranks(f0.elapsed_time(f1)) / a.fp64_steps
        q2_fp64 = outs[1].reshape(Pn + 1, k).copy()
        lib.fastpls_b200_set_product_digits(digits)
        fp64_leg = {"value": world * fits_per_step / (fms / 1000.0), "unit": "fits/s",
                    "ms_per_step": fms, "steps": a.fp64_steps,
                    "q2_max_rel_diff_int8_vs_fp64_products": float(
                        np.max(np.abs(all_q2 - q2_fp64) / np.maximum(np.abs(q2_fp64), 1e-300)))}

    # end to end through the host-pointer ABI
    for _ in range(2):
        step_host()
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(a.steps):
        step_host()
    e1.record(stream)
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1)) / a.steps

    # the plain drop-in: one CV call per permutation through the reference's
    # regression CV entry point (per-fold fits, FP32 storage), sampled
    plain = None
    if a.plain_perms > 0:
        k_ = len(prefixes)
        pm_, q2_, rm_, r2_ = (np.zeros(k_) for _ in range(4))
        st_ = np.zeros(FOLDS, dtype=np.int32)
        xf = np.asfortranarray(x)
        yf = np.asfortranarray(y)
        fo = np.ascontiguousarray(folds, dtype=np.int32)

        def plain_call(b_):
            yb = yf if b_ == 0 else np.asfortranarray(yf[perms[b_ - 1]])
            rc = lib.fastpls_resident_simpls_cv_regression(
                ptr(xf), ptr(yb), ptr(fo), 32, N, P, Q, ptr(prefixes), k_, 1, 3,
                32, 5, C.c_ulonglong(1), 0, None, ptr(st_), ptr(pm_), ptr(q2_),
                ptr(rm_), ptr(r2_), err, cap)
            _lib.check(rc, err)
        plain_call(0)
        plain_q2_observed = q2_.copy()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for b_ in range(a.plain_perms):
            plain_call(b_)
        torch.cuda.synchronize(dev)
        dt = time.perf_counter() - t0
        plain_fits = a.plain_perms * FOLDS
        # one fold-sized fit alone: device time of the fit proper against the
        # HBM bound of its X passes ((1 + 2a) n_train p 4 bytes)
        from fastpls_b200 import api as _fapi
        tr = np.nonzero(fo != 1)[0]
        xtr, ytr = np.asfortranarray(xf[tr]), np.asfortranarray(yf[tr])
        for _ in range(2):
            _fapi.fit_resident(xtr, ytr, ncomp=NCOMP, precision=32).close()
        fms = []
        for _ in range(5):
            _fapi.fit_resident(xtr, ytr, ncomp=NCOMP, precision=32).close()
            fms.append(_fapi.last_fit_times()["fit_ms"])
        fold_ms = float(np.median(fms))
        fold_bytes = (1.0 + 2.0 * NCOMP) * len(tr) * P * 4
        pk = measured_peaks()
        fold_gbs = fold_bytes / (fold_ms * 1e-3) / 1e9
        plain = {"value": plain_fits / dt, "unit": "fits/s",
                 "fold_fit": {"shape": f"{len(tr)}x{P} f32, ncomp {NCOMP}",
                              "fit_ms": fold_ms,
                              "path": "persistent" if _fapi.persistent() else "per-kernel loop",
                              "roofline": {"bound": "hbm", "achieved": fold_gbs,
                                           "peak": pk["hbm_gbs"], "unit": "GB/s",
                                           "frac": fold_gbs / pk["hbm_gbs"],
                                           "algorithmic_bytes": fold_bytes,
                                           "peak_source": pk["source"]}},
                 "sample": f"{a.plain_perms} permutations x {FOLDS} folds through "
                           "fastpls_resident_simpls_cv_regression (one fold fit at a "
                           "time, FP32 storage, host buffers)",
                 "q2_path_max_abs_diff_vs_batched": float(
                     np.max(np.abs(plain_q2_observed - observed_q2)))}

    # measured FP64 FMA peak and int8 tensor peak (roofline denominators),
    # after every timed leg so that their bursts precede none of the timing
    pk64 = C.c_double(0)
    _lib.check(lib.fastpls_b200_fp64_peak(C.byref(pk64), err, cap), err)
    fp64_peak = pk64.value
    i8_peak, i8_source = int8_peak_tops(torch, dev)

    ms_per_step = total_ms / a.steps
    value = world * fits_per_step / (ms_per_step / 1000.0)
    achieved = gfl.value / (gms.value * 1e-3) / 1e12 if gms.value > 0 else None
    i8_achieved = iops.value / (ims.value * 1e-3) / 1e12 if ims.value > 0 else None
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get(
                "int8_split_traffic_bytes_per_launch" if digits > 0
                else "dgemm_traffic_bytes_per_launch")
        except Exception:
            traffic = None
    h2d = Xh.numel() * 4 + Yh.numel() * 4 + Ph.numel() * 4 + folds32.nbytes
    d2h = fits_per_step * (k + 1) * 8 + 4
    line = {
        "metric": METRIC, "value": value, "unit": "fits/s", "n_gpus": world,
        "steps": a.steps, "warmup": max(a.warmup, 3), "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic", "config": workload_config(Pn, digits, lanes),
        "latency_ms": {"p50": float(np.percentile(lat_ms, 50)),
                       "p99": float(np.percentile(lat_ms, 99)),
                       "p99_over_p50": float(np.percentile(lat_ms, 99) / np.percentile(lat_ms, 50)),
                       "steps_measured": len(lat_ms),
                       "timed_steps": [round(v, 3) for v in step_ms]},
        "schedule": sched,
        "e2e": {"value": world * fits_per_step / (e2e_ms / 1000.0), "unit": "fits/s",
                "ms_per_step": e2e_ms, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "roofline": ({"bound": "tensor", "kernel": "ozaki_gemm_kernel (int8 split "
                      "products, tcgen05.mma kind::i8, TMEM accumulators, TMA loads)",
                      "achieved": i8_achieved, "peak": i8_peak, "unit": "TOP/s (int8)",
                      "frac": (i8_achieved / i8_peak) if i8_achieved else None,
                      "peak_source": i8_source,
                      "launches": int(il.value),
                      "measured_on": "one single-lane step after the timed region",
                      "share_of_step": ims.value / roof_step_ms,
                      "fp64_equivalent_tflops": (i8_achieved / (digits * (digits + 1) / 2.0))
                      if i8_achieved else None,
                      "fp64_fma_peak_tflops": fp64_peak,
                      "traffic": traffic}
                     if digits > 0 else
                     {"bound": "fp64", "kernel": "dgemm_mma (FP64 DMMA tensor path)",
                      "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                      "frac": (achieved / fp64_peak) if achieved else None,
                      "peak_source": "measured in this run (FP64 FMA-chain probe); "
                                     "MEASURED_PEAKS.json has no FP64 figure",
                      "launches": int(gl.value),
                      "measured_on": "one single-lane step after the timed region",
                      "share_of_step": gms.value / roof_step_ms,
                      "traffic": traffic}),
        "fp64_products": fp64_leg,
        "gpu_launches": int(launches),
        "plain": plain,
        "batched_over_plain_e2e": (world * fits_per_step / (e2e_ms / 1000.0)) / plain["value"]
        if plain else None,
        "clocks": clocks,
    }
    if rank == 0 and a.served_requests > 0:
        from fastpls_b200 import api as fapi
        reqs = served_workload(a.served_requests)
        run_served(fapi, reqs[:20], mean_gap_ms=0.0, workers=8)  # warm-up
        plain = run_plain(fapi, reqs)
        sweep = [run_served(fapi, reqs, mean_gap_ms=g_, workers=8) for g_ in (2.0, 0.5, 0.0)]
        line["served"] = dict(
            requests=len(reqs), fits=sum(1 for r in reqs if r["kind"] == "fit"),
            workers=8, arrivals="Poisson; mean gap swept (0 = all at once); predictions "
                                "queue behind their model's fit in the server",
            sweep=sweep, **plain,
            saturated_served_over_plain=sweep[-1]["fits_per_s"] / plain["plain_fits_per_s"])
    if rank == 0 and a.served_spec_requests > 0:
        from fastpls_b200 import api as fapi
        reqs = served_spec_workload(a.served_spec_requests)
        nbytes = sum(r["x"].nbytes for r in reqs)
        plain_s = run_plain(fapi, reqs)
        sweep_s = [run_served(fapi, reqs, mean_gap_ms=g_, workers=8) for g_ in (20.0, 0.0)]
        fits_ = [r for r in reqs if r["kind"] == "fit"]
        line["served_spec"] = dict(
            requests=len(reqs), fits=len(fits_),
            input_gb=nbytes / 1e9,
            n_range=[int(min(r["x"].shape[0] for r in fits_)), int(max(r["x"].shape[0] for r in fits_))],
            p_range=[int(min(r["p"] for r in fits_)), int(max(r["p"] for r in fits_))],
            methods={m_: sum(1 for r in fits_ if r["method"] == m_)
                     for m_ in ("simpls", "plssvd", "opls", "kernelpls")},
            classification=sum(1 for r in fits_ if r["labels"] is not None),
            budget_gb=150, workers=8,
            arrivals="Poisson; mean gap 20 ms, then all at once",
            sweep=sweep_s, **plain_s,
            saturated_served_over_plain=sweep_s[-1]["fits_per_s"] / plain_s["plain_fits_per_s"])
        del reqs
    if rank == 0 and world == 1 and not a.no_configs:
        from fastpls_b200 import api as fapi
        from oracle import ref as _ref
        with_ref = _ref.available() and not a.no_cpu_baseline
        peaks = measured_peaks()
        line["configs"] = {
            "plain_fp64_simpls": leg_small_fits(fapi, with_ref),
            "plssvd_lda_full": leg_plssvd_lda(fapi, peaks, with_ref),
            "mixed_precision_bf16_full": leg_mixed_precision(fapi, peaks, with_ref),
        }
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu, ref_out = cpu_reference_sample(x, y, folds, prefixes)
        line["cpu_baseline"] = cpu
        if ref_out is not None:
            line["parity"] = {
                "observed_q2_max_rel_err_vs_fp64_reference": float(
                    np.max(np.abs(observed_q2 - ref_out["q2"]) /
                           np.maximum(np.abs(ref_out["q2"]), 1e-300)))}
    if rank == 0:
        print(json.dumps(line))
    lib.fastpls_b200_set_stream(None)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
