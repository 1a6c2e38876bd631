#!/usr/bin/env python
"""Benchmark of the B200 tree-learning path on the binary 10M-row workload.

Workload (seeded synthetic data, no public dataset): binary objective,
10,000,000 train + 1,000,000 held-out rows x 28 features (21 N(0,1) + 7
heavy-tailed products / ratios), max_bin 255, 255 leaves, learning rate 0.1,
500 rounds. A step is one boosting iteration (gradients, one tree grown on
the device, score updates of the training and held-out rows).

The line reports seconds per 500 rounds of the headline form (quantized
int8 gradients with int16/int32 histograms), the held-out AUC after 500
rounds of every form (FP64, FP32-compensated, quantized), the histogram
kernel's achieved HBM bandwidth against the measured peak, an end-to-end
figure through the C ABI with pinned host buffers, and the CPU oracle timed
on the host's cores.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "lightgbm-rust_b200"))

import numpy as np  # noqa: E402

WORKLOAD = ("binary 10M train + 1M held-out x 28 (21 N(0,1) + 7 heavy-tailed), max_bin 255, 255 leaves, lr 0.1, "
            "500 rounds; forms FP64, FP32-compensated, quantized (int8 g/h, 4 bins, stochastic rounding, FP64 leaf "
            "renewal)")
# DRAM bytes (read + write) per histogrammed row of the quantized histogram
# kernel, from one ncu capture of a 5M-row run (summarised under profiles/):
# the root launch, whose rows are in order, and the next launch, whose rows are
# scattered (each 32-byte row segment then comes with its neighbour sector).
# Traffic grows with the rows of a launch, so a tree's traffic is the root's
# rows times the first plus every other histogrammed row times the second.
HIST_DRAM_BYTES_PER_ROW_ROOT = 36.9
HIST_DRAM_BYTES_PER_ROW_SCATTERED = 69.6
# DRAM bytes per moved row of the partition kernel, from the ncu capture of its
# first launch in a 5M-row run (the root split: every row; summarised under profiles/).
# The index writes stay in L2 during the launch, so this is below the 9 algorithmic bytes.
PART_DRAM_BYTES_PER_ROW = 5.02
METRIC = "s per 500 rounds (quantized hist, equal AUC to FP64) + hist GB/s"
ROUNDS = 500


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, device):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(device), f"--query-gpu={q}", "--format=csv,noheader",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1].split()[0]))
                mx.append(float(parts[2].split()[0]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.f.name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def _auc(y, s):
    """AUC with tied scores sharing credit (metric.rs:701-731)."""
    order = np.argsort(-s, kind="mergesort")
    y = y[order]
    s = s[order]
    pos = (y > 0).astype(np.float64)
    neg = 1.0 - pos
    starts = np.r_[0, np.nonzero(np.diff(s))[0] + 1]
    cp = np.add.reduceat(pos, starts)
    cn = np.add.reduceat(neg, starts)
    before = np.cumsum(cp) - cp
    acc = float(np.sum(cn * (cp * 0.5 + before)))
    tp = float(pos.sum())
    return acc / (tp * (len(s) - tp)) if 0 < tp < len(s) else 1.0


def _barrier():
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def _max_over_ranks(v):
    """The largest of every rank's value (the job's time is its slowest rank's)."""
    import torch
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())
    return v


def hist_bytes_per_row(nf, form):
    """Algorithmic bytes one histogram row costs: its bin row, its gradient
    pair (8 B f32 g/h, or the 4 B packed quantized pair) and its u32 row index."""
    return nf * 1 + (4 if form == "quantized" else 8) + 4


def hist_rows_by_step(t):
    """Rows each split step's histogram launch reads: step 0 the root (every
    row of the tree), step s the smaller child of split s - 1 (the split
    order is the node order)."""
    def count(c):
        return int(t["internal_count"][c]) if c >= 0 else int(t["leaf_count"][~c])

    nl = int(t["num_leaves"])
    if nl < 2:
        return []
    out = [int(np.sum(t["leaf_count"]))]
    for k in range(nl - 2):
        out.append(min(count(int(t["left_child"][k])), count(int(t["right_child"][k]))))
    return out


def hist_by_rows(step_rows, step_ms, bytes_per_row):
    """Histogram launches binned by the rows they read: launches, mean us per
    launch, and GB/s of algorithmic bytes (rows x bytes per row) per bin."""
    edges = [0, 1_000, 10_000, 100_000, 1_000_000, 10**12]
    out = []
    r = np.asarray(step_rows, np.float64)
    ms = np.asarray(step_ms, np.float64)
    for lo, hi in zip(edges[:-1], edges[1:]):
        sel = (r >= lo) & (r < hi)
        if not np.any(sel):
            continue
        t = float(ms[sel].sum()) / 1000.0
        out.append({"rows_from": lo, "rows_to": hi if hi < 10**12 else None, "launches": int(sel.sum()),
                    "us_per_launch": 1e6 * t / int(sel.sum()),
                    "gbs": float(r[sel].sum()) * bytes_per_row / t / 1e9 if t > 0 else None})
    return out


def _shape_key(args, form):
    """Key of a workload's tuned launch shape: workload, scale, histogram form."""
    return f"{args.workload}{'' if args.scale == 1.0 else '@' + format(args.scale, 'g')}/{form}"


def launch_shape_before(L, key, use_record, device):
    """The learner's launch shape before warm-up: the recorded tuned shape of
    this workload when `use_record` and there is one for this device."""
    import torch

    from lgbm_b200 import autotune

    if use_record:
        shape = autotune.lookup(key, torch.cuda.get_device_properties(device).multi_processor_count)
        if shape is not None:
            L.launch_shape = shape
            return L.launch_shape, "tuned (lgbm_b200/launch_shapes.json)"
    return L.launch_shape, "built-in defaults"


def launch_shape_tune(L, key, device):
    """--autotune: search the shapes on the warmed-up learner and record the choice."""
    import torch

    from lgbm_b200 import autotune

    props = torch.cuda.get_device_properties(device)
    default = L.launch_shape
    best, best_ms, default_ms, trials = autotune.tune(L, reps=3)
    autotune.record(key, best, best_ms, default, default_ms, trials, props.name, props.multi_processor_count)
    return L.launch_shape, "autotuned in this run"


def run_form(lgb, data, ds, dv, form, args, device):
    params = dict(data["params"], hist_precision=form, device=device, num_threads=os.cpu_count() or 8,
                  use_cuda_graph=True)
    if form == "quantized":  # the workload's quantized form renews leaf outputs from FP64 gradients
        params["quant_train_renew_leaf"] = True
    bst = lgb.Booster(params, ds, dv)
    L = bst.learner
    key = _shape_key(args, form)
    shape, shape_src = launch_shape_before(L, key, not args.autotune, device)
    for _ in range(args.warmup):
        bst.update()
    extra = 0
    if args.autotune:
        shape, shape_src = launch_shape_tune(L, key, device)
        bst.update()  # captures the tuned launches before the timed steps
        extra = 1
    _barrier()
    L.record(0)
    clocks = Clocks(device)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        bst.update()
    L.record(1)
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    ms = L.elapsed(0, 1) / args.steps
    # histogram kernel timing over the same number of steps, events around every launch
    L.set_timing(True)
    hist_ms = scan_ms = part_ms = 0.0
    rows = prows = 0
    launches = 0
    step_rows, step_hist_ms = [], []
    for _ in range(args.steps):
        bst.update()
        t, r, nl = L.last_timing()
        _, pr = L.last_rows()
        hist_ms += t[0]
        scan_ms += t[1]
        part_ms += t[2]
        rows += r
        prows += pr
        launches = nl
        st = L.step_times()
        rr = hist_rows_by_step(bst.trees[-1])
        step_rows.extend(rr)
        step_hist_ms.extend(st[: len(rr), 0])
    L.set_timing(False)
    done = args.warmup + extra + 2 * args.steps
    for _ in range(max(0, args.rounds - done)):
        if bst.update():
            break
    sv = bst.scores(valid=True)[0]
    t0 = time.perf_counter()
    auc = _auc(data["y_valid"], sv)
    auc_numpy_ms = 1000 * (time.perf_counter() - t0)
    # the same AUC on the device (lgbm_b200_metric_eval: host scores in, copies included)
    lgb.metric("auc", data["y_valid"], sv, device=device)  # warm-up: sizes the device workspace
    t0 = time.perf_counter()
    auc_device = lgb.metric("auc", data["y_valid"], sv, device=device)
    auc_device_ms = 1000 * (time.perf_counter() - t0)
    nf = ds.binned()["num_features"]
    steps_per_tree = int(params["num_leaves"]) - 1
    hist_launches = args.steps * steps_per_tree
    hist_bytes = rows * hist_bytes_per_row(nf, form)
    # the partition moves each row of the split leaf: index in, its byte of the
    # split feature (column copy), index out
    part_bytes = prows * (4 + 1 + 4)
    return {
        "ms_per_step": ms, "wall_ms_per_step": 1000 * wall / args.steps, "s_per_500": ms * ROUNDS / 1000.0,
        "auc": auc, "auc_device": auc_device, "auc_device_ms": auc_device_ms, "auc_numpy_ms": auc_numpy_ms,
        "hist_ms_per_launch": hist_ms / hist_launches, "hist_gbs": hist_bytes / (hist_ms / 1000) / 1e9,
        "hist_bytes_per_launch": hist_bytes / hist_launches, "hist_rows_per_tree": rows / args.steps,
        "scan_ms_per_step": scan_ms / args.steps, "partition_ms_per_step": part_ms / args.steps,
        "part_rows_per_tree": prows / args.steps,
        "part_gbs": part_bytes / (part_ms / 1000) / 1e9 if part_ms > 0 else None,
        "part_bytes_per_launch": part_bytes / (args.steps * steps_per_tree),
        "part_ms_per_launch": part_ms / (args.steps * steps_per_tree),
        "hist_ms_per_step": hist_ms / args.steps, "kernel_launches_per_tree": launches, "clocks": clk,
        "num_trees": bst.num_trees(), "nf": nf, "launch_shape": shape, "launch_shape_source": shape_src,
        "hist_by_rows": hist_by_rows(step_rows, step_hist_ms, hist_bytes_per_row(nf, form)),
    }


def run_e2e(lgb, data, ds, form, args, device):
    """The drop-in call sequence with host buffers: RowObjective::gradients,
    SerialTreeLearner::train and add_leaf_outputs through the C ABI, with
    pinned host memory and every host<->device copy inside the timed region."""

    import torch

    from lgbm_b200.basic import resolve_params

    params = dict(data["params"], hist_precision=form, device=device, num_threads=os.cpu_count() or 8)
    if form == "quantized":
        params["quant_train_renew_leaf"] = True
    p = resolve_params(params)
    learner = lgb.Learner(ds, params)
    launch_shape_before(learner, _shape_key(args, form), True, device)  # recorded by run_form when --autotune
    n = len(data["y"])
    pin = lambda shape, dt: torch.empty(shape, dtype=dt, pin_memory=True).numpy()  # noqa: E731
    label = pin(n, torch.float32)
    label[:] = data["y"]
    score = pin(n, torch.float64)
    pavg = min(max(float(np.mean(data["y"] > 0)), 1e-15), 1 - 1e-15)
    score[:] = np.log(pavg / (1 - pavg))
    g = pin(n, torch.float32)
    h = pin(n, torch.float32)
    lr = float(p["learning_rate"])

    parts = np.zeros(3)

    # the objective holds the labels on the device (RowObjective::init);
    # every step moves the scores in and the gradients out
    obj = lgb.Objective(dict(params), label)

    def step():
        t0 = time.perf_counter()
        obj.gradients(score, g, h)
        t1 = time.perf_counter()
        t = learner.train(g, h)[0]
        t2 = time.perf_counter()
        lv = np.where(np.abs(t["leaf_value"] * lr) <= np.float32(1e-35), 0.0, t["leaf_value"] * lr)
        learner.add_leaf_outputs(0, lv, score)
        parts[:] += (t1 - t0, t2 - t1, time.perf_counter() - t2)

    for _ in range(args.warmup):
        step()
    parts[:] = 0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    ms = 1000 * (time.perf_counter() - t0) / args.steps
    return {"value": ms * ROUNDS / 1000.0, "unit": "s/500 rounds", "ms_per_step": ms,
            "ms_gradients": 1000 * parts[0] / args.steps, "ms_train": 1000 * parts[1] / args.steps,
            "ms_add_leaf_outputs": 1000 * parts[2] / args.steps,
            # gradients: scores in, g/h out; train: g/h in; add_leaf_outputs: scores in and out
            "h2d_bytes_per_step": n * 8 + n * 8 + n * 8, "d2h_bytes_per_step": n * 8 + n * 8}


def _oracle_sample(lgb, form, sample_scale, threads):
    """The oracle's booster on a bounded sample of the workload, binned by the
    oracle's own restatement of the reference's binning (no product code)."""
    from lgbm_b200 import synthetic
    from oracle import oracle as orc

    d = synthetic.make(2, scale=sample_scale)
    params = dict(d["params"], hist_precision=form, num_threads=threads)
    if form == "quantized":
        params["quant_train_renew_leaf"] = True
    p = lgb.resolve_params(params)
    od = orc.Dataset(d["X"], p)
    return orc.train(p, od.binned(), d["y"], 0), len(d["y"])


def run_cpu_baseline(lgb, form, sample_scale, iters, warmup=3, threads=None):
    """The oracle (the reference's CPU learner restated) on the host cores, on
    a bounded sample of the workload: `warmup` boosting iterations, then
    `iters` iterations timed one by one; seconds per 500 rounds scaled to the
    full row count."""
    threads = threads or os.cpu_count() or 8
    m, rows = _oracle_sample(lgb, form, sample_scale, threads)
    for _ in range(warmup):
        m.update()
    per = []
    for _ in range(iters):
        t0 = time.perf_counter()
        m.update()
        per.append(time.perf_counter() - t0)
    per_iter = float(np.mean(per))
    scale = 10_000_000 / rows
    return {"value": per_iter * scale * ROUNDS, "unit": "s/500 rounds", "cores": threads, "kind": "port",
            "sample": f"{rows} rows of the same generator (binned by the oracle), {iters} boosting iterations timed "
                      f"one by one after {warmup} warm-up ones ({form} form, {threads} threads); the mean "
                      f"iteration time scaled by {scale:.0f}x rows and x{ROUNDS} rounds", "warmup": warmup,
            "ms_per_iter_sample": 1000 * per_iter}


def _ndcg_at(y, s, group, k):
    """Mean NDCG@k over queries (dcg.rs: gains 2^label - 1, discounts 1/log2(2 + rank),
    stable descending order of the scores); queries without relevant rows count 1."""
    q = np.repeat(np.arange(len(group)), group)
    order = np.lexsort((np.arange(len(s)), -s, q))
    start = np.r_[0, np.cumsum(group)[:-1]]
    rank = np.arange(len(s)) - np.repeat(start, group)
    gain = (2.0 ** y.astype(np.float64)) - 1.0
    disc = 1.0 / np.log2(2.0 + rank)
    top = rank < k
    dcg = np.bincount(q, weights=np.where(top, gain[order] * disc, 0.0), minlength=len(group))
    ideal_order = np.lexsort((-y, q))
    idcg = np.bincount(q, weights=np.where(top, gain[ideal_order] * disc, 0.0), minlength=len(group))
    return float(np.mean(np.where(idcg > 0, dcg / np.where(idcg > 0, idcg, 1.0), 1.0)))


def run_workload(args, workload=None, predict_trees=None, compare_binning=True):
    """The other benchmark configurations: device time per boosting iteration
    of each form on the seeded synthetic data, a quality figure after the
    timed rounds, and (lambdarank) the batched prediction of a trained model
    over every row. Returns one dict (not the headline metric)."""
    import lgbm_b200 as lgb
    from lgbm_b200 import synthetic

    cfg = {"c1": 1, "c3": 3, "c4": 4}[workload or args.workload]
    d = synthetic.make(cfg, scale=args.scale)
    forms = [f for f in args.forms.split(",") if f] if args.forms != "quantized,f32c,f64" else (
        ["f64", "f32c"] if cfg == 1 else ["quantized", "f64"])
    params = dict(d["params"])
    params.pop("categorical_feature", None)
    params.pop("eval_at", None)
    for kv in args.param:
        k, v = kv.split("=", 1)
        try:
            params[k] = json.loads(v)
        except ValueError:
            params[k] = v
    build_s = same = None
    if compare_binning:
        t0 = time.perf_counter()
        ds = lgb.Dataset(d["X"], d["y"], group=d.get("group"), params=params,
                         categorical_feature=d.get("categorical")).construct(params)
        build_s = time.perf_counter() - t0
    # the same dataset with its rows binned on the device (identical bytes)
    t0 = time.perf_counter()
    ds_dev = lgb.Dataset(d["X"], d["y"], group=d.get("group"), params=dict(params, device_binning=True),
                         categorical_feature=d.get("categorical")).construct(dict(params, device_binning=True))
    build_dev_s = time.perf_counter() - t0
    if compare_binning:
        same = bool(np.array_equal(ds.binned()["bins"], ds_dev.binned()["bins"]))
        del ds_dev
    else:
        ds = ds_dev
    out = {"workload": d["name"], "rows": int(len(d["y"])), "features": int(d["X"].shape[1]),
           "rounds_in_config": d["num_rounds"], "dataset_build_s": build_s,
           "dataset_build_device_binning_s": build_dev_s, "device_binning_identical": same, "forms": {}}
    for form in forms:
        p = dict(params, hist_precision=form, num_threads=os.cpu_count() or 8)
        if form == "quantized":
            p["quant_train_renew_leaf"] = True
        bst = lgb.Booster(p, ds)
        L = bst.learner
        key = _shape_key(args, form)
        shape, shape_src = launch_shape_before(L, key, not args.autotune, 0)
        for _ in range(args.warmup):
            bst.update()
        extra = 0
        if args.autotune:
            shape, shape_src = launch_shape_tune(L, key, 0)
            bst.update()  # captures the tuned launches before the timed steps
            extra = 1
        L.record(0)
        for _ in range(args.steps):
            bst.update()
        L.record(1)
        ms = L.elapsed(0, 1) / args.steps
        # device time per kernel family over a few more iterations (events around every launch)
        L.set_timing(True)
        fam = np.zeros(3)
        timed = 3
        for _ in range(timed):
            bst.update()
            t, _, _ = L.last_timing()
            fam += np.asarray(t[:3])
        L.set_timing(False)
        sc = bst.scores()
        rounds = args.warmup + extra + args.steps + timed
        r = {"ms_per_iter": ms, "s_per_config_rounds": ms * d["num_rounds"] / 1000.0, "rounds_trained": rounds,
             "launch_shape": shape, "launch_shape_source": shape_src,
             "kernel_ms_per_iter": {"hist": fam[0] / timed, "scan": fam[1] / timed, "partition": fam[2] / timed}}
        y = d["y"]
        if cfg == 1:
            r["train_rmse"] = float(np.sqrt(np.mean((sc[0] - y) ** 2)))
        elif cfg == 3:
            z = sc.T - sc.T.max(axis=1, keepdims=True)
            lp = z - np.log(np.exp(z).sum(axis=1, keepdims=True))
            r["train_multi_logloss"] = float(-np.mean(lp[np.arange(len(y)), y.astype(int)]))
        else:
            t0 = time.perf_counter()
            r["train_ndcg@10"] = _ndcg_at(y, sc[0], d["group"], 10)
            r["ndcg_numpy_s"] = time.perf_counter() - t0
            t0 = time.perf_counter()
            r["train_ndcg@10_device"] = float(lgb.ndcg(y, sc[0], d["group"], [10])[0])
            r["ndcg_device_s"] = time.perf_counter() - t0
            if form == forms[0]:
                # batched raw prediction of the model over every row, after
                # training it to `predict_trees` trees (the config's 300)
                want = predict_trees or bst.num_trees()
                while bst.num_trees() < want:
                    if bst.update():
                        break
                r["predict"] = predict_bench(lgb, bst, d["X"])
        out["forms"][form] = r
        del bst
    return out


def predict_bench(lgb, bst, X):
    """Batched prediction (lgbm_b200_predict) of a booster's trees over the
    rows X: kernel-only (rows already in device memory) and from host rows
    (copies included). Node visits are counted from the trees' leaf depths and
    training counts, exact when X holds the training rows (no bagging)."""
    import ctypes as C

    import torch

    L = lgb._lib
    n, ncol = X.shape
    k = bst.num_class
    visits = sum(int(np.sum(t["leaf_count"].astype(np.int64) * t["leaf_depth"])) for t in bst.trees)
    fh = bst._forest_handle()
    xd = torch.from_numpy(X).cuda()
    od = torch.empty(n * k, dtype=torch.float64, device="cuda")
    L.check(L.lib().lgbm_b200_predict(fh, C.c_void_p(xd.data_ptr()), n, ncol, C.c_void_p(od.data_ptr()), L.DEVICE))
    torch.cuda.synchronize()
    reps = 3
    t0 = time.perf_counter()
    for _ in range(reps):  # each call synchronises the forest's stream
        L.check(L.lib().lgbm_b200_predict(fh, C.c_void_p(xd.data_ptr()), n, ncol, C.c_void_p(od.data_ptr()),
                                          L.DEVICE))
    dev_s = (time.perf_counter() - t0) / reps
    del xd
    bst.predict(X[:1000], raw_score=True)
    t0 = time.perf_counter()
    host_out = bst.predict(X, raw_score=True)
    host_s = time.perf_counter() - t0
    same = bool(np.array_equal(np.asarray(host_out).reshape(-1), od.cpu().numpy()))
    first_touch = n * ncol * 4 + 8 * n * k
    return {"rows": int(n), "trees": bst.num_trees(), "kernel_s": dev_s, "rows_per_s": n / dev_s,
            "node_visits": visits, "node_visits_per_s": visits / dev_s, "first_touch_gbs": first_touch / dev_s / 1e9,
            "host_rows_s": host_s, "host_rows_per_s": n / host_s, "device_equals_host": same,
            "note": "kernel_s: rows already on the device (one launch per call); host_rows_s: f32 rows from host "
                    "memory, f64 scores back, copies included"}


def _logloss(y, score):
    """Mean binary logloss of raw scores (sigmoid 1)."""
    pr = 1.0 / (1.0 + np.exp(-score))
    pr = np.clip(pr, 1e-15, 1 - 1e-15)
    return float(-np.mean(y * np.log(pr) + (1 - y) * np.log(1 - pr)))


def run_auc_seeds(lgb, args, device, res, seeds=(3, 4, 5, 6)):
    """Held-out AUC after the workload's 500 rounds, quantized and FP64, on the
    headline seed (from the main run) and four more seeds of the same
    generator at full size: is the quantized form's AUC gap seed noise?"""
    from lgbm_b200 import synthetic

    out = [{"seed": 2, "auc_quantized": res["quantized"]["auc"], "auc_f64": res["f64"]["auc"]}]
    for seed in seeds:
        d = synthetic.make(2, scale=args.scale, seed=seed)
        ds = lgb.Dataset(d["X"], d["y"], params=d["params"]).construct()
        dv = lgb.Dataset(d["X_valid"], d["y_valid"], params=d["params"], reference=ds).construct()
        row = {"seed": seed}
        for form in ("quantized", "f64"):
            params = dict(d["params"], hist_precision=form, device=device, num_threads=os.cpu_count() or 8)
            if form == "quantized":
                params["quant_train_renew_leaf"] = True
            bst = lgb.Booster(params, ds, dv)
            for _ in range(args.rounds):
                if bst.update():
                    break
            row[f"auc_{form}"] = _auc(d["y_valid"], bst.scores(valid=True)[0])
            del bst
        out.append(row)
        del ds, dv, d
    deltas = np.array([r["auc_quantized"] - r["auc_f64"] for r in out])
    return {"rounds": args.rounds, "per_seed": out, "delta_mean": float(deltas.mean()),
            "delta_std": float(deltas.std(ddof=1)), "delta_max_abs": float(np.abs(deltas).max()),
            "note": "held-out AUC of the quantized form minus the FP64 form's, same data and rounds"}


def run_precision(lgb, device, scale=0.02, rounds=50, checkpoints=(0, 10, 25)):
    """Error of the FP32-compensated and quantized forms against the FP64
    oracle on the 10M-row workload's generator at `scale` (200k + 20k rows):
    histogram relative error (all rows, the gradients of each checkpoint),
    split agreement and leaf-value error of one tree grown on the same
    gradients, and the held-out AUC / logloss after `rounds` rounds."""
    from lgbm_b200 import synthetic
    from oracle import oracle as orc

    d = synthetic.make(2, scale=scale)
    base = dict(d["params"], device=device, num_threads=16)
    p64 = lgb.resolve_params(dict(base, hist_precision="f64"))
    ds = lgb.Dataset(d["X"], d["y"], params=base).construct()
    dv = lgb.Dataset(d["X_valid"], d["y_valid"], params=base, reference=ds).construct()
    b = ds.binned()
    om = orc.train(p64, b, d["y"], 0, valid_binned=dv.binned())
    grads = {}
    for it in range(rounds):
        if it in checkpoints:
            grads[it] = orc.gradients(p64, d["y"], om.scores()[0])
        om.update()
    auc64 = orc.auc(d["y_valid"], om.scores(valid=True)[0])
    ll64 = _logloss(d["y_valid"], om.scores(valid=True)[0])
    out = {"rows": int(len(d["y"])), "held_out_rows": int(len(d["y_valid"])), "rounds": rounds,
           "checkpoints": list(checkpoints), "oracle_f64": {"auc": auc64, "logloss": ll64}, "forms": {}}
    for form in ("f64", "f32c", "quantized"):
        params = dict(base, hist_precision=form)
        if form == "quantized":
            params.update(quant_train_renew_leaf=True)
        pf = lgb.resolve_params(params)
        learner = lgb.Learner(ds, params)
        herr_max, herr_mean, agree, nodes, ident, lv_err = [], [], 0, 0, 0, []
        for it, (g, h) in grads.items():
            t = learner.train(g, h)[0]
            want = orc.hist(b, None, g, h).reshape(-1, 2)
            got = learner.histogram(None)
            if form == "quantized":
                _, scales = learner.quantized()
                hi = got & 0xFFFFFFFF
                gi = (got - hi) >> 32
                got = np.stack([gi * scales[0], hi * scales[1]], axis=1)
            else:
                got = got.reshape(-1, 2)
            # relative to the histogram's magnitude (L1 over every cell, g and
            # h apart): per-cell ratios are meaningless on cells near zero
            rel = np.abs(got - want).sum(axis=0) / np.abs(want).sum(axis=0)
            herr_max.append(float(rel.max()))
            herr_mean.append(float(rel.mean()))
            ot = orc.train_trees(p64, b, g, h).trees[0]
            nn = min(t["num_leaves"], ot["num_leaves"]) - 1
            same = (t["split_feature"][:nn] == ot["split_feature"][:nn]) & \
                   (t["threshold_in_bin"][:nn] == ot["threshold_in_bin"][:nn])
            agree += int(np.sum(same))
            nodes += ot["num_leaves"] - 1
            if t["num_leaves"] == ot["num_leaves"] and bool(np.all(same)):
                ident += 1
                lv_err.append(np.abs(t["leaf_value"] - ot["leaf_value"]) /
                              np.maximum(np.abs(ot["leaf_value"]), 1e-300))
        lv = np.concatenate(lv_err) if lv_err else np.zeros(0)
        bst = lgb.Booster(params, ds, dv)
        for _ in range(rounds):
            if bst.update():
                break
        sv = bst.scores(valid=True)[0]
        auc = orc.auc(d["y_valid"], sv)
        out["forms"][form] = {
            "hist_rel_err_l1_max": max(herr_max), "hist_rel_err_l1_mean": float(np.mean(herr_mean)),
            "split_agreement": agree / max(nodes, 1), "identical_trees": ident, "trees_compared": len(grads),
            "leaf_rel_err_max": float(lv.max()) if lv.size else None,
            "leaf_rel_err_mean": float(lv.mean()) if lv.size else None,
            "auc": auc, "auc_delta_vs_oracle_f64": auc - auc64,
            "logloss_delta_vs_oracle_f64": _logloss(d["y_valid"], sv) - ll64}
        del bst, learner
    out["note"] = ("one tree per checkpoint grown by each form and by the FP64 oracle on the same gradients (the "
                   "FP64 oracle run's at that iteration); histogram error = sum |form - oracle| / sum |oracle| over "
                   "all cells of the root histogram (max over g / h and checkpoints); split agreement = splits "
                   "equal in node order / oracle splits; leaf error over the trees whose structure is identical")
    return out


def run_config0(lgb, device):
    """The CPU-runnable binary workload end to end at its exact settings
    (20k + 5k rows x 28, 31 leaves, min_data_in_leaf 20, lr 0.1, 100 rounds,
    FP64 histograms) on the GPU and in the oracle: identical trees, held-out
    AUC / logloss, and the model text of both."""
    from lgbm_b200 import synthetic
    from oracle import oracle as orc

    d = synthetic.config0()
    params = dict(d["params"], device=device)
    p = lgb.resolve_params(params)
    ds = lgb.Dataset(d["X"], d["y"], params=params)
    dv = lgb.Dataset(d["X_valid"], d["y_valid"], params=params, reference=ds)
    ds.construct()
    dv.construct()
    t0 = time.perf_counter()
    bst = lgb.train(params, ds, d["num_rounds"], valid_sets=[dv])
    gpu_s = time.perf_counter() - t0
    od = orc.Dataset(d["X"], p)
    odv = orc.Dataset(d["X_valid"], p, reference=od)
    bins_equal = bool(np.array_equal(ds.binned()["bins"], od.binned()["bins"]) and
                      np.array_equal(dv.binned()["bins"], odv.binned()["bins"]))
    t0 = time.perf_counter()
    om = orc.train(p, od.binned(), d["y"], d["num_rounds"], valid_binned=odv.binned())
    orc_s = time.perf_counter() - t0
    same = 0
    for a, o in zip(bst.trees, om.trees):
        if not (a["num_leaves"] == o["num_leaves"] and np.array_equal(a["split_feature"], o["split_feature"]) and
                np.array_equal(a["threshold_in_bin"], o["threshold_in_bin"])):
            break
        same += 1
    lv = [np.max(np.abs(a["leaf_value"] - o["leaf_value"]) / np.maximum(np.abs(o["leaf_value"]), 1e-300))
          for a, o in zip(bst.trees[:same], om.trees[:same])]
    sg, so = bst.scores(valid=True)[0], om.scores(valid=True)[0]
    tg = bst.model_to_string()
    to = om.model_to_string(d["X"].shape[1], od.feature_infos)
    lg, lo = tg.split("\n"), to.split("\n")
    return {"rows": len(d["y"]), "held_out_rows": len(d["y_valid"]), "rounds": d["num_rounds"],
            "bins_equal_oracle_binning": bins_equal, "trees": len(bst.trees), "identical_trees": same,
            "leaf_rel_err_max": float(max(lv)) if lv else None,
            "auc_gpu": orc.auc(d["y_valid"], sg), "auc_oracle": orc.auc(d["y_valid"], so),
            "logloss_gpu": _logloss(d["y_valid"], sg), "logloss_oracle": _logloss(d["y_valid"], so),
            "model_text_identical": tg == to, "model_text_bytes": len(tg),
            "model_text_lines_differing": int(sum(a != b for a, b in zip(lg, lo)) + abs(len(lg) - len(lo))),
            "gpu_s": gpu_s, "oracle_1t_s": orc_s}


def config_dict(head, world, rows, held_out):
    """The workload's config, the same in both arms."""
    return {"workload": WORKLOAD, "form": head, "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (bin matrix 320 MB, gradients 80 MB)", "rows": rows,
            "held_out_rows": held_out}


def run_reference_arm(args, world):
    """--impl reference: the reference's CPU learner (restated by the oracle:
    the reference is Rust and no Rust toolchain is available) on the host's
    cores, binned by the oracle's own binning, so no product code runs. A step
    is one boosting iteration of a 1M-row sample of the workload (the same
    generator); W warm-up iterations, then exactly K timed ones. The value is
    the mean iteration time scaled to the 10M-row workload and 500 rounds.
    A single-threaded run of the same restatement on a smaller sample
    (cpu_ref_1t) is reported beside it."""
    import lgbm_b200 as lgb  # the Python package only: the product library is never loaded here

    t0 = time.perf_counter()
    threads = os.cpu_count() or 8
    cb = run_cpu_baseline(lgb, "quantized", 0.1 * args.scale, args.steps, args.warmup, threads)
    one = run_cpu_baseline(lgb, "quantized", 0.01, 2, 1, 1)
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "s/500 rounds",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": cb["value"] / ROUNDS * 1000, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "int8", "data": "synthetic (seeded generator with the workload's shapes and "
            "distributions)", "config": config_dict("quantized", world, 10_000_000, 1_000_000),
            "cpu_baseline": cb, "cpu_ref_1t": one,
            "e2e": {"value": cb["value"], "unit": "s/500 rounds", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": time.perf_counter() - t0}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--forms", default="quantized,f32c,f64")
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--predict-trees", type=int, default=None,
                    help="c4: train the model to this many trees before the batched prediction (the config's 300)")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the AUC seeds, precision report, the 20k-row workload and the other workloads")
    ap.add_argument("--rounds", type=int, default=ROUNDS, help="rounds trained per form (AUC after these)")
    ap.add_argument("--autotune", action="store_true",
                    help="search the per-step launch shape after warm-up and record it for the workload")
    ap.add_argument("--param", action="append", default=[], help="extra training parameter k=v (launch-shape sweeps)")
    ap.add_argument("--workload", default="c2", choices=["c2", "c1", "c3", "c4"],
                    help="c2: the headline binary 10M workload; c1 / c3 / c4: the regression, multiclass and "
                         "lambdarank configurations (a separate JSON line)")
    args = ap.parse_args()
    if args.autotune and int(os.environ.get("WORLD_SIZE", "1")) > 1:
        ap.error("--autotune records one device's choice: run it with one process")
    if args.workload != "c2":
        print(json.dumps(run_workload(args, predict_trees=args.predict_trees)), flush=True)
        return
    args.warmup = max(3, args.warmup)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        run_reference_arm(args, world)
        return

    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    import lgbm_b200 as lgb
    from lgbm_b200 import synthetic

    data = synthetic.make(2, scale=args.scale)
    for kv in args.param:
        k, v = kv.split("=", 1)
        try:
            data["params"][k] = json.loads(v)
        except ValueError:
            data["params"][k] = v
    forms = [f for f in args.forms.split(",") if f]
    ds = lgb.Dataset(data["X"], data["y"], params=data["params"]).construct()
    dv = lgb.Dataset(data["X_valid"], data["y_valid"], params=data["params"], reference=ds).construct()
    res = {}
    for form in forms:
        res[form] = run_form(lgb, data, ds, dv, form, args, local_rank)
    head = "quantized" if "quantized" in res else forms[0]
    r = res[head]
    ms = _max_over_ranks(r["ms_per_step"])
    value = ms * ROUNDS / 1000.0 / world
    e2e = None if args.no_e2e else run_e2e(lgb, data, ds, head, args, local_rank)
    cpu = None if (args.no_cpu or rank != 0 or world > 1) else run_cpu_baseline(lgb, head, 0.1 * args.scale, 3)
    peak, peak_kind = _peaks()
    achieved = r["hist_gbs"]
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": "s/500 rounds", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "int8" if head == "quantized" else ("f32" if head == "f32c" else "f64"),
        "data": "synthetic (seeded generator with the workload's shapes and distributions)",
        "config": config_dict(head, world, len(data["y"]), len(data["y_valid"])),
        "launch_shape": r["launch_shape"], "launch_shape_source": r["launch_shape_source"],
        "forms": {k: {"s_per_500_rounds": v["s_per_500"], "ms_per_step": v["ms_per_step"], "auc": v["auc"],
                      "auc_device": v["auc_device"], "auc_device_ms": v["auc_device_ms"],
                      "auc_numpy_ms": v["auc_numpy_ms"],
                      "hist_gbs": v["hist_gbs"], "hist_ms_per_step": v["hist_ms_per_step"],
                      "scan_ms_per_step": v["scan_ms_per_step"], "partition_ms_per_step": v["partition_ms_per_step"],
                      "hist_rows_per_tree": v["hist_rows_per_tree"], "part_gbs": v["part_gbs"],
                      "part_rows_per_tree": v["part_rows_per_tree"], "launch_shape": v["launch_shape"],
                      "launch_shape_source": v["launch_shape_source"], "hist_by_rows": v["hist_by_rows"]}
                  for k, v in res.items()},
        "roofline": {"bound": "hbm", "kernel": f"k_hist ({head})", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": ((HIST_DRAM_BYTES_PER_ROW_ROOT * len(data["y"]) + HIST_DRAM_BYTES_PER_ROW_SCATTERED *
                                  (r["hist_rows_per_tree"] - len(data["y"]))) /
                                 (int(data["params"]["num_leaves"]) - 1) if head == "quantized" else None),
                     "traffic_note": ("ncu DRAM bytes per row of a 5M-row run (root launch: rows in order; next "
                                      "launch: scattered rows) x the rows of an average launch"),
                     "bytes_per_launch": r["hist_bytes_per_launch"], "ms_per_launch": r["hist_ms_per_launch"],
                     # the histogram's achieved fraction of the HBM roofline by leaf size
                     "by_rows": [dict(b, frac=(b["gbs"] / peak if b["gbs"] else None)) for b in r["hist_by_rows"]]},
        "cpu_baseline": cpu, "e2e": e2e,
        # per iteration: the tree's launches (init, 3 per split, leaf renewal), then the
        # gradients, the quantization (max-abs, packing), the leaf shrinkage, the training
        # rows' score update and the held-out rows' scoring
        "gpu_launches": args.steps * (r["kernel_launches_per_tree"] + 1 + (2 if head == "quantized" else 0) + 3),
        # device-time shares of the three split-step kernels (events around every launch)
        "kernel_share": {k: r[f"{k}_ms_per_step"] / (r["hist_ms_per_step"] + r["scan_ms_per_step"] +
                                                     r["partition_ms_per_step"])
                         for k in ("hist", "scan", "partition")},
        "clocks": r["clocks"],
    }
    # the row partition, the largest share of device time (its launches are
    # latency-bound: most leaves are small)
    line["roofline_partition"] = {
        "bound": "hbm", "kernel": "k_partition", "achieved": r["part_gbs"], "peak": peak, "unit": "GB/s",
        "frac": r["part_gbs"] / peak, "peak_kind": peak_kind,
        "traffic": PART_DRAM_BYTES_PER_ROW * r["part_rows_per_tree"] / (int(data["params"]["num_leaves"]) - 1),
        "traffic_note": "ncu DRAM bytes per row of the 5M-row root split x rows per launch (average)",
        "bytes_per_row": 9, "bytes_per_launch": r["part_bytes_per_launch"],
        "ms_per_launch": r["part_ms_per_launch"]}
    if "f64" in res and head in res:
        line["speedup_vs_f64"] = res["f64"]["ms_per_step"] / res[head]["ms_per_step"]
        line["auc_delta_vs_f64"] = res[head]["auc"] - res["f64"]["auc"]
    if world == 1 and not args.no_extras:
        # beside the headline (not part of its timed region): the AUC gap over
        # more seeds, the precision forms' errors against the FP64 oracle, and
        # the other workloads
        t0 = time.perf_counter()
        if "f64" in res and "quantized" in res:
            line["auc_seeds"] = run_auc_seeds(lgb, args, local_rank, res)
        line["precision"] = run_precision(lgb, local_rank)
        line["config0"] = run_config0(lgb, local_rank)
        wargs = argparse.Namespace(**vars(args))
        wargs.forms, wargs.scale, wargs.steps, wargs.warmup, wargs.autotune = "quantized,f32c,f64", 1.0, 5, 3, False
        line["workloads"] = {}
        for w in ("c1", "c3", "c4"):
            wargs.workload = w  # the key of the workload's recorded launch shape
            line["workloads"][w] = run_workload(wargs, w, predict_trees=300 if w == "c4" else None,
                                                compare_binning=False)
        line["extras_s"] = time.perf_counter() - t0
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
