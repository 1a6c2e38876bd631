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
# DRAM bytes per histogrammed row of the quantized histogram kernel, from the
# ncu capture of a 5M-row root launch (summarised under profiles/);
# traffic grows with the rows of a launch, so a launch's traffic is this times its rows
HIST_DRAM_BYTES_PER_ROW = 40.8
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
    fused = False
    for _ in range(args.steps):
        bst.update()
        t, r, nl = L.last_timing()
        _, pr, fused = L.last_rows()
        hist_ms += t[0]
        scan_ms += t[1]
        part_ms += t[2]
        rows += r
        prows += pr
        launches = nl
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
    hist_launches = args.steps * (1 if fused else steps_per_tree)
    hist_bytes = rows * hist_bytes_per_row(nf, form)
    # the partition moves each row of the split leaf: index in, its byte of the
    # split feature (column copy), index out; the fused form also adds the row to
    # its child's histogram: index in, bin row, packed gradient, index out
    part_bytes = prows * ((4 + nf + 4 + 4) if fused else (4 + 1 + 4))
    return {
        "ms_per_step": ms, "wall_ms_per_step": 1000 * wall / args.steps, "s_per_500": ms * ROUNDS / 1000.0,
        "auc": auc, "auc_device": auc_device, "auc_device_ms": auc_device_ms, "auc_numpy_ms": auc_numpy_ms,
        "hist_ms_per_launch": hist_ms / hist_launches, "hist_gbs": hist_bytes / (hist_ms / 1000) / 1e9,
        "hist_bytes_per_launch": hist_bytes / hist_launches, "hist_rows_per_tree": rows / args.steps,
        "scan_ms_per_step": scan_ms / args.steps, "partition_ms_per_step": part_ms / args.steps,
        "fused": fused, "part_rows_per_tree": prows / args.steps,
        "part_gbs": part_bytes / (part_ms / 1000) / 1e9 if part_ms > 0 else None,
        "part_bytes_per_launch": part_bytes / (args.steps * steps_per_tree),
        "part_ms_per_launch": part_ms / (args.steps * steps_per_tree),
        "hist_ms_per_step": hist_ms / args.steps, "kernel_launches_per_tree": launches, "clocks": clk,
        "num_trees": bst.num_trees(), "nf": nf, "launch_shape": shape, "launch_shape_source": shape_src,
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


def run_cpu_baseline(lgb, form, sample_scale, iters, warmup=3):
    """The oracle (the reference's CPU learner restated) on the host cores, on
    a bounded sample of the workload; seconds per 500 rounds scaled to the
    full row count. The iterations after `warmup` ones are timed: a run of
    warmup + iters rounds minus a run of warmup rounds (both seeded alike)."""
    from lgbm_b200 import synthetic
    from oracle import oracle as orc

    d = synthetic.make(2, scale=sample_scale)
    threads = os.cpu_count() or 8
    params = dict(d["params"], hist_precision=form, num_threads=threads)
    if form == "quantized":
        params["quant_train_renew_leaf"] = True
    p = lgb.resolve_params(params)
    ds = lgb.Dataset(d["X"], d["y"], params=params)
    b = ds.binned()
    t0 = time.perf_counter()
    orc.train(p, b, d["y"], warmup)
    t1 = time.perf_counter()
    orc.train(p, b, d["y"], warmup + iters)
    t2 = time.perf_counter()
    per_iter = ((t2 - t1) - (t1 - t0)) / iters
    per_iter = max(per_iter, (t2 - t1) / (warmup + iters))
    rows = len(d["y"])
    scale = 10_000_000 / rows
    return {"value": per_iter * scale * ROUNDS, "unit": "s/500 rounds", "cores": threads, "kind": "port",
            "sample": f"{rows} rows of the same generator, {iters} timed iterations after {warmup} warm-up ones "
                      f"({form} form, {threads} threads), per-iteration time scaled by {scale:.0f}x rows and "
                      f"x{ROUNDS} rounds", "warmup": warmup}


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


def run_workload(args):
    """The other benchmark configurations: device time per boosting iteration
    of each form on the seeded synthetic data, a quality figure after the
    timed rounds, and (lambdarank) the batched prediction of the trained
    model over every row. One JSON line, not the headline metric."""
    import lgbm_b200 as lgb
    from lgbm_b200 import synthetic

    cfg = {"c1": 1, "c3": 3, "c4": 4}[args.workload]
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
    t0 = time.perf_counter()
    ds = lgb.Dataset(d["X"], d["y"], group=d.get("group"), params=params,
                     categorical_feature=d.get("categorical")).construct(params)
    build_s = time.perf_counter() - t0
    # the same dataset with its rows binned on the device (identical bytes)
    t0 = time.perf_counter()
    ds_dev = lgb.Dataset(d["X"], d["y"], group=d.get("group"), params=dict(params, device_binning=True),
                         categorical_feature=d.get("categorical")).construct(dict(params, device_binning=True))
    build_dev_s = time.perf_counter() - t0
    same = bool(np.array_equal(ds.binned()["bins"], ds_dev.binned()["bins"]))
    del ds_dev
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
            # batched raw prediction of the trained model over every row
            bst.predict(d["X"][:1000], raw_score=True)
            t0 = time.perf_counter()
            bst.predict(d["X"], raw_score=True)
            pred_s = time.perf_counter() - t0
            r["predict"] = {"rows": int(len(y)), "trees": bst.num_trees(), "s": pred_s,
                            "rows_per_s": len(y) / pred_s, "tree_rows_per_s": len(y) * bst.num_trees() / pred_s,
                            "note": "host f32 rows in, f64 scores out, copies included"}
        out["forms"][form] = r
        del bst
    print(json.dumps(out), flush=True)


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
        run_workload(args)
        return
    args.warmup = max(3, args.warmup)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        import lgbm_b200 as lgb

        sample = 0.1 * args.scale
        iters = max(1, min(args.steps, 3))
        warm = min(args.warmup, 5)  # at least 3 (above); bounded so the CPU run stays within minutes
        t0 = time.perf_counter()
        cb = run_cpu_baseline(lgb, "quantized", sample, iters, warm)
        line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "s/500 rounds",
                "n_gpus": args.gpus, "steps": iters, "warmup": warm, "ms_per_step": cb["value"] / ROUNDS * 1000,
                "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "int8",
                "data": "synthetic", "config": {"workload": WORKLOAD, "form": "quantized",
                                                "sample_rows": int(10_000_000 * sample)},
                "cpu_baseline": cb, "e2e": {"value": cb["value"], "unit": "s/500 rounds", "h2d_bytes_per_step": 0,
                                             "d2h_bytes_per_step": 0},
                "wall_s": time.perf_counter() - t0}
        print(json.dumps(line), flush=True)
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
    cpu = None if (args.no_cpu or rank != 0) else run_cpu_baseline(lgb, head, 0.1 * args.scale, 3)
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
        "config": {"workload": WORKLOAD, "form": head, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (bin matrix 320 MB, gradients 80 MB)", "rows": len(data["y"]),
                   "held_out_rows": len(data["y_valid"]), "launch_shape": r["launch_shape"],
                   "launch_shape_source": r["launch_shape_source"]},
        "forms": {k: {"s_per_500_rounds": v["s_per_500"], "ms_per_step": v["ms_per_step"], "auc": v["auc"],
                      "auc_device": v["auc_device"], "auc_device_ms": v["auc_device_ms"],
                      "auc_numpy_ms": v["auc_numpy_ms"],
                      "hist_gbs": v["hist_gbs"], "hist_ms_per_step": v["hist_ms_per_step"],
                      "scan_ms_per_step": v["scan_ms_per_step"], "partition_ms_per_step": v["partition_ms_per_step"],
                      "hist_rows_per_tree": v["hist_rows_per_tree"], "fused": v["fused"], "part_gbs": v["part_gbs"],
                      "part_rows_per_tree": v["part_rows_per_tree"], "launch_shape": v["launch_shape"],
                      "launch_shape_source": v["launch_shape_source"]} for k, v in res.items()},
        "roofline": ({"bound": "hbm", "kernel": "k_partition_fused (row partition + both children's histograms)",
                      "achieved": r["part_gbs"], "peak": peak, "unit": "GB/s", "frac": r["part_gbs"] / peak,
                      "peak_kind": peak_kind, "traffic": None,
                      "bytes_per_launch": r["part_bytes_per_launch"], "ms_per_launch": r["part_ms_per_launch"]}
                     if r["fused"] else
                     {"bound": "hbm", "kernel": f"k_hist ({head})", "achieved": achieved, "peak": peak,
                      "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                      "traffic": (HIST_DRAM_BYTES_PER_ROW * r["hist_rows_per_tree"] /
                                  (int(data["params"]["num_leaves"]) - 1) if head == "quantized" else None),
                      "traffic_note": "ncu DRAM bytes per row of a 5M-row launch x rows per launch (average)",
                      "bytes_per_launch": r["hist_bytes_per_launch"], "ms_per_launch": r["hist_ms_per_launch"]}),
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
    if not r["fused"]:
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
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
