"""Launch-shape autotuner for the tree learner's per-step kernels.

A split step launches the histogram of the smaller leaf, the threshold scans
and the row partition. Three knobs of those launches change their speed and
nothing else (every shape grows the same trees):

- ``partition_ctas``: CTAs of the row partition per tree slot;
- ``hist_ctas``: histogram CTAs per tree slot and feature tile (a multiple of
  the histogram cluster size);
- ``hist_rows_per_block``: the least rows a histogram CTA takes, which sets
  how many CTAs a small leaf spreads over.

``tune`` searches them one knob at a time around the learner's built-in
shape, then confirms the winner against that shape in one more pass. Each
candidate is timed on the device by regrowing the trees of the learner's
last train call (``lgbm_b200_learner_autotune``: the same
gradients and quantization offsets, so the same trees, and the random
streams of later trees untouched). The learner keeps the fastest shape.
``record`` and ``lookup`` keep the choices per workload in
``launch_shapes.json`` beside this module, keyed by workload and histogram
form, with the device they were measured on.
"""
import json
import os

SHAPES_FILE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "launch_shapes.json")

KNOBS = ("partition_ctas", "hist_ctas", "hist_rows_per_block")


def candidates(base, knob):
    """The values of one knob to try, around the built-in shape ``base``
    (ascending, duplicates removed, ``base[knob]`` included).

    The partition's default is 3 CTAs per SM, which the kernel's registers
    allow resident at once; the candidates go down to one CTA per 16 SMs
    (tree slots batched in one launch share the SMs: K = 10 class trees
    measured fastest at the lowest candidates). The histogram's default is
    every cluster resident at once; the candidates are an eighth, a quarter,
    a half and all of it."""
    if knob not in KNOBS:
        raise ValueError(f"unknown launch-shape knob {knob!r}")
    d = int(base[knob])
    if knob == "partition_ctas":
        vals = {max(1, d * f // 48) for f in (1, 2, 4, 8, 16, 32, 48)}
    elif knob == "hist_ctas":
        vals = {max(1, d // 8), max(1, d // 4), max(1, d // 2), d}
    else:
        vals = {128, 256, 512, 1024, 2048, d}
    return sorted(vals)


def tune(learner, reps=3):
    """Coordinate search over KNOBS, starting from the learner's current
    shape, then a final pass timing that shape and the winner side by side
    (the passes are timed separately, so the winner is confirmed against the
    start in one measurement). The learner must have trained once (its last
    trees are the ones regrown). Returns (best shape, its ms per tree, the
    start shape's ms per tree in the same pass, trials), each trial a shape
    dict with its median ``ms_per_tree``; the learner keeps the best shape."""
    start = learner.launch_shape
    best = dict(start)
    trials = []
    for knob in KNOBS:
        shapes = [dict(best, **{knob: v}) for v in candidates(start, knob)]
        i, ms = learner.time_shapes(shapes, reps)
        trials += [dict(s, ms_per_tree=m) for s, m in zip(shapes, ms)]
        best = dict(shapes[i])  # hist_ctas as asked: the learner rounds it to whole clusters the same way each time
    final = [dict(start), best]
    i, ms = learner.time_shapes(final, reps)
    trials += [dict(s, ms_per_tree=m, final=True) for s, m in zip(final, ms)]
    return dict(final[i]), ms[i], ms[0], trials


def load(path=SHAPES_FILE):
    if not os.path.exists(path):
        return {}
    with open(path) as f:
        return json.load(f)


def record(key, best, best_ms, default_shape, default_ms, trials, device_name, sms, path=SHAPES_FILE):
    """Store the tuned shape of workload ``key`` (rewrites that entry only)."""
    data = load(path)
    data[key] = {"shape": {k: int(best[k]) for k in KNOBS}, "ms_per_tree": best_ms,
                 "default_shape": {k: int(default_shape[k]) for k in KNOBS}, "default_ms_per_tree": default_ms,
                 "device": device_name, "sms": int(sms), "trials": trials}
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
        f.write("\n")
    os.replace(tmp, path)


def lookup(key, sms, path=SHAPES_FILE):
    """The recorded shape of workload ``key``, or None when there is none or
    it was measured on a device with another SM count."""
    e = load(path).get(key)
    if e is None or int(e.get("sms", -1)) != int(sms):
        return None
    return dict(e["shape"])
