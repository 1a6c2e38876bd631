"""The model text format on the host side: Gbdt::save_model_to_string
(crates/lgbm-core/src/io.rs:13-85), Tree::to_model_string (tree.rs:718-773)
and the %g / %.17g number formatting of fmt.rs.

The trees come back from the device as the reference's Tree arrays, so the
text is written from them exactly as the reference writes it. The text ends
after the feature importances: the "parameters:" block that follows in the
reference is the Config's own text (config.rs:1169-1187), not part of the
tree-learning path.
"""
import math

import numpy as np

K_EPSILON = float(np.float32(1e-15))  # consts.rs


def fmt_g(v, prec):
    """fmt.rs fmt_g: C printf("%.{prec}g", v)."""
    v = float(v)
    if math.isnan(v):
        return "-nan" if math.copysign(1.0, v) < 0 else "nan"
    return "%.*g" % (prec, v)


def _join(a, f):
    return " ".join(f(x) for x in a)


def tree_to_string(t, shrinkage):
    """Tree::to_model_string (tree.rs:718-773) of a tree dict (non-linear)."""
    n = int(t["num_leaves"])
    ni = n - 1
    g6 = lambda x: fmt_g(x, 6)  # noqa: E731
    g17 = lambda x: fmt_g(x, 17)  # noqa: E731
    i2s = lambda x: str(int(x))  # noqa: E731
    lines = [
        "num_leaves=%d" % n,
        "num_cat=%d" % int(t["num_cat"]),
        "split_feature=" + _join(t["split_feature"][:ni], i2s),
        "split_gain=" + _join(np.asarray(t["split_gain"][:ni], np.float32).astype(np.float64), g6),
        "threshold=" + _join(t["threshold"][:ni], g17),
        "decision_type=" + _join(t["decision_type"][:ni], i2s),
        "left_child=" + _join(t["left_child"][:ni], i2s),
        "right_child=" + _join(t["right_child"][:ni], i2s),
        "leaf_value=" + _join(t["leaf_value"][:n], g17),
        "leaf_weight=" + _join(t["leaf_weight"][:n], g17),
        "leaf_count=" + _join(t["leaf_count"][:n], i2s),
        "internal_value=" + _join(t["internal_value"][:ni], g6),
        "internal_weight=" + _join(t["internal_weight"][:ni], g6),
        "internal_count=" + _join(t["internal_count"][:ni], i2s),
    ]
    if int(t["num_cat"]) > 0:
        lines.append("cat_boundaries=" + _join(t["cat_boundaries"][: int(t["num_cat"]) + 1], i2s))
        lines.append("cat_threshold=" + _join(t["cat_threshold"], i2s))
    lines.append("is_linear=0")
    lines.append("shrinkage=" + g6(shrinkage))
    return "\n".join(lines) + "\n\n"


def objective_string(p):
    """The objectives' to_model_string (binary.rs:168-170,
    regression.rs:346-348, multiclass.rs:169-171, rank.rs:338-340)."""
    obj = p["objective"]
    if obj == "binary":
        return "binary sigmoid:" + fmt_g(p["sigmoid"], 6)
    if obj in ("multiclass", "softmax"):
        return "multiclass num_class:%d" % int(p["num_class"])
    if obj == "lambdarank":
        return "lambdarank"
    return "regression"


def model_to_string(p, trees, shrinkages, num_tree_per_iteration, num_total_features, feature_infos,
                    monotone_constraints=None):
    """Gbdt::save_model_to_string (io.rs:13-85) up to the feature
    importances (split counts, boosting.rs:1337-1360)."""
    num_class = int(p["num_class"]) if p["objective"] in ("multiclass", "softmax") else 1
    out = ["tree", "version=v4", "num_class=%d" % num_class,
           "num_tree_per_iteration=%d" % num_tree_per_iteration, "label_index=0",
           "max_feature_idx=%d" % (num_total_features - 1), "objective=" + objective_string(p),
           "feature_names=" + " ".join("Column_%d" % c for c in range(num_total_features))]
    if monotone_constraints is not None and len(monotone_constraints):
        out.append("monotone_constraints=" + " ".join(str(int(m)) for m in monotone_constraints))
    out.append("feature_infos=" + " ".join(feature_infos))
    texts = ["Tree=%d\n%s\n" % (i, tree_to_string(t, s)) for i, (t, s) in enumerate(zip(trees, shrinkages))]
    out.append("tree_sizes=" + " ".join(str(len(x.encode())) for x in texts))
    s = "\n".join(out) + "\n\n" + "".join(texts) + "end of trees\n"
    imp = np.zeros(num_total_features, np.int64)
    for t in trees:
        ni = int(t["num_leaves"]) - 1
        for k in range(ni):
            if float(t["split_gain"][k]) > 0.0:
                imp[int(t["split_feature"][k])] += 1
    order = sorted((c for c in range(num_total_features) if imp[c] > 0), key=lambda c: -imp[c])  # stable
    s += "\nfeature_importances:\n" + "".join("Column_%d=%d\n" % (c, imp[c]) for c in order)
    return s
