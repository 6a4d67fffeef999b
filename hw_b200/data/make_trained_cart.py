"""Generates hw_b200/data/trained_cart.npz: the activity labeler's trained
CART as the reference ships it (ActivityLabeler::TrainedCart,
src/basecaller/dataTypes/TrainedCartParams.cpp), read from the reference
checkout.  The HF-metrics tests and the benchmark pass these arrays through
hw_hfmetrics_set_cart, as an integrating basecaller passes its own table.

    python hw_b200/data/make_trained_cart.py <reference project root>
"""
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def parse(path):
    text = open(path).read()
    out = {}
    m = re.search(r"maxAcceptableHalfsandwichRate\s*=\s*([-0-9.eE+]+)f?;", text)
    out["max_acceptable_halfsandwich_rate"] = np.float32(float(m.group(1)))
    m = re.search(r"hswCurve\s*\{\{([^}]*)\}\}", text)
    out["hsw_curve"] = np.array([float(x) for x in m.group(1).split(",")], np.float32)
    for name, key, dt in (("childrenLeft", "children_left", np.int16), ("childrenRight", "children_right", np.int16),
                          ("feature", "feature", np.int8), ("threshold", "threshold", np.float32),
                          ("value", "value", np.int8)):
        m = re.search(r"TrainedCart::" + name + r"\s*\{([^}]*)\}", text)
        vals = [v.strip() for v in m.group(1).replace("\n", " ").split(",") if v.strip()]
        out[key] = np.array([float(v) if dt == np.float32 else int(v) for v in vals], dt)
    n = len(out["children_left"])
    assert all(len(out[k]) == n for k in ("children_right", "feature", "threshold", "value"))
    return out


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_trained_cart.py <reference project root>")
    root = sys.argv[1]
    arrays = parse(os.path.join(root, "src/basecaller/dataTypes/TrainedCartParams.cpp"))
    np.savez(os.path.join(HERE, "trained_cart.npz"), **arrays)
    print({k: v.shape for k, v in arrays.items()})


if __name__ == "__main__":
    main()
