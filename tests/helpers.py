"""Shared test helpers: golden cases, materialised trajectories, error metrics."""
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def cases():
    with open(os.path.join(GOLDEN, "cases.json")) as f:
        return json.load(f)


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def materialise(case, directory):
    import make_golden
    return make_golden.materialise(case, directory)


def rel(a, b):
    """Max abs difference relative to the max magnitude of the reference b."""
    a = np.asarray(a)
    b = np.asarray(b)
    scale = np.abs(b).max()
    return float(np.abs(a - b).max() / (scale if scale > 0 else 1.0))


def rel2d(R, ref):
    """2D response error relative to the largest element over all six files."""
    return float(np.abs(np.asarray(R) - ref).max() / np.abs(ref).max())


def R12_to_files(R):
    """12 raw arrays -> [6 files][Re, Im][t3][t1]."""
    return np.asarray(R).reshape(6, 2, R.shape[-2], R.shape[-1])


def uses_eigen(case):
    kw = case["keywords"]
    t2 = int(str(kw.get("RunTimes", "0 0 0")).split()[1])
    return kw.get("Propagation") in ("Sparse", "Diagonal") or (kw["Technique"] != "Absorption" and t2 > 0)
