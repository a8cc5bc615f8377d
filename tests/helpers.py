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
    """Whether the case goes through an eigendecomposition (FP64 here, the
    reference's ssyev_ in FP32): Sparse/Diagonal propagation, the 2D t2 step,
    the exact Boltzmann weights of luminescence."""
    kw = case["keywords"]
    t2 = int(str(kw.get("RunTimes", "0 0 0")).split()[1])
    lum = kw["Technique"] in ("Luminescence", "PL", "Fluorescence") and int(kw.get("ImaginaryTimesteps", 0)) == 0
    return kw.get("Propagation") in ("Sparse", "Diagonal") or (kw["Technique"] != "Absorption" and t2 > 0) or lum


def td_channels(technique, linear_files):
    """Channels of a linear technique that have a time-domain file, in the
    order of the golden td arrays (luminescence writes the total's only)."""
    return [k for k, (td, _) in enumerate(linear_files[technique]) if td]


def fft2d_case(name):
    """Inputs and reference outputs of a 2D FFT golden case: ({name: text}, {name: text})."""
    d = np.load(os.path.join(GOLDEN, "fft2d_%s.npz" % name))
    return json.loads(str(d["inputs"])), json.loads(str(d["outputs"]))


def fft2d_case_names():
    with open(os.path.join(GOLDEN, "fft2d_cases.json")) as f:
        return sorted(json.load(f))


def compare_spectrum_text(got, ref, tol):
    """Compare two text files of the 2D FFT step.

    The line structure (blank lines, tokens per line, the '###' header) must be
    identical; "%f" tokens (frequency axes) must be identical text; "%e" tokens
    (spectral values) must agree within tol times the largest |value| in the
    file.  Returns the worst relative value difference.
    """
    a, b = got.splitlines(), ref.splitlines()
    assert len(a) == len(b), "line count %d != %d" % (len(a), len(b))
    worst, vals_a, vals_b = 0.0, [], []
    for la, lb in zip(a, b):
        ta, tb = la.split(), lb.split()
        assert len(ta) == len(tb), (la, lb)
        if lb.startswith("#"):
            assert la == lb
            continue
        for x, y in zip(ta, tb):
            if "e" in y:
                vals_a.append(float(x))
                vals_b.append(float(y))
            else:
                assert x == y, "axis token %s != %s" % (x, y)
    if vals_b:
        va, vb = np.array(vals_a), np.array(vals_b)
        scale = np.abs(vb).max() or 1.0
        worst = float(np.abs(va - vb).max() / scale)
        assert worst <= tol, "values differ by %.3g of the largest (tolerance %.3g)" % (worst, tol)
    return worst
