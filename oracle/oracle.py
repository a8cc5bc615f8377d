"""ORACLE — test infrastructure, not product code.

Python access to the two checkers of the NISE propagation path:
  * the reference programs compiled from their own sources (oracle/_ref/NISE_acc,
    NISE_fast, 2DFFT; recipe in oracle/Makefile), run on keyword files, and
  * the C restatement nise_oracle.c in FP32 (reference arithmetic) and FP64.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

TECHNIQUES = {"Absorption": 0, "2DIR": 1, "GBIR": 2, "SEIR": 3, "EAIR": 4, "noEAIR": 5,
              "2DUVvis": 6, "GBUVvis": 7, "SEUVvis": 8, "EAUVvis": 9, "noEAUVvis": 10,
              "LD": 11, "Raman": 12, "SFG": 13, "DOS": 14, "CD": 15,
              "Luminescence": 16, "PL": 16, "Fluorescence": 16}
# output files of the linear techniques per channel (calc_LD.c, raman.c, sfg.c, calc_DOS.c, calc_CD.c)
LINEAR_FILES = {"LD": [("TD_LD.dat", "LD.dat")],
                "Raman": [("TD_Raman_VV.dat", "Raman_VV.dat"), ("TD_Raman_VH.dat", "Raman_VH.dat")],
                "SFG": [("TD_SFG_PPP.dat", "SFG_PPP.dat"), ("TD_SFG_SSP.dat", "SFG_SSP.dat")],
                "DOS": [("TD_DOS.dat", "DOS.dat")], "CD": [("TD_CD.dat", "CD.dat")],
                # luminescence.c:223-234: the time-domain file of the total only
                "Luminescence": [("TD_Lum.dat", "Luminescence.dat"), (None, "Luminescence_x.dat"),
                                 (None, "Luminescence_y.dat"), (None, "Luminescence_z.dat")]}
LINEAR_FILES["PL"] = LINEAR_FILES["Fluorescence"] = LINEAR_FILES["Luminescence"]
ICM2IFS = np.float32(2.99792458e-5)
TWOPI = np.float32(2 * 3.14159265359)


class OracleParams(ctypes.Structure):
    _fields_ = [
        ("singles", ctypes.c_int), ("doubles", ctypes.c_int),
        ("length", ctypes.c_int), ("sample", ctypes.c_int), ("begin", ctypes.c_int), ("end", ctypes.c_int),
        ("tmax1", ctypes.c_int), ("tmax2", ctypes.c_int), ("tmax3", ctypes.c_int),
        ("deltat", ctypes.c_float), ("ts", ctypes.c_int),
        ("lifetime", ctypes.c_float), ("homogen", ctypes.c_float), ("inhomogen", ctypes.c_float),
        ("window", ctypes.c_int), ("fft", ctypes.c_int),
        ("thres", ctypes.c_float), ("couplingcut", ctypes.c_float), ("anharmonicity", ctypes.c_float),
        ("min1", ctypes.c_float), ("max1", ctypes.c_float), ("min2", ctypes.c_float),
        ("max2", ctypes.c_float), ("min3", ctypes.c_float), ("max3", ctypes.c_float),
        ("ham_coupling", ctypes.c_int), ("propagation", ctypes.c_int), ("technique", ctypes.c_int),
        ("energy", ctypes.c_char * 256), ("dipole", ctypes.c_char * 256), ("coupling", ctypes.c_char * 256),
        ("anharm", ctypes.c_char * 256), ("overtone", ctypes.c_char * 256), ("shift", ctypes.c_char * 256),
        ("ham_onfly", ctypes.c_int), ("position", ctypes.c_char * 256), ("pbc", ctypes.c_char * 256),
        ("alpha", ctypes.c_char * 256), ("temperature", ctypes.c_float), ("imag_steps", ctypes.c_int),
    ]


def params(keywords, files):
    """Oracle parameters from a keyword dict (readinput.c:24-289 semantics for
    the keywords on the path) and the trajectory file dict."""
    kw = {k: str(v) for k, v in keywords.items()}
    p = OracleParams()
    p.ts = 5
    p.tmax1, p.tmax2, p.tmax3 = 256, 0, 256
    p.singles = int(kw.get("Singles", 0))
    p.doubles = int(kw.get("Doubles", 0))
    p.length = int(kw["Length"])
    p.sample = int(kw["Samplerate"])
    p.begin = int(kw.get("BeginPoint", 0))
    p.end = int(kw.get("EndPoint", 0))
    if "RunTimes" in kw:
        p.tmax1, p.tmax2, p.tmax3 = (int(x) for x in kw["RunTimes"].split()[:3])
    p.deltat = float(kw["Timestep"])
    p.ts = int(kw.get("Trotter", 5))
    p.lifetime = float(kw.get("Lifetime", 0))
    p.homogen = float(kw.get("Homogeneous", 0))
    p.inhomogen = float(kw.get("Inhomogeneous", 0))
    p.window = 1 if kw.get("Window", "") == "Hann" else 0
    p.fft = int(kw.get("FFT", 0))
    p.couplingcut = float(kw.get("Couplingcut", 0))
    p.anharmonicity = float(kw.get("Anharmonicity", 0))
    mins = [float(x) for x in kw.get("MinFrequencies", "0 0 0").split()[:3]]
    maxs = [float(x) for x in kw.get("MaxFrequencies", "0 0 0").split()[:3]]
    p.min1, p.min2, p.min3 = mins
    p.max1, p.max2, p.max3 = maxs
    p.ham_coupling = 1 if kw.get("HamiltonianType", "Full") == "Coupling" else 0
    p.ham_onfly = {"TransitionDipole": 1, "ExtendedDipole": 2}.get(kw.get("HamiltonianType", "Full"), 0)
    prop = kw.get("Propagation", "")
    p.propagation = {"Coupling": 1, "Diagonal": 2, "RK4": 3}.get(prop, 0)
    p.technique = TECHNIQUES[kw.get("Technique", "Absorption")]
    p.temperature = float(kw.get("Temperature", 300))  # readinput.c:32
    p.imag_steps = int(kw.get("ImaginaryTimesteps", 0))  # readinput.c:28
    if 1 <= p.technique <= 10:
        p.tmax3 = p.tmax1  # readinput.c:212
    thres = np.float32(float(kw.get("Threshold", 0)))
    if p.propagation == 0:  # readinput.c:264-267, in float arithmetic
        s = np.float32(np.float32(np.float32(p.deltat) * ICM2IFS) * TWOPI) / np.float32(p.ts)
        thres = np.float32(thres * np.float32(s * s))
    p.thres = float(thres)
    for key in ("energy", "dipole", "coupling", "anharm", "overtone", "shift", "position", "pbc", "alpha"):
        setattr(p, key, (files.get(key) or "").encode())
    return p


_libs = {}


def lib(prec="f64"):
    if prec not in _libs:
        path = os.path.join(REF_DIR, "liboracle_%s.so" % prec)
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        P = ctypes.POINTER(OracleParams)
        dp = ctypes.POINTER(ctypes.c_double)
        L.oracle_absorption.argtypes = [P, dp, dp, ctypes.POINTER(ctypes.c_int)]
        L.oracle_2dir.argtypes = [P, dp, ctypes.POINTER(ctypes.c_int)]
        L.oracle_linear.argtypes = [P, dp, dp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        L.oracle_1dfft.argtypes = [P, dp, dp, ctypes.c_int, dp, dp, dp, ctypes.c_int]
        L.oracle_print2d_normalize.argtypes = [P, dp, dp, ctypes.c_int]
        fp = ctypes.POINTER(ctypes.c_float)
        L.oracle_propagate_vector.argtypes = [P, fp, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        L.oracle_propagate_doubles.argtypes = [P, fp, ctypes.c_void_p, ctypes.c_void_p, fp]
        L.oracle_propagate_t2.argtypes = [P, fp, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        L.oracle_dipole_double.argtypes = [P, fp, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_void_p, fp]
        L.oracle_dipole_double_last.argtypes = L.oracle_dipole_double.argtypes
        L.oracle_eigh.argtypes = [ctypes.c_int, dp, dp, dp]
        _libs[prec] = L
    return _libs[prec]


# Where the reference's sources are read from when the reference programs are
# compiled (NISE_REFERENCE_SRC overrides the default location).
REF_SRC = os.environ.get("NISE_REFERENCE_SRC", "/root/reference/src")


def reference_present():
    return os.path.isdir(REF_SRC)


def build(ref=True):
    """Compile the restatement and, when the reference sources are present, the reference."""
    import sysconfig
    targets = ["oracle"]
    if ref and reference_present():
        targets.append("ref")
    subprocess.run(["make", "-s", "REF=" + REF_SRC, "PYLIB=" + sysconfig.get_paths()["purelib"]] + targets,
                   cwd=HERE, check=True)


def _ptr(a, t=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(t))


def absorption(p, prec="f64"):
    """Raw response sums and the normaliser (absorption.c:92-192)."""
    re = np.zeros(p.tmax1)
    im = np.zeros(p.tmax1)
    n = ctypes.c_int(0)
    rc = lib(prec).oracle_absorption(ctypes.byref(p), _ptr(re), _ptr(im), ctypes.byref(n))
    if rc != 0:
        raise RuntimeError("oracle_absorption failed (%d)" % rc)
    return re, im, n.value


def _f32(x):
    return float(np.float32(x))


def exact_step_factor(deltat):
    """f = deltat * icm2ifs * twoPi (propagate.c:67) from the float constants of types.h."""
    return _f32(deltat) * _f32(2.99792458e-5) * _f32(2 * 3.14159265359)


def read_frames(keywords, files, frames):
    """Shifted, cut Hamiltonians (FP64 copies of the float32 values the
    reference's readers produce, read_trajectory.c:73-314) of the given frames,
    and the dipole reader for HamiltonianType Coupling (static dipoles of frame
    0, read_trajectory.c:61-67) or Full (per-frame, :357-377)."""
    n = int(keywords["Singles"])
    mins = [float(v) for v in str(keywords["MinFrequencies"]).split()]
    maxs = [float(v) for v in str(keywords["MaxFrequencies"]).split()]
    shift = np.float32((np.float32(maxs[0]) + np.float32(mins[0])) / np.float32(2))
    cut = np.float32(keywords.get("Couplingcut", 0))
    coupling = keywords.get("HamiltonianType", "Full") == "Coupling"
    iu = np.triu_indices(n)
    e = np.fromfile(files["energy"], dtype=np.float32)
    d = np.fromfile(files["dipole"], dtype=np.float32)
    if coupling:
        hc = np.fromfile(files["coupling"], dtype=np.float32)[1:1 + n * (n + 1) // 2]
    H = {}
    for t in frames:
        if coupling:
            packed = hc.copy()
            rec = e[t * (1 + n) + 1:(t + 1) * (1 + n)]
            diag = rec
        else:
            w = 1 + n * (n + 1) // 2
            packed = e[t * w + 1:(t + 1) * w].copy()
            diag = packed[[a * n + a - a * (a + 1) // 2 for a in range(n)]]
        M = np.zeros((n, n), np.float32)
        M[iu] = packed
        off = np.abs(M) < cut
        M[off] = 0
        M = np.triu(M, 1)
        M = M + M.T
        M[np.arange(n), np.arange(n)] = (diag.astype(np.float32) - shift).astype(np.float32)
        H[t] = M.astype(np.float64)

    def mu(t, x):
        tt = 0 if coupling else t
        return d[tt * (1 + 3 * n) + 1 + x * n:tt * (1 + 3 * n) + 1 + (x + 1) * n].astype(np.float64)
    return H, mu


def exact_propagators(H, f, thres=0.0):
    """U = V exp(-i e f) V^T of every frame (propagate_vec_DIA,
    propagate.c:60-125, in FP64; the eigendecomposition is numpy's); with
    0 < thres <= 1 only the elements with |U_ab|^2 > thres are kept
    (propagate_vec_DIA_S, propagate.c:185-258; propagate_vector's dispatch,
    propagate.c:24-28)."""
    U = {}
    for t, M in H.items():
        e, V = np.linalg.eigh(M)
        Ut = (V * np.exp(-1j * e * f)) @ V.T
        if thres != 0 and not thres > 1:
            Ut[np.abs(Ut) ** 2 <= thres] = 0
        U[t] = Ut
    return U


def absorption_exact(keywords, files):
    """FP64 linear absorption with the exact propagator (Sparse, Threshold 0):
    the sample loop of absorption.c:92-192 (response before propagation,
    :119-145) with one U per frame shared by every vector that crosses it.
    Returns (re_S, im_S, samples) like absorption()."""
    n = int(keywords["Singles"])
    length = int(keywords["Length"])
    sample = int(keywords["Samplerate"])
    tmax = int(str(keywords["RunTimes"]).split()[0])
    begin = int(keywords.get("BeginPoint", 0))
    nsamp = (length - tmax - 1) // sample + 1  # NISE_subs.c:197-221
    end = int(keywords.get("EndPoint", 0)) or nsamp
    assert 0 < end <= nsamp and not keywords.get("SingleShift")
    frames = sorted({s * sample + t1 for s in range(begin, end) for t1 in range(tmax)})
    H, mu = read_frames(keywords, files, frames)
    thres = 0.0
    if keywords.get("Propagation", "Sparse") not in ("Coupling", "RK4", "Diagonal"):
        thres = float(params(keywords, files).thres)  # Threshold scaled by (f/ts)^2 as readinput.c:264-267
    U = exact_propagators(H, exact_step_factor(float(keywords["Timestep"])), thres)
    S = np.zeros(tmax, np.complex128)
    for s in range(begin, end):
        ti = s * sample
        for x in range(3):
            c = mu(ti, x).astype(np.complex128)
            for t1 in range(tmax):
                S[t1] += mu(ti + t1, x) @ c
                c = U[ti + t1] @ c
    return S.real.copy(), S.imag.copy(), end


def spectrum(p, re, im, samples, prec="f64"):
    fft = max(p.fft, p.tmax1)
    w = np.zeros(fft)
    sr = np.zeros(fft)
    si = np.zeros(fft)
    rows = lib(prec).oracle_1dfft(ctypes.byref(p), _ptr(np.ascontiguousarray(re, dtype=np.float64)),
                                  _ptr(np.ascontiguousarray(im, dtype=np.float64)), samples, _ptr(w), _ptr(sr),
                                  _ptr(si), fft)
    return w[:rows], sr[:rows], si[:rows]


def linear(p, prec="f64"):
    """LD, Raman, SFG, DOS, CD, Luminescence: raw response sums re, im [channel][tmax1] and the normaliser."""
    re = np.zeros((4, p.tmax1))
    im = np.zeros((4, p.tmax1))
    ch = ctypes.c_int(0)
    n = ctypes.c_int(0)
    rc = lib(prec).oracle_linear(ctypes.byref(p), _ptr(re), _ptr(im), ctypes.byref(ch), ctypes.byref(n))
    if rc != 0:
        raise RuntimeError("oracle_linear failed (%d)" % rc)
    return re[:ch.value], im[:ch.value], n.value


def twodir(p, prec="f64"):
    """Raw 12 x tmax3 x tmax1 response sums and the sample count."""
    R = np.zeros((12, p.tmax3, p.tmax1))
    n = ctypes.c_int(0)
    rc = lib(prec).oracle_2dir(ctypes.byref(p), _ptr(R), ctypes.byref(n))
    if rc != 0:
        raise RuntimeError("oracle_2dir failed (%d)" % rc)
    return R, n.value


def normalize_2d(p, R, count, prec="f64"):
    out = R.copy()
    for k in range(0, 12, 2):
        re = np.ascontiguousarray(out[k])
        im = np.ascontiguousarray(out[k + 1])
        lib(prec).oracle_print2d_normalize(ctypes.byref(p), _ptr(re), _ptr(im), count)
        out[k], out[k + 1] = re, im
    return out


# ------------------------------------------------------------ reference binary
def run_reference(input_path, workdir, binary="NISE_acc", threads=1, timeout=3600):
    exe = os.path.join(REF_DIR, binary)
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    r = subprocess.run([exe, os.path.abspath(input_path)], cwd=workdir, env=env, stdout=subprocess.PIPE,
                       stderr=subprocess.STDOUT, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError("reference failed (%d):\n%s" % (r.returncode, r.stdout[-2000:]))
    return r.stdout


def read_td_absorption(path):
    a = np.loadtxt(path, ndmin=2)
    return a[:, 0], a[:, 1], a[:, 2]


def read_spectrum(path):
    a = np.loadtxt(path, ndmin=2)
    return a[:, 0], a[:, 1], a[:, 2]


def read_2d(path, tmax1, tmax3):
    a = np.loadtxt(path, ndmin=2)
    re = a[:, 3].reshape(tmax1, tmax3).T
    im = a[:, 4].reshape(tmax1, tmax3).T
    return re, im


R2D_FILES = ["RparI.dat", "RparII.dat", "RperI.dat", "RperII.dat", "RcroI.dat", "RcroII.dat"]
