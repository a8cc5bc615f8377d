"""nise_2017_b200 — B200 engine for the NISE wavefunction-propagation path.

Python mirror of the reference's operator interface for this path, over the
C ABI in include/nise_b200.h (libnise_b200.so, built in-tree by
nise_2017_b200/build.py):

  read_input(path)                  readInput      (readinput.c:13-289)
  Context(params).load_files()      open_files / read_coupling / read_shift + frame readers
  Context.absorption()              absorption     (absorption.c:18-202)
  Context.absorption_fft(...)       do_1DFFT       (1DFFT.c:144-228)
  Context.twodir()                  calc_2DIR      (calc_2DIR.c:22-629)
  Context.propagate(H, re, im, s)   propagate_vector, batched (propagate.c:20-39)

Failures raise NiseError carrying the library's status code and message (the
reference prints and exits instead).  There is no CPU fallback: every compute
call runs the CUDA kernels, and loading fails loudly if the library is missing.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnise_b200.so")

PROP = {"Sparse": 0, "Coupling": 1, "Diagonal": 2, "RK4": 3}
HAM = {"Full": 0, "Coupling": 1}
TECH = {"Absorption": 0, "2DIR": 1, "GBIR": 2, "SEIR": 3, "EAIR": 4, "noEAIR": 5,
        "2DUVvis": 6, "GBUVvis": 7, "SEUVvis": 8, "EAUVvis": 9, "noEAUVvis": 10,
        "LD": 11, "Raman": 12, "SFG": 13, "DOS": 14, "CD": 15, "Luminescence": 16, "PL": 16, "Fluorescence": 16}
FP32, FP64 = 0, 1
BATCHED, PLAIN = 0, 1
R2D_NAMES = ["RparI.dat", "RparII.dat", "RperI.dat", "RperII.dat", "RcroI.dat", "RcroII.dat"]

EXPORTED = [
    "nise_params_default", "nise_read_input", "nise_create", "nise_destroy", "nise_last_error",
    "nise_global_error", "nise_load_files", "nise_set_trajectory", "nise_set_singleshift", "nise_absorption",
    "nise_absorption_fft", "nise_2dir", "nise_propagate", "nise_propagate_doubles", "nise_write_td_absorption",
    "nise_write_spectrum", "nise_write_2d", "nise_set_stream", "nise_last_timing", "nise_last_work",
    "nise_probe_fp32_peak", "nise_absorption_noalloc", "nise_2dfft_files", "nise_absorption_model",
    "nise_backward_absorption", "nise_absorption_tune", "nise_batch_create", "nise_batch_run", "nise_batch_result",
    "nise_batch_spectrum", "nise_batch_timing", "nise_batch_error", "nise_batch_destroy", "nise_set_trajectory_onfly",
    "nise_set_operators", "nise_linear", "nise_linear_file", "nise_write_td", "nise_translate",
    "nise_rotation_schedule",
]


class NiseError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (status %d)" % (msg, code))
        self.code = code


class Params(ctypes.Structure):
    """nise_params (include/nise_b200.h), the t_non fields on this path."""
    _fields_ = [
        ("singles", ctypes.c_int), ("doubles", ctypes.c_int), ("length", ctypes.c_int), ("sample", ctypes.c_int),
        ("begin", ctypes.c_int), ("end", ctypes.c_int), ("tmax1", ctypes.c_int), ("tmax2", ctypes.c_int),
        ("tmax3", ctypes.c_int), ("deltat", ctypes.c_float), ("ts", ctypes.c_int), ("lifetime", ctypes.c_float),
        ("homogen", ctypes.c_float), ("inhomogen", ctypes.c_float), ("window", ctypes.c_int), ("fft", ctypes.c_int),
        ("thres", ctypes.c_float), ("couplingcut", ctypes.c_float), ("anharmonicity", ctypes.c_float),
        ("min1", ctypes.c_float), ("max1", ctypes.c_float), ("min2", ctypes.c_float), ("max2", ctypes.c_float),
        ("min3", ctypes.c_float), ("max3", ctypes.c_float), ("hamiltonian", ctypes.c_int),
        ("propagation", ctypes.c_int), ("technique", ctypes.c_int), ("technique_name", ctypes.c_char * 64),
        ("energyFName", ctypes.c_char * 256), ("dipoleFName", ctypes.c_char * 256),
        ("couplingFName", ctypes.c_char * 256), ("anharFName", ctypes.c_char * 256),
        ("overdipFName", ctypes.c_char * 256), ("singleShiftFName", ctypes.c_char * 256),
        ("precision", ctypes.c_int), ("launch_mode", ctypes.c_int), ("device", ctypes.c_int),
        ("kernel_config", ctypes.c_int), ("positionFName", ctypes.c_char * 256), ("pbcFName", ctypes.c_char * 256),
        ("alphaFName", ctypes.c_char * 256), ("temperature", ctypes.c_float), ("imag_steps", ctypes.c_int),
    ]


_lib = None


def lib():
    """Load libnise_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError("libnise_b200.so is missing; run `python -m nise_2017_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER(Params)
        vp = ctypes.c_void_p
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.nise_params_default.argtypes = [P]
        L.nise_read_input.argtypes = [ctypes.c_char_p, P]
        L.nise_create.argtypes = [P, ctypes.POINTER(vp)]
        L.nise_destroy.argtypes = [vp]
        L.nise_destroy.restype = None
        L.nise_last_error.argtypes = [vp]
        L.nise_last_error.restype = ctypes.c_char_p
        L.nise_global_error.restype = ctypes.c_char_p
        L.nise_load_files.argtypes = [vp]
        L.nise_set_trajectory.argtypes = [vp, vp, ctypes.c_size_t, vp, ctypes.c_size_t, vp, ctypes.c_size_t, vp,
                                          ctypes.c_size_t, vp, ctypes.c_size_t]
        L.nise_set_singleshift.argtypes = [vp, ctypes.c_int, ip, ctypes.POINTER(ctypes.c_float),
                                           ctypes.POINTER(ctypes.c_float)]
        L.nise_absorption.argtypes = [vp, dp, dp, ip]
        L.nise_absorption_fft.argtypes = [vp, dp, dp, ctypes.c_int, dp, dp, dp, ctypes.c_int, ip]
        L.nise_2dir.argtypes = [vp, dp, ip]
        L.nise_propagate.argtypes = [vp, ctypes.POINTER(ctypes.c_float), vp, vp, ctypes.c_int, ctypes.c_int]
        L.nise_propagate_doubles.argtypes = [vp, ctypes.POINTER(ctypes.c_float), vp, vp, ctypes.c_int,
                                             ctypes.POINTER(ctypes.c_float)]
        L.nise_write_td_absorption.argtypes = [ctypes.c_char_p, P, dp, dp, ctypes.c_int]
        L.nise_write_spectrum.argtypes = [ctypes.c_char_p, dp, dp, dp, ctypes.c_int]
        L.nise_write_2d.argtypes = [ctypes.c_char_p, P, dp, dp, ctypes.c_int]
        L.nise_set_stream.argtypes = [vp, vp]
        L.nise_last_timing.argtypes = [vp, dp, dp, ctypes.POINTER(ctypes.c_long)]
        L.nise_last_work.argtypes = [vp, dp, dp]
        L.nise_probe_fp32_peak.argtypes = [ctypes.c_int, dp]
        L.nise_absorption_tune.argtypes = [vp]
        L.nise_batch_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)]
        L.nise_batch_run.argtypes = [vp]
        L.nise_batch_result.argtypes = [vp, ctypes.c_int, dp, dp, ip]
        L.nise_batch_spectrum.argtypes = [vp, ctypes.c_int, dp, dp, dp, ctypes.c_int, ip]
        L.nise_batch_timing.argtypes = [vp, dp, ctypes.POINTER(ctypes.c_long)]
        L.nise_batch_error.argtypes = [vp]
        L.nise_batch_error.restype = ctypes.c_char_p
        L.nise_batch_destroy.argtypes = [vp]
        L.nise_batch_destroy.restype = None
        L.nise_set_operators.argtypes = [vp, vp, ctypes.c_size_t, vp, ctypes.c_size_t]
        L.nise_linear.argtypes = [vp, dp, dp, ctypes.c_int, ip, ip]
        L.nise_linear_file.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.nise_linear_file.restype = ctypes.c_char_p
        L.nise_write_td.argtypes = [ctypes.c_char_p, P, dp, dp, ctypes.c_int, ctypes.c_int]
        L.nise_translate.argtypes = [ctypes.c_char_p]
        L.nise_rotation_schedule.argtypes = [ip, ctypes.c_int, ctypes.c_int, ip, ip, ip, ip, ip, ip]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def rotation_schedule(pairs, n):
    """The engine's Trotter rotation order for a lexicographic coupling list
    (host only): (perm, level bounds, chunk bounds, flip) as numpy int arrays;
    flip[q] = 1 applies rotation perm[q] with its two sites swapped."""
    ab = np.ascontiguousarray(np.asarray(pairs, dtype=np.int32).reshape(-1, 2))
    k = len(ab)
    perm = np.zeros(max(k, 1), np.int32)
    lv = np.zeros(k + 1, np.int32)
    chk = np.zeros(k + 1, np.int32)
    flip = np.zeros(max(k, 1), np.int32)
    nlev, nchk = ctypes.c_int(), ctypes.c_int()
    ip = ctypes.POINTER(ctypes.c_int)
    rc = lib().nise_rotation_schedule(ab.ctypes.data_as(ip), k, n, perm.ctypes.data_as(ip), lv.ctypes.data_as(ip),
                                      ctypes.byref(nlev), chk.ctypes.data_as(ip), ctypes.byref(nchk),
                                      flip.ctypes.data_as(ip))
    if rc != 0:
        raise NiseError(rc, lib().nise_global_error().decode())
    return perm[:k], lv[:nlev.value + 1], chk[:nchk.value + 1], flip[:k]


def translate(keyword_file):
    """Run a translate keyword file (trajectory format conversion, host only)."""
    rc = lib().nise_translate(os.fsencode(keyword_file))
    if rc != 0:
        raise NiseError(rc, lib().nise_global_error().decode())


def linear_files(technique):
    """[(TD file, spectrum file)] of each channel of a linear technique."""
    code = TECH[technique] if isinstance(technique, str) else technique
    out = []
    while True:
        sp = lib().nise_linear_file(code, len(out), 0)
        if sp is None:
            return out
        td = lib().nise_linear_file(code, len(out), 1)  # None: the channel has no time-domain file
        out.append((td.decode() if td else None, sp.decode()))


def default_params():
    p = Params()
    lib().nise_params_default(ctypes.byref(p))
    return p


def read_input(path):
    """Parse a NISE keyword file (readinput.c semantics)."""
    p = default_params()
    rc = lib().nise_read_input(os.fsencode(path), ctypes.byref(p))
    if rc != 0:
        raise NiseError(rc, lib().nise_global_error().decode())
    return p


def params_from_keywords(keywords, files=None, **engine):
    """Build params by writing the keywords through the same parser."""
    import tempfile
    lines = []
    for k, v in (files or {}).items():
        key = {"energy": "Hamiltonianfile", "dipole": "Dipolefile", "coupling": "Couplingfile",
               "anharm": "Anharmonicfile", "overtone": "Overtonedipolefile", "shift": "SingleShiftfile",
               "position": "Positionfile", "pbc": "PBCfile", "alpha": "Alphafile"}[k]
        if v:
            lines.append("%s %s" % (key, v))
    lines += ["%s %s" % (k, v) for k, v in keywords.items()]
    with tempfile.NamedTemporaryFile("w", suffix=".inp", delete=False) as f:
        f.write("\n".join(lines) + "\n")
        path = f.name
    try:
        p = read_input(path)
    finally:
        os.unlink(path)
    for k, v in engine.items():
        setattr(p, k, v)
    return p


class Context:
    """One engine context (one device stream); mirrors the reference's t_non-driven calls."""

    def __init__(self, params):
        self.params = params
        h = ctypes.c_void_p()
        rc = lib().nise_create(ctypes.byref(params), ctypes.byref(h))
        if rc != 0:
            raise NiseError(rc, lib().nise_global_error().decode())
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().nise_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc):
        if rc != 0:
            raise NiseError(rc, lib().nise_last_error(self._h).decode())

    def load_files(self):
        self._check(lib().nise_load_files(self._h))
        return self

    def set_trajectory(self, energy, dipole, coupling=None, anharm=None, overtone=None):
        """Record images (bytes-like or numpy arrays) of the trajectory files."""
        keep = []

        def buf(x):
            if x is None:
                return None, 0
            a = np.ascontiguousarray(np.frombuffer(x, dtype=np.uint8) if isinstance(x, (bytes, bytearray)) else x)
            keep.append(a)
            return a.ctypes.data, a.nbytes
        args = []
        for x in (energy, dipole, coupling, anharm, overtone):
            args += list(buf(x))
        self._check(lib().nise_set_trajectory(self._h, *args))
        return self

    def set_singleshift(self, sites, a, b):
        s = np.ascontiguousarray(sites, dtype=np.int32)
        fa = np.ascontiguousarray(a, dtype=np.float32)
        fb = np.ascontiguousarray(b, dtype=np.float32)
        self._check(lib().nise_set_singleshift(self._h, len(s), s.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                               fa.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                               fb.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))

    def absorption(self):
        """Raw response sums (re, im) over samples and polarisations and the normaliser."""
        t = self.params.tmax1
        re = np.zeros(t)
        im = np.zeros(t)
        n = ctypes.c_int(0)
        self._check(lib().nise_absorption(self._h, _dp(re), _dp(im), ctypes.byref(n)))
        return re, im, n.value

    def absorption_fft(self, re, im, samples):
        fft = max(self.params.fft, self.params.tmax1)
        w = np.zeros(fft)
        sr = np.zeros(fft)
        si = np.zeros(fft)
        rows = ctypes.c_int(0)
        re = np.ascontiguousarray(re, dtype=np.float64)
        im = np.ascontiguousarray(im, dtype=np.float64)
        self._check(lib().nise_absorption_fft(self._h, _dp(re), _dp(im), samples, _dp(w), _dp(sr), _dp(si), fft,
                                              ctypes.byref(rows)))
        r = rows.value
        return w[:r], sr[:r], si[:r]

    def set_operators(self, alpha=None, position=None):
        """Alphafile (Raman, SFG) and CD Positionfile record images."""
        keep = []
        args = []
        for x in (alpha, position):
            if x is None:
                args += [None, 0]
                continue
            a = np.ascontiguousarray(np.frombuffer(x, dtype=np.uint8) if isinstance(x, (bytes, bytearray)) else x)
            keep.append(a)
            args += [a.ctypes.data, a.nbytes]
        self._check(lib().nise_set_operators(self._h, *args))
        return self

    def linear(self):
        """LD, Raman, SFG, DOS or CD (the context's technique): raw response
        sums re[channel][tmax1], im[channel][tmax1] and the normaliser."""
        t = self.params.tmax1
        re = np.zeros((4, t))
        im = np.zeros((4, t))
        ch = ctypes.c_int(0)
        n = ctypes.c_int(0)
        self._check(lib().nise_linear(self._h, _dp(re), _dp(im), 4, ctypes.byref(ch), ctypes.byref(n)))
        return re[:ch.value], im[:ch.value], n.value

    def twodir(self):
        p = self.params
        R = np.zeros((12, p.tmax3, p.tmax1))
        n = ctypes.c_int(0)
        self._check(lib().nise_2dir(self._h, _dp(R), ctypes.byref(n)))
        return R, n.value

    def _vec_dtype(self):
        return np.float32 if self.params.precision == FP32 else np.float64

    def propagate(self, H, re, im, sign=1):
        """One propagate_vector step for each row of re/im with its own packed H row."""
        H = np.ascontiguousarray(H, dtype=np.float32)
        dt = self._vec_dtype()
        re = np.array(re, dtype=dt, order="C", copy=True)
        im = np.array(im, dtype=dt, order="C", copy=True)
        nvec = re.shape[0]
        self._check(lib().nise_propagate(self._h, H.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), re.ctypes.data,
                                         im.ctypes.data, nvec, sign))
        return re, im

    def propagate_doubles(self, H, re, im, anh=None):
        H = np.ascontiguousarray(H, dtype=np.float32)
        dt = self._vec_dtype()
        re = np.array(re, dtype=dt, order="C", copy=True)
        im = np.array(im, dtype=dt, order="C", copy=True)
        a = None if anh is None else np.ascontiguousarray(anh, dtype=np.float32)
        self._check(lib().nise_propagate_doubles(
            self._h, H.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), re.ctypes.data, im.ctypes.data, re.shape[0],
            None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return re, im

    def absorption_model(self, shift, scale, lifetime):
        """Differentiable FP64 spectrum (nise_absorption_model): site shifts
        (cm^-1), coupling scale and lifetime (fs) -> (w, spec_re, spec_im)."""
        fft = max(self.params.fft, self.params.tmax1)
        w, sr, si = np.zeros(fft), np.zeros(fft), np.zeros(fft)
        rows = ctypes.c_int(0)
        shift = np.ascontiguousarray(shift, dtype=np.float64)
        self._check(lib().nise_absorption_model(self._h, _dp(shift), ctypes.c_double(scale), ctypes.c_double(lifetime),
                                                _dp(w), _dp(sr), _dp(si), fft, ctypes.byref(rows)))
        r = rows.value
        return w[:r], sr[:r], si[:r]

    def backward_absorption(self, shift, scale, lifetime, dl_dre, dl_dim):
        """Adjoint of absorption_model: (dL/dshift [N], dL/dscale, dL/dlifetime)."""
        shift = np.ascontiguousarray(shift, dtype=np.float64)
        dl_dre = np.ascontiguousarray(dl_dre, dtype=np.float64)
        dl_dim = np.ascontiguousarray(dl_dim, dtype=np.float64)
        g = np.zeros(self.params.singles)
        gs, gl = ctypes.c_double(0), ctypes.c_double(0)
        self._check(lib().nise_backward_absorption(self._h, _dp(shift), ctypes.c_double(scale),
                                                   ctypes.c_double(lifetime), _dp(dl_dre), _dp(dl_dim), len(dl_dre),
                                                   _dp(g), ctypes.byref(gs), ctypes.byref(gl)))
        return g, gs.value, gl.value

    def tune(self):
        """Autotune the absorption kernels for this context's job (nise_absorption_tune)."""
        self._check(lib().nise_absorption_tune(self._h))

    def set_stream(self, stream_ptr):
        """Enqueue this context's device work on a caller CUDA stream (int handle, 0 = own)."""
        self._check(lib().nise_set_stream(self._h, ctypes.c_void_p(stream_ptr or None)))

    def timing(self):
        """(total ms, main kernel ms, kernel launches) of the last compute call."""
        tot = ctypes.c_double(0)
        main = ctypes.c_double(0)
        n = ctypes.c_long(0)
        lib().nise_last_timing(self._h, ctypes.byref(tot), ctypes.byref(main), ctypes.byref(n))
        return tot.value, main.value, n.value

    def work(self):
        """(flops, hbm_bytes) of the last compute call's main kernel(s)."""
        f = ctypes.c_double(0)
        b = ctypes.c_double(0)
        lib().nise_last_work(self._h, ctypes.byref(f), ctypes.byref(b))
        return f.value, b.value


def fp32_peak(device=0):
    """Measured FP32 FMA throughput (TFLOP/s) of a device."""
    t = ctypes.c_double(0)
    rc = lib().nise_probe_fp32_peak(device, ctypes.byref(t))
    if rc != 0:
        raise NiseError(rc, lib().nise_global_error().decode())
    return t.value


def write_td_absorption(path, params, re, im, samples):
    rc = lib().nise_write_td_absorption(os.fsencode(path), ctypes.byref(params), _dp(np.ascontiguousarray(re)),
                                        _dp(np.ascontiguousarray(im)), samples)
    if rc != 0:
        raise NiseError(rc, "cannot write %s" % path)


def write_spectrum(path, w, sr, si):
    rc = lib().nise_write_spectrum(os.fsencode(path), _dp(np.ascontiguousarray(w)), _dp(np.ascontiguousarray(sr)),
                                   _dp(np.ascontiguousarray(si)), len(w))
    if rc != 0:
        raise NiseError(rc, "cannot write %s" % path)


def write_2d(path, params, re, im, count):
    rc = lib().nise_write_2d(os.fsencode(path), ctypes.byref(params), _dp(np.ascontiguousarray(re)),
                             _dp(np.ascontiguousarray(im)), count)
    if rc != 0:
        raise NiseError(rc, "cannot write %s" % path)


def fft2d_files(input_path, device=0):
    """The 2DFFT program (2DFFT.c): 2D spectra from the R*.dat files of the
    current directory, with the keyword file `input_path`."""
    rc = lib().nise_2dfft_files(os.fsencode(input_path), device)
    if rc != 0:
        raise NiseError(rc, lib().nise_global_error().decode())


class Batch:
    """Many contexts' absorption jobs as one CUDA graph (nise_batch_*)."""

    def __init__(self, contexts, autotune=False):
        self.contexts = list(contexts)
        arr = (ctypes.c_void_p * len(self.contexts))(*[c._h for c in self.contexts])
        h = ctypes.c_void_p()
        rc = lib().nise_batch_create(arr, len(self.contexts), 1 if autotune else 0, ctypes.byref(h))
        if rc != 0:
            raise NiseError(rc, lib().nise_global_error().decode())
        self._h = h

    def _check(self, rc):
        if rc != 0:
            raise NiseError(rc, lib().nise_batch_error(self._h).decode())

    def run(self):
        self._check(lib().nise_batch_run(self._h))

    def result(self, i):
        t = self.contexts[i].params.tmax1
        re, im, n = np.zeros(t), np.zeros(t), ctypes.c_int(0)
        self._check(lib().nise_batch_result(self._h, i, _dp(re), _dp(im), ctypes.byref(n)))
        return re, im, n.value

    def spectrum(self, i):
        p = self.contexts[i].params
        fft = max(p.fft, p.tmax1)
        w, sr, si = np.zeros(fft), np.zeros(fft), np.zeros(fft)
        rows = ctypes.c_int(0)
        self._check(lib().nise_batch_spectrum(self._h, i, _dp(w), _dp(sr), _dp(si), fft, ctypes.byref(rows)))
        r = rows.value
        return w[:r], sr[:r], si[:r]

    def timing(self):
        """(device ms of the last run, kernels in the graph)."""
        ms, n = ctypes.c_double(0), ctypes.c_long(0)
        lib().nise_batch_timing(self._h, ctypes.byref(ms), ctypes.byref(n))
        return ms.value, n.value

    def close(self):
        if self._h:
            lib().nise_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

