"""Seeded synthetic NISE trajectories (GROBIN binary layout) and keyword files.

The workloads mirror the benchmark configurations of the NISE propagation path:
  c0  linear absorption, Trotter "Coupling": 16-site chain, 10000 frames x 2 fs
  c1  linear absorption, "Sparse": 1024 sites on an 8x8x16 lattice, 100000 x 1 fs
  c2  2DIR, "Coupling": 64 oscillators in a random cluster, 20000 x 2 fs
  c3  absorption for the adjoint: 256-site chain, 20000 frames (c3_spec, c3_keywords)
  c4  mixed-size batch: 64 lattice trajectories, 8..2048 sites, 5000 x 1 fs
Every function takes overrides so tests can shrink sites, frames and times.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))

CHAIN, LATTICE, CLUSTER = 0, 1, 2
FULL, COUPLING = 0, 1


class SynthSpec(ctypes.Structure):
    _fields_ = [
        ("n_sites", ctypes.c_int), ("frames", ctypes.c_int), ("dt_fs", ctypes.c_float),
        ("geometry", ctypes.c_int), ("spacing", ctypes.c_float), ("eps0", ctypes.c_float),
        ("sigma", ctypes.c_float), ("tau_fs", ctypes.c_float), ("j_nn", ctypes.c_float),
        ("j_sigma", ctypes.c_float), ("jcut", ctypes.c_float), ("mu_jitter", ctypes.c_float),
        ("ham_type", ctypes.c_int), ("dipole_frames", ctypes.c_int),
        ("anharm_mean", ctypes.c_float), ("anharm_sigma", ctypes.c_float), ("seed", ctypes.c_uint64),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "libnise_synth.so")
        if not os.path.exists(path):
            from . import build
            build.build_synth()
        _lib = ctypes.CDLL(path)
        _lib.nise_synth_write.argtypes = [ctypes.POINTER(SynthSpec)] + [ctypes.c_char_p] * 5
        _lib.nise_synth_fill.argtypes = [ctypes.POINTER(SynthSpec)] + [ctypes.c_void_p] * 5
        _lib.nise_synth_energy_record_floats.argtypes = [ctypes.POINTER(SynthSpec)]
        _lib.nise_synth_energy_record_floats.restype = ctypes.c_long
    return _lib


def spec(**kw):
    s = SynthSpec()
    defaults = dict(n_sites=16, frames=1000, dt_fs=2.0, geometry=CHAIN, spacing=4.5, eps0=1650.0,
                    sigma=10.0, tau_fs=100.0, j_nn=-8.0, j_sigma=2.0, jcut=0.0, mu_jitter=0.05,
                    ham_type=FULL, dipole_frames=0, anharm_mean=16.0, anharm_sigma=2.0, seed=1)
    defaults.update(kw)
    for k, v in defaults.items():
        setattr(s, k, v)
    return s


def write(s, directory, anharm=False, prefix=""):
    """Write Energy.bin / Dipole.bin (+ Coupling.bin, Anharmonicity.bin,
    OvertoneDipole.bin) into `directory`; returns the path dict."""
    os.makedirs(directory, exist_ok=True)
    p = {k: os.path.join(directory, prefix + v) for k, v in dict(
        energy="Energy.bin", dipole="Dipole.bin", coupling="Coupling.bin",
        anharm="Anharmonicity.bin", overtone="OvertoneDipole.bin").items()}
    rc = lib().nise_synth_write(
        ctypes.byref(s), p["energy"].encode(), p["dipole"].encode(),
        p["coupling"].encode() if s.ham_type == COUPLING else None,
        p["anharm"].encode() if anharm else None, p["overtone"].encode() if anharm else None)
    if rc != 0:
        raise RuntimeError("nise_synth_write failed (%d)" % rc)
    if s.ham_type != COUPLING:
        p["coupling"] = ""
    if not anharm:
        p["anharm"] = p["overtone"] = ""
    return p


def write_positions(directory, n_sites, frames, mode="tdc", seed=1, spacing=5.0, box=0.0, prefix=""):
    """Seeded site positions for couplings computed on the fly (Positionfile,
    dipole-file record layout: int32 tag, then the x, y and z blocks of N
    floats).  Sites sit on a cubic grid of the given spacing (inside `box` when
    a periodic box is given) and move by 0.05 A (standard deviation) per
    frame.  mode "edc" writes two records per frame, the two ends of each
    extended dipole (+-0.6 A along a fixed random direction per site).
    With box > 0 a PBCfile (int32 tag + 3 floats per frame) is written too.
    Returns {"position": path[, "pbc": path]}."""
    import numpy as np
    rng = np.random.default_rng(seed)
    side = int(np.ceil(n_sites ** (1.0 / 3)))
    grid = np.array([(i % side, (i // side) % side, i // (side * side)) for i in range(n_sites)], float) * spacing
    base = grid + rng.normal(0, 0.3, size=grid.shape)
    u = rng.normal(size=(n_sites, 3))
    u /= np.linalg.norm(u, axis=1)[:, None]
    out = {"position": os.path.join(directory, prefix + "Position.bin")}
    with open(out["position"], "wb") as f:
        for t in range(frames):
            r = base + rng.normal(0, 0.05, size=base.shape)
            ends = [r] if mode == "tdc" else [r - 0.6 * u, r + 0.6 * u]
            for e in ends:
                if box > 0:
                    e = np.mod(e, box)
                f.write(np.int32(t).tobytes())
                f.write(np.ascontiguousarray(e.T, dtype=np.float32).tobytes())
    if box > 0:
        out["pbc"] = os.path.join(directory, prefix + "PBC.bin")
        with open(out["pbc"], "wb") as f:
            for t in range(frames):
                f.write(np.int32(t).tobytes())
                f.write(np.array([box, box, box], np.float32).tobytes())
    return out


def write_alpha(directory, n_sites, frames, seed=1, prefix=""):
    """Seeded polarisability records (Alphafile, read_alpha layout: int32 tag,
    then the xx, xy, xz, yy, yz, zz blocks of N floats).  Each site has an
    anisotropic tensor (diagonal near 1, off-diagonal near 0.2) that moves by
    2 % per frame.  Returns {"alpha": path}."""
    import numpy as np
    rng = np.random.default_rng(seed)
    base = np.empty((6, n_sites))
    base[[0, 3, 5]] = rng.uniform(0.5, 1.5, size=(3, n_sites))
    base[[1, 2, 4]] = rng.normal(0, 0.2, size=(3, n_sites))
    out = {"alpha": os.path.join(directory, prefix + "Alpha.bin")}
    with open(out["alpha"], "wb") as f:
        for t in range(frames):
            a = base * (1 + rng.normal(0, 0.02, size=base.shape))
            f.write(np.int32(t).tobytes())
            f.write(np.ascontiguousarray(a, dtype=np.float32).tobytes())
    return out


# ---------------------------------------------------------------- workloads
def c0_spec(**kw):
    d = dict(n_sites=16, frames=10000, dt_fs=2.0, geometry=CHAIN, eps0=1650.0, sigma=10.0, tau_fs=100.0,
             j_nn=-8.0, j_sigma=2.0, mu_jitter=0.05, ham_type=FULL, seed=20170)
    d.update(kw)
    return spec(**d)


def c0_keywords(**kw):
    d = dict(Propagation="Coupling", Couplingcut=0.1, Singles=16, Length=10000, Samplerate=20,
             Timestep=2, RunTimes="128 0 0", Lifetime=1000, Trotter=5, MinFrequencies="1550 1550 1550",
             MaxFrequencies="1750 1750 1750", Technique="Absorption", HamiltonianType="Full")
    d.update(kw)
    return d


def c3_spec(**kw):
    """Adjoint workload: the c0 chain statistics on 256 sites, 20000 frames."""
    d = dict(n_sites=256, frames=20000)
    d.update(kw)
    return c0_spec(**d)


def c3_keywords(**kw):
    d = dict(Singles=256, Length=20000)
    d.update(kw)
    return c0_keywords(**d)


def c1_spec(**kw):
    d = dict(n_sites=1024, frames=100000, dt_fs=1.0, geometry=LATTICE, spacing=8.0, eps0=15000.0,
             sigma=300.0, tau_fs=50.0, jcut=2.0, mu_jitter=0.0, ham_type=COUPLING, dipole_frames=1,
             seed=20171)
    d.update(kw)
    return spec(**d)


def c1_keywords(**kw):
    d = dict(Propagation="Sparse", Threshold=0, Couplingcut=2, Singles=1024, Length=100000, Samplerate=50,
             Timestep=1, RunTimes="256 0 0", Lifetime=500, Trotter=5, MinFrequencies="13500 13500 13500",
             MaxFrequencies="16500 16500 16500", Technique="Absorption", HamiltonianType="Coupling")
    d.update(kw)
    return d


def c2_spec(**kw):
    d = dict(n_sites=64, frames=20000, dt_fs=2.0, geometry=CLUSTER, spacing=6.0, eps0=1650.0, sigma=12.0,
             tau_fs=200.0, jcut=0.0, mu_jitter=0.0, ham_type=COUPLING, dipole_frames=1, seed=20172)
    d.update(kw)
    return spec(**d)


def c2_keywords(**kw):
    d = dict(Propagation="Coupling", Couplingcut=0.1, Singles=64, Length=20000, Samplerate=100, Timestep=2,
             RunTimes="64 0 64", Trotter=5, Anharmonicity=16, Lifetime=1000,
             MinFrequencies="1550 1550 1550", MaxFrequencies="1750 1750 1750", Technique="2DIR",
             HamiltonianType="Coupling")
    d.update(kw)
    return d


def write_input(path, keywords, files):
    """Write a NISE keyword file.  `files` is the dict returned by write()."""
    lines = ["Hamiltonianfile %s" % files["energy"], "Dipolefile %s" % files["dipole"]]
    if files.get("coupling"):
        lines.append("Couplingfile %s" % files["coupling"])
    if files.get("anharm"):
        lines.append("Anharmonicfile %s" % files["anharm"])
        lines.append("Overtonedipolefile %s" % files["overtone"])
    if files.get("shift"):
        lines.append("SingleShiftfile %s" % files["shift"])
    if files.get("position"):
        lines.append("Positionfile %s" % files["position"])
    if files.get("pbc"):
        lines.append("PBCfile %s" % files["pbc"])
    if files.get("alpha"):
        lines.append("Alphafile %s" % files["alpha"])
    for k, v in keywords.items():
        lines.append("%s %s" % (k, v))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path
