"""Generate the golden fixtures of the NISE propagation path.

Each case is a seeded synthetic trajectory (nise_2017_b200.synth, regenerated
by the tests from the spec stored in cases.json) run through the reference
program compiled from its own sources (oracle/_ref/NISE_acc, recipe in
oracle/Makefile).  The reference's output files are stored as arrays:
  absorption cases: td = TD_Absorption.dat columns, spec = Absorption.dat columns
  2D cases:         R  = [6 files][Re, Im][t3][t1] of RparI.dat ... RcroII.dat

Run from the repository root:  python tests/golden/make_golden.py [case ...]
"""
import json
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from nise_2017_b200 import synth  # noqa: E402
import oracle  # noqa: E402

L, C = synth.LATTICE, synth.CLUSTER
CASES = {
    # linear absorption
    "abs_coupling_full": dict(
        spec=dict(n_sites=16, frames=600, dt_fs=2.0, geometry=synth.CHAIN, seed=11),
        keywords=synth.c0_keywords(Length=600, RunTimes="64 0 0", FFT=1024)),
    "abs_coupling_static": dict(
        spec=dict(n_sites=24, frames=400, dt_fs=1.0, geometry=L, spacing=8.0, eps0=15000.0, sigma=300.0,
                  tau_fs=50.0, jcut=2.0, mu_jitter=0.0, ham_type=synth.COUPLING, dipole_frames=1, seed=12),
        keywords=synth.c1_keywords(Singles=24, Length=400, RunTimes="48 0 0", Samplerate=40,
                                   Propagation="Coupling", FFT=512)),
    "abs_sparse_static": dict(
        spec=dict(n_sites=32, frames=400, dt_fs=1.0, geometry=L, spacing=8.0, eps0=15000.0, sigma=300.0,
                  tau_fs=50.0, jcut=2.0, mu_jitter=0.0, ham_type=synth.COUPLING, dipole_frames=1, seed=13),
        keywords=synth.c1_keywords(Singles=32, Length=400, RunTimes="64 0 0", Samplerate=50, FFT=1000)),
    "abs_rk4_full": dict(
        spec=dict(n_sites=12, frames=500, dt_fs=2.0, geometry=synth.CHAIN, seed=14),
        keywords=synth.c0_keywords(Singles=12, Length=500, RunTimes="64 0 0", Propagation="RK4", Trotter=3,
                                   FFT=2048)),
    "abs_shift_window": dict(
        spec=dict(n_sites=10, frames=400, dt_fs=2.0, geometry=synth.CHAIN, seed=15),
        keywords=synth.c0_keywords(Singles=10, Length=400, RunTimes="50 0 0", Samplerate=30, Window="Hann",
                                   Homogeneous=800, Inhomogeneous=300, FFT=256, BeginPoint=1, EndPoint=9),
        shift=[(2, 1.0, 5.0), (7, 1.02, -3.0)]),
    "abs_sparse_full": dict(
        spec=dict(n_sites=12, frames=400, dt_fs=2.0, geometry=synth.CHAIN, seed=16),
        keywords=synth.c0_keywords(Singles=12, Length=400, RunTimes="48 0 0", Samplerate=30, Propagation="Sparse",
                                   Threshold=0, FFT=512)),
    "abs_sparse_trunc": dict(
        spec=dict(n_sites=10, frames=400, dt_fs=2.0, geometry=synth.CHAIN, j_nn=-12.0, seed=17),
        keywords=synth.c0_keywords(Singles=10, Length=400, RunTimes="40 0 0", Samplerate=30, Propagation="Sparse",
                                   Threshold=100000, FFT=256)),
    "abs_sparse_trunc_static": dict(
        spec=dict(n_sites=24, frames=300, dt_fs=1.0, geometry=L, spacing=8.0, eps0=15000.0, sigma=300.0,
                  tau_fs=50.0, jcut=2.0, mu_jitter=0.0, ham_type=synth.COUPLING, dipole_frames=1, seed=18),
        keywords=synth.c1_keywords(Singles=24, Length=300, RunTimes="40 0 0", Samplerate=40, Threshold=20000,
                                   FFT=512)),
    "abs_tdc": dict(
        spec=dict(n_sites=10, frames=300, dt_fs=2.0, geometry=C, sigma=12.0, ham_type=synth.COUPLING,
                  dipole_frames=300, mu_jitter=0.05, seed=31),
        keywords=synth.c0_keywords(Singles=10, Length=300, RunTimes="40 0 0", Samplerate=30,
                                   HamiltonianType="TransitionDipole", Couplingcut=0.1, FFT=512),
        positions=dict(mode="tdc", seed=32, spacing=5.0)),
    "abs_edc_pbc": dict(
        spec=dict(n_sites=9, frames=300, dt_fs=2.0, geometry=C, sigma=12.0, ham_type=synth.COUPLING,
                  dipole_frames=300, mu_jitter=0.05, seed=33),
        keywords=synth.c0_keywords(Singles=9, Length=300, RunTimes="40 0 0", Samplerate=30,
                                   HamiltonianType="ExtendedDipole", Couplingcut=0.1, FFT=512),
        positions=dict(mode="edc", seed=34, spacing=5.0, box=14.0)),
    "2d_tdc": dict(
        spec=dict(n_sites=5, frames=300, dt_fs=2.0, geometry=C, sigma=12.0, ham_type=synth.COUPLING,
                  dipole_frames=300, mu_jitter=0.05, seed=35),
        keywords=synth.c2_keywords(Singles=5, Length=300, RunTimes="8 0 8", Samplerate=40,
                                   HamiltonianType="TransitionDipole"),
        positions=dict(mode="tdc", seed=36, spacing=4.5)),
    # 2DIR family
    "2d_coupling": dict(
        spec=dict(n_sites=5, frames=300, dt_fs=2.0, geometry=C, spacing=6.0, sigma=12.0, tau_fs=200.0,
                  mu_jitter=0.0, ham_type=synth.COUPLING, dipole_frames=1, seed=21),
        keywords=synth.c2_keywords(Singles=5, Length=300, RunTimes="8 0 8", Samplerate=40)),
    "2d_coupling_t2": dict(
        spec=dict(n_sites=5, frames=300, dt_fs=2.0, geometry=C, spacing=6.0, sigma=12.0, tau_fs=200.0,
                  mu_jitter=0.0, ham_type=synth.COUPLING, dipole_frames=1, seed=22),
        keywords=synth.c2_keywords(Singles=5, Length=300, RunTimes="8 3 8", Samplerate=40)),
    "2d_rk4": dict(
        spec=dict(n_sites=5, frames=300, dt_fs=2.0, geometry=C, spacing=6.0, sigma=12.0, tau_fs=200.0,
                  mu_jitter=0.0, ham_type=synth.COUPLING, dipole_frames=1, seed=23),
        keywords=synth.c2_keywords(Singles=5, Length=300, RunTimes="8 0 8", Samplerate=40, Propagation="RK4")),
    "2d_sparse": dict(
        spec=dict(n_sites=5, frames=300, dt_fs=2.0, geometry=C, spacing=6.0, sigma=12.0, tau_fs=200.0,
                  mu_jitter=0.0, ham_type=synth.COUPLING, dipole_frames=1, seed=24),
        keywords=synth.c2_keywords(Singles=5, Length=300, RunTimes="8 0 8", Samplerate=40, Propagation="Sparse",
                                   Threshold=0)),
    "2d_sparse_trunc": dict(
        spec=dict(n_sites=5, frames=300, dt_fs=2.0, geometry=C, spacing=5.0, sigma=12.0, tau_fs=200.0,
                  mu_jitter=0.0, ham_type=synth.COUPLING, dipole_frames=1, seed=27),
        keywords=synth.c2_keywords(Singles=5, Length=300, RunTimes="8 0 8", Samplerate=40, Propagation="Sparse",
                                   Threshold=20000)),
    "2d_full_anhfile": dict(
        spec=dict(n_sites=4, frames=260, dt_fs=2.0, geometry=synth.CHAIN, j_nn=-6.0, j_sigma=1.5, seed=25),
        keywords=synth.c2_keywords(Singles=4, Length=260, RunTimes="6 0 6", Samplerate=30, Anharmonicity=0,
                                   HamiltonianType="Full"),
        anharm=True),
    "2d_gbir": dict(
        spec=dict(n_sites=5, frames=300, dt_fs=2.0, geometry=C, spacing=6.0, seed=26, ham_type=synth.COUPLING,
                  dipole_frames=1, mu_jitter=0.0),
        keywords=synth.c2_keywords(Singles=5, Length=300, RunTimes="8 2 8", Samplerate=40, Technique="GBIR")),
    "2d_seir": dict(
        spec=dict(n_sites=5, frames=300, dt_fs=2.0, geometry=C, spacing=6.0, seed=26, ham_type=synth.COUPLING,
                  dipole_frames=1, mu_jitter=0.0),
        keywords=synth.c2_keywords(Singles=5, Length=300, RunTimes="8 2 8", Samplerate=40, Technique="SEIR")),
    "2d_eair": dict(
        spec=dict(n_sites=5, frames=300, dt_fs=2.0, geometry=C, spacing=6.0, seed=26, ham_type=synth.COUPLING,
                  dipole_frames=1, mu_jitter=0.0),
        keywords=synth.c2_keywords(Singles=5, Length=300, RunTimes="8 2 8", Samplerate=40, Technique="EAIR")),
    # 2DUVvis family (calc_2DES.c): two-level doubles, no anharmonicity or overtone files
    "2d_uvvis": dict(
        spec=dict(n_sites=5, frames=300, dt_fs=2.0, geometry=C, spacing=6.0, sigma=12.0, tau_fs=200.0,
                  mu_jitter=0.0, ham_type=synth.COUPLING, dipole_frames=1, seed=41),
        keywords=synth.c2_keywords(Singles=5, Length=300, RunTimes="8 2 8", Samplerate=40, Technique="2DUVvis",
                                   Anharmonicity=0)),
    "2d_uvvis_rk4": dict(
        spec=dict(n_sites=5, frames=300, dt_fs=2.0, geometry=C, spacing=6.0, sigma=12.0, tau_fs=200.0,
                  mu_jitter=0.0, ham_type=synth.COUPLING, dipole_frames=1, seed=42),
        keywords=synth.c2_keywords(Singles=5, Length=300, RunTimes="8 0 8", Samplerate=40, Technique="2DUVvis",
                                   Propagation="RK4", Anharmonicity=0)),
    "2d_uvvis_sparse": dict(
        spec=dict(n_sites=5, frames=300, dt_fs=2.0, geometry=C, spacing=6.0, sigma=12.0, tau_fs=200.0,
                  mu_jitter=0.0, ham_type=synth.COUPLING, dipole_frames=1, seed=43),
        keywords=synth.c2_keywords(Singles=5, Length=300, RunTimes="8 0 8", Samplerate=40, Technique="2DUVvis",
                                   Propagation="Sparse", Threshold=0, Anharmonicity=0)),
    "2d_eauvvis_full": dict(
        spec=dict(n_sites=4, frames=260, dt_fs=2.0, geometry=synth.CHAIN, j_nn=-6.0, j_sigma=1.5, seed=44),
        keywords=synth.c2_keywords(Singles=4, Length=260, RunTimes="6 1 6", Samplerate=30, Technique="EAUVvis",
                                   HamiltonianType="Full", Anharmonicity=0)),
    "2d_noeauvvis": dict(
        spec=dict(n_sites=5, frames=300, dt_fs=2.0, geometry=C, spacing=6.0, seed=45, ham_type=synth.COUPLING,
                  dipole_frames=1, mu_jitter=0.0),
        keywords=synth.c2_keywords(Singles=5, Length=300, RunTimes="8 2 8", Samplerate=40,
                                   Technique="noEAUVvis")),
    # linear techniques besides absorption (calc_LD.c, raman.c, sfg.c, calc_DOS.c, calc_CD.c)
    "lin_ld": dict(
        spec=dict(n_sites=10, frames=300, dt_fs=2.0, geometry=synth.CHAIN, seed=51),
        keywords=synth.c0_keywords(Singles=10, Length=300, RunTimes="40 0 0", Samplerate=30, Technique="LD",
                                   FFT=256)),
    "lin_ld_static_sparse": dict(
        spec=dict(n_sites=12, frames=300, dt_fs=1.0, geometry=L, spacing=8.0, eps0=15000.0, sigma=300.0,
                  tau_fs=50.0, jcut=2.0, mu_jitter=0.0, ham_type=synth.COUPLING, dipole_frames=1, seed=52),
        keywords=synth.c1_keywords(Singles=12, Length=300, RunTimes="32 0 0", Samplerate=40, Technique="LD",
                                   Threshold=0, FFT=256)),
    "lin_raman_rk4": dict(
        spec=dict(n_sites=8, frames=300, dt_fs=2.0, geometry=synth.CHAIN, seed=53),
        keywords=synth.c0_keywords(Singles=8, Length=300, RunTimes="40 0 0", Samplerate=30, Technique="Raman",
                                   Propagation="RK4", Trotter=2, FFT=256),
        alpha=dict(seed=54)),
    "lin_sfg_shift": dict(
        spec=dict(n_sites=9, frames=300, dt_fs=2.0, geometry=C, spacing=6.0, sigma=12.0, mu_jitter=0.0,
                  ham_type=synth.COUPLING, dipole_frames=1, seed=55),
        keywords=synth.c2_keywords(Singles=9, Length=300, RunTimes="40 0 0", Samplerate=30, Technique="SFG",
                                   FFT=256),
        shift=[(1, 1.0, 6.0), (4, 0.98, -2.0)], alpha=dict(seed=56)),
    "lin_dos": dict(
        spec=dict(n_sites=10, frames=300, dt_fs=2.0, geometry=synth.CHAIN, seed=57),
        keywords=synth.c0_keywords(Singles=10, Length=300, RunTimes="40 0 0", Samplerate=30, Technique="DOS",
                                   FFT=256)),
    "lin_dos_sparse": dict(
        spec=dict(n_sites=8, frames=300, dt_fs=2.0, geometry=synth.CHAIN, seed=58),
        keywords=synth.c0_keywords(Singles=8, Length=300, RunTimes="32 0 0", Samplerate=30, Technique="DOS",
                                   Propagation="Sparse", Threshold=0, FFT=256)),
    "lin_cd": dict(
        spec=dict(n_sites=8, frames=300, dt_fs=2.0, geometry=synth.CHAIN, seed=59),
        keywords=synth.c0_keywords(Singles=8, Length=300, RunTimes="32 0 0", Samplerate=40, Technique="CD",
                                   FFT=256),
        cd_positions=dict(seed=60, spacing=4.5)),
    "lin_cd_static": dict(
        spec=dict(n_sites=9, frames=300, dt_fs=2.0, geometry=C, spacing=6.0, sigma=12.0, mu_jitter=0.0,
                  ham_type=synth.COUPLING, dipole_frames=1, seed=61),
        keywords=synth.c2_keywords(Singles=9, Length=300, RunTimes="32 0 0", Samplerate=40, Technique="CD",
                                   FFT=256),
        cd_positions=dict(seed=62, spacing=5.0)),
    # luminescence (luminescence.c), from the reference built with zero-initialised
    # automatic variables (oracle/_ref/NISE_lum; its partition function Q is otherwise
    # summed from an uninitialised float)
    "lum_exact": dict(
        spec=dict(n_sites=8, frames=300, dt_fs=2.0, geometry=synth.CHAIN, seed=71),
        keywords=synth.c0_keywords(Singles=8, Length=300, RunTimes="32 0 0", Samplerate=30,
                                   Technique="Luminescence", FFT=256, Temperature=300)),
    "lum_itime": dict(
        spec=dict(n_sites=8, frames=300, dt_fs=2.0, geometry=synth.CHAIN, seed=72),
        keywords=synth.c0_keywords(Singles=8, Length=300, RunTimes="32 0 0", Samplerate=30, Technique="PL",
                                   FFT=256, Temperature=200, ImaginaryTimesteps=20)),
    "lum_static": dict(
        spec=dict(n_sites=9, frames=300, dt_fs=2.0, geometry=C, spacing=6.0, sigma=12.0, mu_jitter=0.0,
                  ham_type=synth.COUPLING, dipole_frames=1, seed=73),
        keywords=synth.c2_keywords(Singles=9, Length=300, RunTimes="32 0 0", Samplerate=30,
                                   Technique="Luminescence", FFT=256)),
}


def materialise(case, directory):
    """Write the trajectory (and shift file) of a case; returns the file dict."""
    s = synth.spec(**case["spec"])
    files = synth.write(s, directory, anharm=case.get("anharm", False))
    if case.get("shift"):
        path = os.path.join(directory, "Shift.txt")
        with open(path, "w") as f:
            f.write("%d\n" % len(case["shift"]))
            for site, a, b in case["shift"]:
                f.write("%d %f %f\n" % (site, a, b))
        files["shift"] = path
    if case.get("positions"):
        pos = case["positions"]
        files.update(synth.write_positions(directory, case["spec"]["n_sites"], case["spec"]["frames"], **pos))
        files["coupling"] = ""  # couplings come from the positions
    if case.get("cd_positions"):  # CD: positions only for the rotatory strengths
        files.update(synth.write_positions(directory, case["spec"]["n_sites"], case["spec"]["frames"],
                                           **case["cd_positions"]))
    if case.get("alpha"):
        files.update(synth.write_alpha(directory, case["spec"]["n_sites"], case["spec"]["frames"], **case["alpha"]))
    return files


def main(names=None):
    """Regenerate every case, or only `names` (kept in cases.json with the rest)."""
    manifest = {}
    if names:
        with open(os.path.join(HERE, "cases.json")) as f:
            manifest = json.load(f)
    for name, case in CASES.items():
        if names and name not in names:
            continue
        work = tempfile.mkdtemp(prefix="golden_")
        try:
            files = materialise(case, work)
            inp = synth.write_input(os.path.join(work, "input"), case["keywords"], files)
            tech = case["keywords"]["Technique"]
            oracle.run_reference(inp, work, binary="NISE_lum" if oracle.TECHNIQUES.get(tech) == 16 else "NISE_acc")
            out = {}
            if tech == "Absorption":
                out["td"] = np.loadtxt(os.path.join(work, "TD_Absorption.dat"), ndmin=2)
                out["spec"] = np.loadtxt(os.path.join(work, "Absorption.dat"), ndmin=2)
            elif tech in oracle.LINEAR_FILES:
                # per channel: td [tmax1][t, Re, Im], spec [rows][w, Re, Im]
                out["td"] = np.stack([np.loadtxt(os.path.join(work, td), ndmin=2) for td, _ in oracle.LINEAR_FILES[tech]
                                      if td])
                out["spec"] = np.stack([np.loadtxt(os.path.join(work, sp), ndmin=2)
                                        for _, sp in oracle.LINEAR_FILES[tech]])
            else:
                p = oracle.params(case["keywords"], files)
                R = np.zeros((6, 2, p.tmax3, p.tmax1))
                for k, fn in enumerate(oracle.R2D_FILES):
                    R[k, 0], R[k, 1] = oracle.read_2d(os.path.join(work, fn), p.tmax1, p.tmax3)
                out["R"] = R
            np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
            manifest[name] = {k: v for k, v in case.items()}
            print("golden", name, {k: v.shape for k, v in out.items()})
        finally:
            shutil.rmtree(work, ignore_errors=True)
    with open(os.path.join(HERE, "cases.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main(sys.argv[1:])
