"""Golden fixtures at the benchmark sizes (N = 1024 lattice, N = 64 cluster).

The reference's CPU path costs about 33 s per vector step at N = 1024
(propagate_vec_DIA, propagate.c:60-125: ssyev_ plus naive N^3 loops), so
these fixtures are generated once, here, and the GPU tests only read them.

  large_c1_vectors.npz    8 vectors on the 1024-site lattice propagated 2 steps
                          (Propagation Sparse, Threshold 0) by the reference's
                          own propagate_vector (oracle/_ref/ref_bench), and the
                          same steps with the FP64 exact propagator
  large_c1_absorption.npz linear absorption on the 1024-site lattice:
                          "wide": 400 start points (1200 vectors, more than one
                            wave of 8-vector CTAs), FP64 exact responses
                          "ref":  the first start point, the reference program's
                            TD_Absorption.dat (oracle/_ref/NISE_acc) and the
                            FP64 exact responses
  large_c2_2dir.npz       2DIR on the 64-site cluster (2 start points, t2 = 0
                          and t2 > 0), the reference program's R*.dat files

The trajectories are regenerated by the tests from the stored generator
arguments (nise_2017_b200.synth, seeded).

  large_eig.npz           absorption with per-frame couplings on a 256-site chain
                          (Propagation Sparse, Threshold 0 and truncating), the
                          reference program's TD_Absorption.dat and the FP64
                          exact responses

Run from the repository root:  python tests/golden/make_golden_large.py [c1v] [c1a] [c2] [eig]
"""
import json
import os
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from nise_2017_b200 import synth  # noqa: E402
import oracle  # noqa: E402

C1_VECTORS = dict(spec=dict(frames=2, seed=91), steps=2, nvec=8)
C1_WIDE = dict(spec=dict(frames=408, seed=92),
               keywords=synth.c1_keywords(Length=408, RunTimes="8 0 0", Samplerate=1))
C1_REF = dict(spec=C1_WIDE["spec"],
              keywords=synth.c1_keywords(Length=408, RunTimes="8 0 0", Samplerate=1, EndPoint=1))
# the eigen route above the shared-memory Jacobi's 120 sites: per-frame
# couplings (HamiltonianType Full), exact and truncated
EIG_CASES = {
    "full_256": dict(spec=dict(n_sites=256, frames=60, dt_fs=2.0, geometry=synth.CHAIN, seed=95),
                     keywords=synth.c0_keywords(Singles=256, Length=60, RunTimes="8 0 0", Samplerate=20,
                                                Propagation="Sparse", Threshold=0, EndPoint=1)),
    "trunc_256": dict(spec=dict(n_sites=256, frames=60, dt_fs=2.0, geometry=synth.CHAIN, j_nn=-12.0, seed=96),
                      keywords=synth.c0_keywords(Singles=256, Length=60, RunTimes="8 0 0", Samplerate=20,
                                                 Propagation="Sparse", Threshold=100000, EndPoint=1)),
}
C2_CASES = {
    "t2_0": dict(spec=dict(frames=220, seed=93),
                 keywords=synth.c2_keywords(Length=220, RunTimes="8 0 8", Samplerate=100, EndPoint=2)),
    "t2_4": dict(spec=dict(frames=220, seed=93),
                 keywords=synth.c2_keywords(Length=220, RunTimes="8 4 8", Samplerate=100, EndPoint=2)),
}


def c1_vectors():
    work = tempfile.mkdtemp(prefix="golden_c1v_")
    try:
        files = synth.write(synth.c1_spec(**C1_VECTORS["spec"]), work)
        n, nvec = 1024, C1_VECTORS["nvec"]
        kw = synth.c1_keywords(Length=2)
        H, mu = oracle.read_frames(kw, files, [0])
        rng = np.random.default_rng(94)
        init = np.zeros((nvec, 2, n), np.float32)
        for x in range(3):  # the three dipole start vectors of absorption.c:107-117
            init[x, 0] = mu(0, x)
        for v in range(3, nvec):
            z = rng.normal(size=n) + 1j * rng.normal(size=n)
            z /= np.linalg.norm(z)
            init[v, 0], init[v, 1] = z.real, z.imag
        vin, vout = os.path.join(work, "in.bin"), os.path.join(work, "out.bin")
        init.tofile(vin)
        t0 = time.time()
        cmd = [os.path.join(oracle.REF_DIR, "ref_bench"), files["energy"], files["coupling"], str(n), "0",
               str(kw["Couplingcut"]), str(kw["Timestep"]), str(kw["Trotter"]), "0",
               str(kw["MinFrequencies"]).split()[0], str(kw["MaxFrequencies"]).split()[0], str(nvec),
               str(C1_VECTORS["steps"]), vin, vout]
        env = dict(os.environ, OPENBLAS_NUM_THREADS="1")
        r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, check=True, env=env)
        print(r.stdout.strip(), "%.0f s" % (time.time() - t0))
        ref = np.fromfile(vout, np.float32).reshape(nvec, 2, n)
        U = oracle.exact_propagators(H, oracle.exact_step_factor(kw["Timestep"]))[0]
        c = (init[:, 0].astype(np.float64) + 1j * init[:, 1].astype(np.float64)).T
        for _ in range(C1_VECTORS["steps"]):
            c = U @ c
        exact = np.stack([c.real.T, c.imag.T], 1)
        np.savez_compressed(os.path.join(HERE, "large_c1_vectors.npz"), init=init, ref=ref, exact=exact,
                            meta=json.dumps(dict(C1_VECTORS, keywords=kw)))
        err = np.abs((ref[:, 0] + 1j * ref[:, 1]) - (exact[:, 0] + 1j * exact[:, 1])).max()
        print("large_c1_vectors: reference vs FP64 exact, max |diff| %.3e" % err)
    finally:
        shutil.rmtree(work, ignore_errors=True)


def c1_absorption():
    work = tempfile.mkdtemp(prefix="golden_c1a_")
    try:
        files = synth.write(synth.c1_spec(**C1_WIDE["spec"]), work)
        t0 = time.time()
        wre, wim, wn = oracle.absorption_exact(C1_WIDE["keywords"], files)
        rre, rim, rn = oracle.absorption_exact(C1_REF["keywords"], files)
        print("FP64 exact responses: %.0f s" % (time.time() - t0))
        t0 = time.time()
        inp = synth.write_input(os.path.join(work, "input"), C1_REF["keywords"], files)
        oracle.run_reference(inp, work, timeout=4 * 3600)
        td = np.loadtxt(os.path.join(work, "TD_Absorption.dat"), ndmin=2)
        print("reference NISE_acc: %.0f s" % (time.time() - t0))
        np.savez_compressed(os.path.join(HERE, "large_c1_absorption.npz"),
                            wide_exact=np.stack([wre, wim]), wide_samples=wn,
                            ref_exact=np.stack([rre, rim]), ref_samples=rn, ref_td=td,
                            meta=json.dumps(dict(wide=C1_WIDE, ref=C1_REF)))
        e = np.abs(td[:, 1] + 1j * td[:, 2] - (rre + 1j * rim) / rn).max() / np.abs((rre + 1j * rim) / rn).max()
        print("large_c1_absorption: reference vs FP64 exact %.3e" % e)
    finally:
        shutil.rmtree(work, ignore_errors=True)


def eig_large():
    out = {}
    for name, case in EIG_CASES.items():
        work = tempfile.mkdtemp(prefix="golden_eig_")
        try:
            files = synth.write(synth.spec(**case["spec"]), work)
            inp = synth.write_input(os.path.join(work, "input"), case["keywords"], files)
            t0 = time.time()
            oracle.run_reference(inp, work, timeout=4 * 3600)
            print("reference NISE_acc %s: %.0f s" % (name, time.time() - t0))
            out[name + "_td"] = np.loadtxt(os.path.join(work, "TD_Absorption.dat"), ndmin=2)
            re, im, n = oracle.absorption_exact(case["keywords"], files)
            out[name + "_exact"] = np.stack([re, im])
            out[name + "_samples"] = n
        finally:
            shutil.rmtree(work, ignore_errors=True)
    np.savez_compressed(os.path.join(HERE, "large_eig.npz"), meta=json.dumps(EIG_CASES), **out)


def c2_2dir():
    out = {}
    for name, case in C2_CASES.items():
        work = tempfile.mkdtemp(prefix="golden_c2_")
        try:
            files = synth.write(synth.c2_spec(**case["spec"]), work)
            inp = synth.write_input(os.path.join(work, "input"), case["keywords"], files)
            t0 = time.time()
            oracle.run_reference(inp, work, threads=8, timeout=4 * 3600)
            print("reference NISE_acc 2DIR %s: %.0f s" % (name, time.time() - t0))
            p = oracle.params(case["keywords"], files)
            R = np.zeros((6, 2, p.tmax3, p.tmax1))
            for k, fn in enumerate(oracle.R2D_FILES):
                R[k, 0], R[k, 1] = oracle.read_2d(os.path.join(work, fn), p.tmax1, p.tmax3)
            out[name] = R
        finally:
            shutil.rmtree(work, ignore_errors=True)
    np.savez_compressed(os.path.join(HERE, "large_c2_2dir.npz"), meta=json.dumps(C2_CASES), **out)


if __name__ == "__main__":
    which = sys.argv[1:] or ["c1v", "c1a", "c2", "eig"]
    if "c1v" in which:
        c1_vectors()
    if "c1a" in which:
        c1_absorption()
    if "c2" in which:
        c2_2dir()
    if "eig" in which:
        eig_large()
