"""Generate the golden fixtures of the 2D FFT step (the reference's 2DFFT program).

Each case writes seeded synthetic 2D response files in the reference's print2D
format (MPI_subs.c:20-34: "t1 t2 t3 Re Im", t1 outer, t3 inner), a keyword file,
and optionally a Waitingtime.dat, then runs the reference's 2DFFT program
compiled from its own sources (oracle/_ref/2DFFT, recipe in oracle/Makefile;
its FFTW calls go to the FP64 transform of oracle/shim) in a scratch directory.
Every file the program writes is stored as text in fft2d_<case>.npz together
with the inputs, so the tests can rebuild the directory and compare.

Run from the repository root:  python tests/golden/make_golden_fft2d.py
"""
import json
import os
import shutil
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_2DFFT = os.path.join(ROOT, "oracle", "_ref", "2DFFT")

POL = ("par", "per", "cro")

BASE = dict(Timestep=2, RunTimes="16 0 16", FFT=256, MinFrequencies="1200 1200 1200",
            MaxFrequencies="2100 2100 2100", Technique="2DIR")

CASES = {
    "dislin": dict(keywords=dict(BASE)),
    "gnuplot_apodised": dict(keywords=dict(BASE, RunTimes="24 0 20", FFT=512, Format="Gnuplot", Window="Hann",
                                           Homogeneous=400, Inhomogeneous=300)),
    "matlab": dict(keywords=dict(BASE, Format="Matlab", Homogeneous=600)),
    "waiting_times": dict(keywords=dict(BASE, RunTimes="12 0 12", FFT=192), waiting=["0", "100"]),
    "raman": dict(keywords=dict(BASE, Technique="2DIRraman", Format="Gnuplot"), raman=True),
    "missing_cro": dict(keywords=dict(BASE, Inhomogeneous=200), pols=("par", "per")),
    "odd_fft": dict(keywords=dict(BASE, RunTimes="10 0 14", FFT=270, Window="Hann")),
}


def response(rng, kind, tmax1, tmax3, dt):
    """Seeded damped oscillations around the rotating-frame centre (cm^-1 offsets)."""
    c_v = 2.99792458e-5
    w = rng.uniform(-300, 300, size=(3, 2)) * 2 * np.pi * c_v      # rad/fs
    amp = rng.normal(size=3) + 1j * rng.normal(size=3)
    t1 = np.arange(tmax1)[:, None] * dt
    t3 = np.arange(tmax3)[None, :] * dt
    sign = -1 if kind == "I" else 1
    R = np.zeros((tmax1, tmax3), complex)
    for k in range(3):
        R += amp[k] * np.exp(1j * (sign * w[k, 0] * t1 + w[k, 1] * t3) - (t1 + t3) / 300.0)
    return R * 1e-2


def write_response(path, R, dt, t2):
    with open(path, "w") as f:
        for i in range(R.shape[0]):
            for k in range(R.shape[1]):
                f.write("%f %f %f %e %e\n" % (i * dt, t2 * dt, k * dt, R[i, k].real, R[i, k].imag))


def inputs(name, case):
    """Input file texts of a case: {file name: text}."""
    kw = case["keywords"]
    rng = np.random.default_rng(sum(map(ord, name)))
    tmax1, _, tmax3 = (int(x) for x in kw["RunTimes"].split())
    dt = float(kw["Timestep"])
    files = {"input": "".join("%s %s\n" % (k, v) for k, v in kw.items())}
    waits = case.get("waiting", [None])
    if case.get("waiting"):
        files["Waitingtime.dat"] = "".join(w + "\n" for w in waits)
    tmp = tempfile.mkdtemp()
    try:
        for wt in waits:
            for p in case.get("pols", POL):
                for kind in ("I", "II"):
                    if case.get("raman"):
                        fn = "R%s%s.IRraman.dat" % (p, kind)
                    elif wt is not None:
                        fn = "R%s%s_%sfs.dat" % (p, kind, wt)
                    else:
                        fn = "R%s%s.dat" % (p, kind)
                    path = os.path.join(tmp, fn)
                    write_response(path, response(rng, kind, tmax1, tmax3, dt), dt, 0 if wt is None else int(wt) // 2)
                    with open(path) as f:
                        files[fn] = f.read()
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return files


def main():
    manifest = {}
    for name, case in CASES.items():
        work = tempfile.mkdtemp(prefix="golden_fft2d_")
        try:
            ins = inputs(name, case)
            for fn, text in ins.items():
                with open(os.path.join(work, fn), "w") as f:
                    f.write(text)
            subprocess.run([REF_2DFFT, "input"], cwd=work, check=True, stdout=subprocess.DEVNULL)
            outs = {fn: open(os.path.join(work, fn)).read() for fn in sorted(os.listdir(work)) if fn not in ins}
            np.savez_compressed(os.path.join(HERE, "fft2d_%s.npz" % name),
                                inputs=np.array(json.dumps(ins)), outputs=np.array(json.dumps(outs)))
            manifest[name] = sorted(outs)
            print("golden fft2d", name, len(ins), "inputs ->", sorted(outs))
        finally:
            shutil.rmtree(work, ignore_errors=True)
    with open(os.path.join(HERE, "fft2d_cases.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
