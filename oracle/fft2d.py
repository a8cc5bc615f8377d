"""CPU restatement of the reference's 2DFFT program (2DFFT.c:20-830) — TEST
INFRASTRUCTURE ONLY.

Pinned against tests/golden/fft2d_*.npz, the text files that the reference's
own 2DFFT (compiled from its sources, oracle/Makefile) writes for seeded
response files.  Only the tests import this module, as a checker.

run(files) takes the input directory as {file name: text} and returns the
files the program writes, as {file name: text}.  Float variables of the
reference are float32 here and every float expression is evaluated in float32
in the reference's operation order; apodisation factors are float64 as in the
reference's calls to exp()/cos(); the transform is numpy's FP64 forward FFT
(the sign convention of FFTW_FORWARD).
"""
import numpy as np

F = np.float32
C_V = F(2.99792458e-5)            # 2DFFT.c:46
TWO_PI = F(2 * 3.14159265359)     # types.h:7
POL = ("par", "per", "cro")
RAMAN = ("2DIRraman", "2DIRraman1", "2DIRraman2", "2DIRraman3", "2DIRramanI", "2DIRramanII")


def round_ref(x):
    """2DFFT.c:11: (x)>0 ? (long)(x+0.5) : (long)(x-0.5), the +-0.5 in double."""
    x = np.asarray(x, np.float64)
    return np.where(x > 0, np.trunc(x + 0.5), np.trunc(x - 0.5)).astype(np.int64)


def parse(text):
    """Keyword file (2DFFT.c:98-234), strncmp over the label length."""
    kw = dict(fft=0, deltat=F(0), homo=F(0), inhomo=F(0), window=0, form=0, tmax=(0, 0, 0), raman=False,
              wmin=(F(0),) * 3, wmax=(F(0),) * 3)
    for line in text.splitlines(True):
        label = line.split(" ")[0]
        words = line.split()
        value = line[len(label):].lstrip(" ")

        def is_(name):
            return name.startswith(label)
        if is_("FFT"):
            kw["fft"] = int(float(value.split()[0])) if value.split() else 0
            continue
        if is_("Timestep"):
            kw["deltat"] = F(float(value.split()[0]))
            continue
        if is_("Homogeneous"):
            kw["homo"] = F(float(value.split()[0]))
            continue
        if is_("Inhomogeneous"):
            kw["inhomo"] = F(float(value.split()[0]))
            continue
        if is_("Window") and len(words) > 1 and words[1] == "Hann":
            kw["window"] = 1
        if is_("Format"):
            if len(words) > 1:
                kw["form"] = {"Dislin": 0, "Python": 0, "Matlab": 1, "Gnuplot": 2}.get(words[1], kw["form"])
            continue
        if is_("RunTimes"):
            kw["tmax"] = tuple(int(w) for w in words[1:4])
            continue
        if is_("MinFrequencies"):
            kw["wmin"] = tuple(F(float(w)) for w in words[1:4])
            continue
        if is_("MaxFrequencies"):
            kw["wmax"] = tuple(F(float(w)) for w in words[1:4])
            continue
        if is_("Technique"):
            kw["raman"] = len(words) > 1 and words[1] in RAMAN
            continue
    return kw


def read_response(text, kw, kind):
    """2DFFT.c:327-360 (kI) / :477-513 (kII): the n x n transform input."""
    n, dt = kw["fft"], kw["deltat"]
    tmax1, _, tmax3 = kw["tmax"]
    rows = np.array([[float(x) for x in l.split()] for l in text.splitlines() if l.strip()])[:tmax1 * tmax3]
    ti1, ti3 = rows[:, 0].astype(F), rows[:, 2].astype(F)
    rr, ir = rows[:, 3].astype(F), rows[:, 4].astype(F)
    if kind == 0:
        index = round_ref(ti3 / dt + F(n) * ti1 / dt)
    else:
        index = round_ref(ti3 / dt + F(n) * (ti1 / dt))
    if kw["homo"] > 0:
        e = np.exp((-(ti1 + ti3) / F(2) / kw["homo"]).astype(np.float64))
        rr, ir = (rr * e).astype(F), (ir * e).astype(F)
    if kw["inhomo"] > 0:
        d = ti1 - ti3 if kind == 0 else ti1 + ti3
        e = np.exp((-d * d / F(2) / kw["inhomo"] / kw["inhomo"]).astype(np.float64))
        rr, ir = (rr * e).astype(F), (ir * e).astype(F)
    if kw["window"] == 1:
        c1 = np.cos((ti1 * TWO_PI / F(4 * tmax1 - 4) / dt).astype(np.float64))
        c3 = np.cos((ti3 * TWO_PI / F(4 * tmax3 - 4) / dt).astype(np.float64))
        rr = (rr * c1 * c1).astype(F)
        rr = (rr * c3 * c3).astype(F)
        ir = (ir * c1 * c1).astype(F)
        ir = (ir * c3 * c3).astype(F)
    line = np.arange(len(rows))
    half = np.where(line // tmax3 == 0, F(0.5), F(1)) * np.where(line % tmax3 == 0, F(0.5), F(1))
    rr, ir = rr * half, ir * half
    a = np.zeros(n * n, complex)
    ok = (index >= 0) & (index < n * n)
    if kind == 0:
        a[index[ok]] = rr[ok] + 1j * ir[ok].astype(np.float64)
    else:
        np.add.at(a, index[ok], rr[ok].astype(np.float64) + 1j * ir[ok].astype(np.float64))
    return a.reshape(n, n)


def write_spectrum(o, kw, kind, shift1, shift3, rng):
    """Rw*.dat text (2DFFT.c:368-438 kI, :514-624 kII) and the waxis.dat text."""
    n, dt, form = kw["fft"], kw["deltat"], kw["form"]
    (mi1, _, mi3), (ma1, _, ma3) = kw["wmin"], kw["wmax"]
    idx = np.arange(n)
    nf = F(n)
    if kind == 0:
        w1 = np.where(idx >= n // 2, (idx - n).astype(F) / dt / C_V / nf - shift1, idx.astype(F) / dt / C_V / nf - shift1)
        w3 = np.where(idx < n // 2, idx.astype(F) / dt / C_V / nf - shift3, (idx - n).astype(F) / dt / C_V / nf - shift3)
    else:
        sw = F(1) / dt / C_V
        w1 = np.where(idx >= n // 2, idx.astype(F) / dt / C_V / nf + shift1 - sw,
                      (idx + n).astype(F) / dt / C_V / nf + shift1 - sw)
        w3 = np.where(idx < n // 2, (idx + n).astype(F) / dt / C_V / nf + shift3 - sw,
                      idx.astype(F) / dt / C_V / nf + shift3 - sw)
    w1, w3 = w1.astype(F), w3.astype(F)
    order = np.concatenate([np.arange(n // 2, n), np.arange(0, n // 2)])
    out, axis = [], []
    for i in order:
        last_w1 = w1[i]
        for jh, js in enumerate((np.arange(n // 2, n), np.arange(0, n // 2))):
            if kind == 0:
                inside = (w1[i] > -ma1) & (w3[js] < ma3) & (w1[i] < -mi1) & (w3[js] > mi3)
            else:
                inside = (w1[i] < ma1) & (w3[js] < ma3) & (w1[i] > mi1) & (w3[js] > mi3)
            for j in js[inside]:
                x1 = w1[i]
                if kind == 1:
                    rng[0], rng[1] = min(rng[0], x1), max(rng[1], x1)
                    rng[2], rng[3] = min(rng[2], w3[j]), max(rng[3], w3[j])
                    if kw["raman"]:
                        x1 = F(x1 + (shift3 if (i < n // 2 and jh == 0) else shift1))
                if form in (0, 2):
                    out.append("%f %f %e %e\n" % (x1, w3[j], o[i, j].real, o[i, j].imag))
                else:
                    out.append("%e " % o[i, j].imag)
            last_w1 = x1 if (len(js) and inside[-1]) else w1[i]
        row_in = (last_w1 > -ma1) & (last_w1 < -mi1) if kind == 0 else (last_w1 < ma1) & (last_w1 > mi1)
        if form in (1, 2) and row_in:
            out.append("\n")
            if kind == 1 and form == 1:
                axis.append("%f\n" % last_w1)
    return "".join(out), "".join(axis)


def read_table(text, p1, p3, prev, negate):
    """p1 x p3 rows of "%f %f %e %e"; missing rows keep the previous values."""
    vals = [np.float32(float(x)) for x in text.split()]
    t = [a.copy() for a in prev]
    for e in range(p1 * p3):
        if 4 * e + 3 < len(vals):
            for c in range(4):
                t[c].flat[e] = vals[4 * e + c]
        if negate:
            t[0].flat[e] = -t[0].flat[e]
    return t


def table_text(t1, t3, re, im, form):
    out = []
    for k in range(t1.shape[0]):
        for l in range(t1.shape[1]):
            out.append("%f %f %e %e\n" % (t1[k, l], t3[k, l], re[k, l], im[k, l]))
        if form == 2:
            out.append("\n")
    return "".join(out)


def pp_text(v, axis):
    acc = np.zeros(v.shape[1], F)
    for k in range(v.shape[0]):
        acc = (acc + v[k]).astype(F)
    return "### Broadband pump probe spectrum\n" + "".join("%f %e\n" % (axis[l], acc[l]) for l in range(len(acc)))


def one_pass(files, kw, wt, out):
    """2DFFT.c:274-826 for one waiting time (wt None: no Waitingtime.dat)."""
    (mi1, _, mi3), (ma1, _, ma3) = kw["wmin"], kw["wmax"]
    shift1 = F(0.5 * (np.float64(mi1 + ma1)))
    shift3 = F(-0.5 * (np.float64(mi3 + ma3)))

    def names(p, K):
        if kw["raman"]:
            return "R%s%s.IRraman.dat" % (p, K), "Rw%sIRraman.%s.dat" % (p, K)
        t = "R%s%s_%sfs.dat" % (p, K, wt) if wt is not None else "R%s%s.dat" % (p, K)
        return t, "Rw%s.%s.dat" % (p, K)
    for p in POL:
        tn, fn = names(p, "I")
        if tn in files:
            o = np.fft.fft2(read_response(files[tn], kw, 0))
            out[fn], _ = write_spectrum(o, kw, 0, shift1, shift3, None)
    shift3 = F(-shift3)
    rng = [shift1, shift1, shift3, shift3]
    for p in POL:
        tn, fn = names(p, "II")
        if tn in files:
            o = np.fft.fft2(read_response(files[tn], kw, 1))
            rng = [shift1, shift1, shift3, shift3]
            out[fn], ax = write_spectrum(o, kw, 1, shift1, shift3, rng)
            if kw["form"] == 1:
                out["waxis.dat"] = ax
    if kw["form"] == 1:
        return
    n, dt = kw["fft"], kw["deltat"]
    dw = F(1) / dt / C_V / F(n)
    p1 = int(round_ref(F((F(rng[1] - rng[0]) / dw) + F(1))))
    p3 = int(round_ref(F((F(rng[3] - rng[2]) / dw) + F(1))))
    zero = [np.zeros((p1, p3), F) for _ in range(4)]
    kI, kII = zero, [a.copy() for a in zero]
    ax3 = [F(rng[2] + F(F(F(rng[3] - rng[2]) * F(l + 1)) / F(p3))) for l in range(p3)]
    for p in POL:
        if kw["raman"]:
            n1, n2 = "Rw%sIRraman.I.dat" % p, "Rw%sIRraman.II.dat" % p
        else:
            n1, n2 = "Rw%s.I.dat" % p, "Rw%s.II.dat" % p
        if n1 not in out:
            continue
        kI = read_table(out[n1], p1, p3, kI, True)
        if n2 in out:
            kII = read_table(out[n2], p1, p3, kII, False)
        if kw["raman"]:
            out["2DIRraman.I.%s.dat" % p] = table_text(*kI, kw["form"])
            out["2DIRraman.II.%s.dat" % p] = table_text(*kII, kw["form"])
            out["PPIRraman.I.%s.dat" % p] = pp_text(kI[3], kI[1][0])
            out["PPIRraman.II.%s.dat" % p] = pp_text(kII[3], kII[1][0])
            continue
        IR = (kI[3][::-1] + kII[3]).astype(F)
        IRi = (kI[2][::-1] + kII[2]).astype(F)
        sfx = "_%sfs" % wt if wt is not None else ""
        out["2D.%s%s.dat" % (p, sfx)] = table_text(kII[0], kII[1], IRi, IR, kw["form"])
        out["PP.%s%s.dat" % (p, sfx)] = pp_text(IR, ax3)


def run(files):
    """The program on an input directory given as {name: text}; returns {name: text} written."""
    kw = parse(files["input"])
    out = {}
    if "Waitingtime.dat" in files:
        for wt in files["Waitingtime.dat"].split():
            one_pass(files, kw, wt, out)
    else:
        one_pass(files, kw, None, out)
    return out
