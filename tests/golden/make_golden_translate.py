"""Generate the golden fixtures of trajectory format translation (the
reference's translate program).

Each case writes seeded synthetic input files in one of the reference's
formats (GROBIN, SKIBIN, GROASC, MITASC, MITTXT, SPECTRON) and a translate
keyword file, then runs the reference's translate compiled from its own
sources (oracle/_ref/translate, recipe in oracle/Makefile) in a scratch
directory.  Inputs and every file the program writes are stored base64-coded
in translate_<case>.npz, so the tests can rebuild the directory and compare
byte for byte.

Run from the repository root:  python tests/golden/make_golden_translate.py
"""
import base64
import json
import os
import shutil
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_TRANSLATE = os.path.join(ROOT, "oracle", "_ref", "translate")


def system(n, frames, seed):
    """Seeded frames: packed Hamiltonians (cm^-1), dipoles, polarisabilities,
    anharmonicities and overtone dipoles."""
    rng = np.random.default_rng(seed)
    out = []
    for t in range(frames):
        H = np.zeros((n, n))
        H[np.diag_indices(n)] = 1650 + rng.normal(0, 10, n)
        for a in range(n - 1):
            H[a, a + 1] = H[a + 1, a] = rng.normal(-8, 2)
        H[0, n - 1] = H[n - 1, 0] = rng.normal(1.5, 0.3)
        packed = np.array([H[a, b] for a in range(n) for b in range(a, n)], np.float32)
        out.append(dict(tag=10 + t, He=packed, mu=rng.normal(0, 1, 3 * n).astype(np.float32),
                        alpha=rng.normal(0, 1, 6 * n).astype(np.float32),
                        anh=rng.normal(16, 2, n).astype(np.float32),
                        over=rng.normal(0, 1.4, 3 * n).astype(np.float32)))
    return out


def rec(tag, *blocks):
    return np.int32(tag).tobytes() + b"".join(np.asarray(b, np.float32).tobytes() for b in blocks)


def write_inputs(fmt, n, frames, seed, doubles_block=False):
    """{file name: bytes} of a system in an input format."""
    S = system(n, frames, seed)
    nd = n * (n + 1) // 2
    files = {}
    if fmt in ("GROBIN", "SKIBIN"):
        rng = np.random.default_rng(seed + 1)
        e = d = a = an = ov = b""
        for f in S:
            extra_e = [rng.normal(0, 5, nd * (nd + 1) // 2)] if doubles_block else []
            extra_d = [rng.normal(0, 1, 3 * n * nd)] if doubles_block else []
            e += rec(f["tag"], f["He"], *extra_e)
            d += rec(f["tag"] + 100, f["mu"], *extra_d)
            a += rec(f["tag"] + 200, f["alpha"])
            an += rec(f["tag"] + 300, f["anh"])
            ov += rec(f["tag"] + 400, f["over"])
        files.update({"in_E.bin": e, "in_D.bin": d})
        if fmt == "GROBIN":
            files["in_A.bin"] = a
        else:
            files.update({"in_An.bin": an, "in_Ov.bin": ov})
    elif fmt == "GROASC":
        e = d = a = ""
        for f in S:
            e += "%d " % f["tag"] + "".join("%f " % v for v in f["He"]) + "\n"
            d += "%d " % f["tag"] + "".join("%f " % v for v in f["mu"]) + "\n"
            a += "%d " % f["tag"] + "".join("%f " % v for v in f["alpha"]) + "\n"
        files.update({"in_E.txt": e.encode(), "in_D.txt": d.encode(), "in_A.txt": a.encode()})
    elif fmt == "MITASC":
        e = ""
        dx = dy = dz = ""
        for f in S:
            H = np.zeros((n, n), np.float32)
            k = 0
            for i in range(n):
                for j in range(i, n):
                    H[i, j] = H[j, i] = f["He"][k]
                    k += 1
            # rows separated by an extra tab, the layout the reader expects
            e += "\t".join("\t".join("%f" % v for v in H[i]) + "\t" for i in range(n)) + "\n"
            dx += "".join("%f\t" % v for v in f["mu"][:n]) + "\n"
            dy += "".join("%f\t" % v for v in f["mu"][n:2 * n]) + "\n"
            dz += "".join("%f\t" % v for v in f["mu"][2 * n:]) + "\n"
        files.update({"in_E.txt": e.encode(), "in_Dx.txt": dx.encode(), "in_Dy.txt": dy.encode(),
                      "in_Dz.txt": dz.encode()})
    elif fmt == "MITTXT":
        e = d = ""
        for f in S:
            H = np.zeros((n, n), np.float32)
            k = 0
            for i in range(n):
                for j in range(i, n):
                    H[i, j] = H[j, i] = f["He"][k]
                    k += 1
            e += "".join("".join("%f " % v for v in H[i]) + "\n" for i in range(n)) + "\n"
            d += "".join("%f %f %f \n" % (f["mu"][i], f["mu"][n + i], f["mu"][2 * n + i]) for i in range(n)) + "\n"
        files.update({"in_E.txt": e.encode(), "in_D.txt": d.encode()})
    elif fmt == "SPECTRON":
        e = d = ""
        for t, f in enumerate(S):
            H = np.zeros((n, n), np.float32)
            k = 0
            for i in range(n):
                for j in range(i, n):
                    H[i, j] = H[j, i] = f["He"][k]
                    k += 1
            e += "SNAPSHOT %d\n" % (t + 1) + "".join("".join("%f " % H[i, j] for j in range(i + 1)) + "\n"
                                                      for i in range(n))
            d += "SNAPSHOT %d\n" % (t + 1) + "".join(
                "%f %f %f \n" % (f["mu"][i], f["mu"][n + i], f["mu"][2 * n + i]) for i in range(n))
        files.update({"in_E.txt": e.encode(), "in_D.txt": d.encode()})
    return files


IN_KEYS = {
    "GROBIN": {"InputEnergy": "in_E.bin", "InputDipole": "in_D.bin", "InputAlpha": "in_A.bin"},
    "SKIBIN": {"InputEnergy": "in_E.bin", "InputDipole": "in_D.bin", "InputAnharm": "in_An.bin",
               "InputOverto": "in_Ov.bin"},
    "GROASC": {"InputEnergy": "in_E.txt", "InputDipole": "in_D.txt", "InputAlpha": "in_A.txt"},
    "MITASC": {"InputEnergy": "in_E.txt", "InputDipoleX": "in_Dx.txt", "InputDipoleY": "in_Dy.txt",
               "InputDipoleZ": "in_Dz.txt"},
    "MITTXT": {"InputEnergy": "in_E.txt", "InputDipole": "in_D.txt"},
    "SPECTRON": {"InputEnergy": "in_E.txt", "InputDipole": "in_D.txt"},
}
OUT_KEYS = {
    "GROBIN": {"OutputEnergy": "out_E.bin", "OutputDipole": "out_D.bin", "OutputAlpha": "out_A.bin"},
    "SKIBIN": {"OutputEnergy": "out_E.bin", "OutputDipole": "out_D.bin", "OutputAnharm": "out_An.bin",
               "OutputOverto": "out_Ov.bin"},
    "GROASC": {"OutputEnergy": "out_E.txt", "OutputDipole": "out_D.txt", "OutputAlpha": "out_A.txt"},
    "MITASC": {"OutputEnergy": "out_E.txt", "OutputDipoleX": "out_Dx.txt", "OutputDipoleY": "out_Dy.txt",
               "OutputDipoleZ": "out_Dz.txt"},
    "MITTXT": {"OutputEnergy": "out_E.txt", "OutputDipole": "out_D.txt"},
    "SPECTRON": {"OutputEnergy": "out_E.txt", "OutputDipole": "out_D.txt"},
}

MODIFY = "Modify\nSelect 3\n3 0 2\nLabel\n1 0 2\nShift\n5.5 0 -2.25\n"

CASES = {
    "grobin_groasc": dict(i="GROBIN", o="GROASC", kw=dict(Singles=5, Doubles=0, Length=3)),
    "groasc_grobin_doubles": dict(i="GROASC", o="GROBIN", kw=dict(Singles=4, Length=3, Anharmonicity=14)),
    "grobin_full_doubles": dict(i="GROBIN", o="GROBIN", kw=dict(Singles=3, Length=2), doubles_block=True),
    "grobin_mitasc": dict(i="GROBIN", o="MITASC", kw=dict(Singles=4, Doubles=0, Length=3)),
    "mitasc_grobin": dict(i="MITASC", o="GROBIN", kw=dict(Singles=4, Length=2, Skip="Doubles")),
    "grobin_mittxt": dict(i="GROBIN", o="MITTXT", kw=dict(Singles=4, Doubles=0, Length=2)),
    "mittxt_groasc": dict(i="MITTXT", o="GROASC", kw=dict(Singles=4, Length=3)),
    "grobin_spectron": dict(i="GROBIN", o="SPECTRON", kw=dict(Singles=5, Doubles=0, Length=2)),
    "spectron_grobin": dict(i="SPECTRON", o="GROBIN", kw=dict(Singles=4, Length=2, Skip="Doubles")),
    "skibin_skibin_modify": dict(i="SKIBIN", o="SKIBIN", kw=dict(Singles=5, Length=3), modify=True),
    "grobin_skibin": dict(i="GROBIN", o="SKIBIN", kw=dict(Singles=4, Doubles=0, Length=2)),
    "grobin_modify_doubles": dict(i="GROBIN", o="GROBIN", kw=dict(Singles=5, Doubles=0, Length=2), modify=True),
    "groasc_modify_skip": dict(i="GROASC", o="GROBIN", kw=dict(Singles=5, Length=2, Skip="Doubles"), modify=True),
}


def keyword_text(case):
    lines = ["InputFormat %s" % case["i"], "OutputFormat %s" % case["o"]]
    lines += ["%s %s" % kv for kv in IN_KEYS[case["i"]].items()]
    lines += ["%s %s" % kv for kv in OUT_KEYS[case["o"]].items()]
    lines += ["%s %s" % kv for kv in case["kw"].items()]
    text = "\n".join(lines) + "\n"
    if case.get("modify"):
        text += MODIFY
    return text


def inputs(name, case):
    """{file name: bytes} of a case's inputs (keyword file included)."""
    n = case["kw"]["Singles"]
    files = write_inputs(case["i"], n, case["kw"].get("Length", 1), seed=sum(map(ord, name)),
                         doubles_block=case.get("doubles_block", False))
    files["input"] = keyword_text(case).encode()
    return files


def main():
    manifest = {}
    for name, case in CASES.items():
        work = tempfile.mkdtemp(prefix="golden_translate_")
        try:
            ins = inputs(name, case)
            for fn, data in ins.items():
                with open(os.path.join(work, fn), "wb") as f:
                    f.write(data)
            subprocess.run([REF_TRANSLATE, "input"], cwd=work, check=True, stdout=subprocess.DEVNULL)
            outs = {fn: open(os.path.join(work, fn), "rb").read() for fn in sorted(os.listdir(work)) if fn not in ins}
            enc = lambda d: json.dumps({k: base64.b64encode(v).decode() for k, v in d.items()})
            np.savez_compressed(os.path.join(HERE, "translate_%s.npz" % name),
                                inputs=np.array(enc(ins)), outputs=np.array(enc(outs)))
            manifest[name] = sorted(outs)
            print("golden translate", name, "->", {k: len(v) for k, v in outs.items()})
        finally:
            shutil.rmtree(work, ignore_errors=True)
    with open(os.path.join(HERE, "translate_cases.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
