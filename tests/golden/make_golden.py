"""Regenerate the committed golden fixtures of this directory.

    python tests/golden/make_golden.py            # CPU part (needs the reference checkout)
    python tests/golden/make_golden.py --gpu-ref [--out DIR]  # also run the reference's own CUDA tools

CPU part: copies the reference's sample graph and its given constants
(datasets/sample/sample.egr, sample.env of SPADE-IITJ/ExCent) and records
their SHA-256. --gpu-ref (on a machine with a GPU, after `make -C oracle ref`)
runs the reference's FP64 oracle binary (tools/centrality_reference.cu) and
its engine binary (src/excent.cu) built from source into oracle/_ref/, and
stores their outputs: sample_ref_<measure>.f64 (FP64 oracle vectors) and
sample_excent_<measure>.f32 (the reference engine's result dumps).
"""
import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def reference_root():
    """The reference checkout: $EXCENT_REFERENCE, else oracle/Makefile's REF default."""
    r = os.environ.get("EXCENT_REFERENCE")
    if r:
        return r
    out = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "print-ref"], capture_output=True,
                         text=True)
    return out.stdout.strip()


REF = os.path.join(reference_root(), "datasets", "sample")
REF_BIN = os.path.join(ROOT, "oracle", "_ref")


def sha(p):
    return hashlib.sha256(open(p, "rb").read()).hexdigest()


def env_args(env, measure):
    a = ["--measure", measure]
    if measure in ("katz", "all"):
        a += ["--alpha", env["ALPHA"], "--beta", env["BETA"], "--eps-katz", env["EPS_KATZ"]]
    if measure in ("ev", "all"):
        a += ["--lambda", env["LAMBDA"], "--eps-ev", env["EPS_EV"]]
    if measure == "all":
        a += ["--eps-pr", env["EPS_PR"]]
    return a


def read_env(p):
    env = {}
    for line in open(p):
        line = line.strip()
        if line and not line.startswith("#") and "=" in line:
            k, v = line.split("=", 1)
            env[k] = v
    return env


# A small MatrixMarket file with what real files hold: comments, a weight
# column, repeated entries, self-loops, lists out of order, an empty vertex and
# an entry whose source is past n (the reference converter skips it).
EDGE_CASES_MTX = """%%MatrixMarket matrix coordinate real general
% comment line
7 6 14
3 1 0.5
1 2 1.0
1 2 2.0
2 2 1
5 1
9 3
3 7
2 1 4e-1
1 6
6 1
1 1
3 2
7 3
4 5
"""


def converter_goldens(meta):
    """The reference's own converter (tools/efficient_converter.py, run here from the reference
    checkout) on the sample's .mtx and on EDGE_CASES_MTX: golden EGR outputs."""
    conv = os.path.join(os.path.dirname(os.path.dirname(REF)), "tools", "efficient_converter.py")
    if not os.path.exists(conv):
        return
    edge = os.path.join(HERE, "edge_cases.mtx")
    with open(edge, "w") as f:
        f.write(EDGE_CASES_MTX)
    # the sample's .mtx converts to exactly the sample's .egr: only its digest is kept
    tmp = os.path.join(tempfile.mkdtemp(), "sample_converted.egr")
    for src, dst in (("sample.mtx", tmp), ("edge_cases.mtx", os.path.join(HERE, "edge_cases_converted.egr"))):
        subprocess.run([sys.executable, conv, os.path.join(HERE, src), dst], capture_output=True, text=True,
                       check=True)
        meta[f"efficient_converter {src}"] = sha(dst)
    meta["edge_cases.mtx"] = sha(edge)
    # the reference's egr_info line for the sample (oracle/_ref/egr_info, built from tools/egr_info.cpp)
    info = os.path.join(REF_BIN, "egr_info")
    if os.path.exists(info):
        r = subprocess.run([info, os.path.join(HERE, "sample.egr")], capture_output=True, text=True, check=True)
        meta["egr_info sample.egr"] = r.stdout.strip()


def main():
    out_dir = HERE
    if "--out" in sys.argv:
        out_dir = sys.argv[sys.argv.index("--out") + 1]
        os.makedirs(out_dir, exist_ok=True)
    meta_p = os.path.join(out_dir, "golden.json")
    meta = json.load(open(meta_p)) if os.path.exists(meta_p) else {}
    if os.path.isdir(REF):
        for f in ("sample.egr", "sample.env", "sample.mtx"):
            shutil.copyfile(os.path.join(REF, f), os.path.join(HERE, f))
            meta[f] = sha(os.path.join(HERE, f))
        converter_goldens(meta)
    if "--gpu-ref" in sys.argv:
        egr = os.path.join(HERE, "sample.egr")
        env = read_env(os.path.join(HERE, "sample.env"))
        for m in ("pr", "katz", "ev"):
            out = os.path.join(out_dir, f"sample_ref_{m}.f64")
            cmd = [os.path.join(REF_BIN, "centrality_reference"), egr, m, out]
            if m == "katz":
                cmd += ["--alpha", env["ALPHA"], "--beta", env["BETA"]]
            r = subprocess.run(cmd, capture_output=True, text=True, check=True)
            meta[f"centrality_reference {m}"] = r.stdout.strip()
        tmp = os.path.join(out_dir, "_tmp_dump")
        for m in ("pr", "katz", "ev", "all"):
            cmd = [os.path.join(REF_BIN, "excent"), egr, *env_args(env, m), "--stream-ratio", "2",
                   "--dump", tmp]
            r = subprocess.run(cmd, capture_output=True, text=True, check=True,
                               env=dict(os.environ, HOME=tempfile.mkdtemp()))
            meta[f"excent {m}"] = [l for l in r.stdout.splitlines() if l.startswith("passes")]
            names = ("pr", "katz", "ev") if m == "all" else (m,)
            for k in names:
                dst = os.path.join(out_dir, f"sample_excent_{m}_{k}.f32")
                os.replace(f"{tmp}.{k}.bin", dst)
    json.dump(meta, open(meta_p, "w"), indent=1, sort_keys=True)
    print(json.dumps(meta, indent=1))


if __name__ == "__main__":
    main()
