"""The excent command line end to end on a GPU, in every fetch mode (HBM
chunk cache, streamed chunks, gathered lists, high-degree cache, zero copy),
against the FP64 oracle and against the reference binary built from source
(oracle/_ref/excent) on the same graph and flags."""
import os
import re
import subprocess

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN, read_env

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a GPU", allow_module_level=True)

import excent_b200._capi as K  # noqa: E402

CLI = K.CLI_PATH
REF_CLI = os.path.join(O.REF_DIR, "excent")
SAMPLE = os.path.join(GOLDEN, "sample.egr")


def env_args(env, measure):
    a = ["--measure", measure]
    if measure in ("katz", "all"):
        a += ["--alpha", env["ALPHA"], "--beta", env["BETA"], "--eps-katz", env["EPS_KATZ"]]
    if measure in ("ev", "all"):
        a += ["--lambda", env["LAMBDA"], "--eps-ev", env["EPS_EV"]]
    return a


def run(binary, args, tmp):
    e = dict(os.environ, HOME=str(tmp))
    r = subprocess.run([binary, *args], capture_output=True, text=True, env=e, timeout=600)
    assert r.returncode == 0, r.stderr + r.stdout
    return r.stdout


@pytest.fixture(scope="module")
def rmat14(tmp_path_factory):
    d = tmp_path_factory.mktemp("cli")
    n, idx, adj = O.rmat_graph(14, 16, 5)
    p = str(d / "r14.egr")
    O.write_egr(p, idx, adj, wide=True)
    par = O.params(n, idx, adj)
    env = {k: par[k] for k in ("LAMBDA", "ALPHA", "BETA", "EPS_PR", "EPS_KATZ", "EPS_EV")}
    return p, n, idx, adj, env


MODES = {
    "cached": ["--stream-ratio", "2", "--cache", "chunks"],
    "stream": ["--stream-ratio", "0", "--cache", "none"],
    "gather": ["--stream-ratio", "2", "--cache", "none"],
    "mixed": ["--stream-ratio", "0.3", "--cache", "none", "--chunk-medges", "0.02"],
    "hot": ["--stream-ratio", "0.3", "--cache", "hot", "--chunk-medges", "0.02", "--gpu-budget-gb", "0.0012",
            "--reserve-mb", "0"],
    "hot-start": ["--stream-ratio", "2", "--cache", "hot", "--hot-when", "both", "--hot-order", "ranges",
                  "--chunk-medges", "0.02", "--gpu-budget-gb", "0.0012", "--reserve-mb", "0"],
    "zero-copy": ["--stream-ratio", "0.3", "--cache", "none", "--zero-copy", "on", "--chunk-medges", "0.02"],
    "device-loop": ["--stream-ratio", "2", "--cache", "chunks", "--device-loop"],
    "nodedup": ["--stream-ratio", "2", "--cache", "none", "--dedup", "off", "--chunk-medges", "0.05"],
    "host-cache": ["--stream-ratio", "2", "--host-cache", "pinned", "--chunk-medges", "0.02", "--gpu-budget-gb", "0.0004",
                   "--reserve-mb", "0"],
}


@pytest.mark.parametrize("mode", sorted(MODES))
@pytest.mark.parametrize("measure", ["pr", "all"])
def test_cli_modes_vs_oracle(rmat14, tmp_path, mode, measure):
    p, n, idx, adj, env = rmat14
    out = run(CLI, [p, *env_args(env, measure), *MODES[mode], "--dump", str(tmp_path / "o"), "--count-pushes"],
              tmp_path)
    assert re.search(r"^passes \d+  measure", out, re.M), out
    if mode in ("stream", "mixed", "zero-copy"):
        assert re.search(r"stream [1-9]", out), out
    if mode in ("gather", "mixed", "nodedup"):
        assert re.search(r"gather [1-9]", out), out
    if mode == "host-cache":
        assert re.search(r"host cache: pinned, [0-9.]+ GB \([1-9]\d* chunks past the GPU cache\)", out), out
        assert re.search(r"gather [0-9.]*[1-9][0-9.]* GB", out), out
    if mode.startswith("hot"):
        assert "GPU degree cache:" in out
        assert re.search(r"cached high-degree pending [1-9]", out), out
    names = ["pr", "katz", "ev"] if measure == "all" else ["pr"]
    for k in names:
        x = np.fromfile(str(tmp_path / f"o.{k}.bin"), dtype=np.float32)
        ref = O.reference_solution(n, idx, adj, k, alpha=float(env["ALPHA"]))
        c = O.compare(k, ref, x)
        assert c["l1_rel"] < 0.05 and c["top100"] >= 95, (mode, k, c)


def test_cli_sample_matches_reference_binary(tmp_path):
    if not os.path.exists(REF_CLI):
        pytest.skip("reference binary not built")
    env = read_env(os.path.join(GOLDEN, "sample.env"))
    for measure in ("pr", "all"):
        args = [SAMPLE, *env_args(env, measure), "--stream-ratio", "2"]
        ours = run(CLI, args + ["--dump", str(tmp_path / "a")], tmp_path)
        ref = run(REF_CLI, args + ["--dump", str(tmp_path / "b")], tmp_path)
        # same line structure (first words of every line)
        num = r"[-+]?\d+(?:\.\d+)?(?:e[-+]?\d+)?"
        heads = lambda s: [re.sub(num, "#", l)[:25] for l in s.splitlines() if not l.startswith("throughput")]  # noqa: E731
        h1, h2 = heads(ours), heads(ref)
        assert h1[:4] == h2[:4]
        assert [l for l in h1 if l.startswith("passes")] and [l for l in h2 if l.startswith("passes")]
        names = ["pr", "katz", "ev"] if measure == "all" else ["pr"]
        for k in names:
            a = np.fromfile(str(tmp_path / f"a.{k}.bin"), dtype=np.float32)
            b = np.fromfile(str(tmp_path / f"b.{k}.bin"), dtype=np.float32)
            ref_x = O.reference_solution(len(a), *O.read_egr(SAMPLE)[1:], k, alpha=float(env["ALPHA"]))
            ca, cb = O.compare(k, ref_x, a), O.compare(k, ref_x, b)
            assert ca["l1_rel"] <= cb["l1_rel"] * 1.05, (k, ca, cb)


@pytest.fixture(scope="module")
def rmat16_cfg(tmp_path_factory):
    """The reference's CPU-runnable configuration: R-MAT scale 16, edge factor 16, seed 1,
    symmetric, written as wide EGR, with its given constants (tools/excent_params.cu rules)."""
    d = tmp_path_factory.mktemp("cfg1")
    n, idx, adj = O.rmat_graph(16, 16, 1)
    p = str(d / "r16.egr")
    O.write_egr(p, idx, adj, wide=True)
    par = O.params(n, idx, adj)
    env = {k: par[k] for k in ("LAMBDA", "ALPHA", "BETA", "EPS_PR", "EPS_KATZ", "EPS_EV")}
    return p, n, idx, adj, env


@pytest.mark.parametrize("measure", ["pr", "all"])
@pytest.mark.parametrize("mode", ["host", "device-loop"])
def test_error_no_looser_than_reference_binary_rmat16(rmat16_cfg, tmp_path, measure, mode):
    """Error against the FP64 oracle (L1 relative, max per-vertex, top-1000 overlap) of this
    repo's CLI against the reference binary's on the same R-MAT scale-16 file and flags.
    Both add FP32 residuals with atomics in a run-dependent order (the reference's own Katz
    L1 moved by 9 % between two runs here), so L1 and the top-1000 overlap are medians (three
    runs of ours, five of the reference's), with an allowance of 5 % of L1 and 5 of the top
    1000. The max per-vertex error of both engines sits at one vertex, the top hub (vertex 0,
    degree 6274, first in every measure); its size and sign follow the push order, and the
    reference's own eigenvector error there spread from under 1.05e-5 to 4.3e-5 over six
    identical runs. So that figure is held to 1.25 x the reference's largest of its five runs."""
    if not os.path.exists(REF_CLI):
        pytest.skip("reference binary not built")
    p, n, idx, adj, env = rmat16_cfg
    args = [p, *env_args(env, measure), "--stream-ratio", "2", "--cache", "chunks"]
    kinds = ["pr", "katz", "ev"] if measure == "all" else ["pr"]
    refs = {k: O.reference_solution(n, idx, adj, k, alpha=float(env["ALPHA"])) for k in kinds}
    med = {}
    for side, binary, extra in (("ours", CLI, ["--device-loop"] if mode == "device-loop" else []),
                                ("reference", REF_CLI, [])):
        runs = {k: [] for k in kinds}
        for rep in range(3 if side == "ours" else 5):
            out = str(tmp_path / f"{side}{rep}")
            run(binary, args + extra + ["--dump", out], tmp_path)
            for k in kinds:
                runs[k].append(O.compare(k, refs[k], np.fromfile(f"{out}.{k}.bin", dtype=np.float32)))
        med[side] = {k: {q: float(np.median([r[q] for r in runs[k]])) for q in ("l1_rel", "max_abs", "top1000")}
                     for k in kinds}
        for k in kinds:
            med[side][k]["max_abs_worst"] = float(max(r["max_abs"] for r in runs[k]))
    for k in kinds:
        a, b = med["ours"][k], med["reference"][k]
        print(k, "ours", a, "reference", b)
        assert a["l1_rel"] <= 1.05 * b["l1_rel"] + 1e-7, (k, a, b)
        assert a["max_abs"] <= 1.25 * b["max_abs_worst"] + 1e-7, (k, a, b)
        assert a["top1000"] >= b["top1000"] - 5, (k, a, b)


def test_cli_trace_and_hot_rank_roundtrip(rmat14, tmp_path):
    """--trace-pending writes uint16 pass counts; they drive --hot-rank."""
    p, n, idx, adj, env = rmat14
    tr = str(tmp_path / "trace.u16")
    run(CLI, [p, "--measure", "pr", "--stream-ratio", "2", "--trace-pending", tr], tmp_path)
    t = np.fromfile(tr, dtype=np.uint16)
    assert len(t) == n and t.max() > 0
    out = run(CLI, [p, "--measure", "pr", "--stream-ratio", "0.3", "--cache", "hot", "--hot-rank", tr,
                    "--chunk-medges", "0.02", "--gpu-budget-gb", "0.0012", "--reserve-mb", "0",
                    "--dump", str(tmp_path / "h")], tmp_path)
    assert "GPU cache ranked by passes pending" in out
    x = np.fromfile(str(tmp_path / "h.pr.bin"), dtype=np.float32)
    ref = O.reference_solution(n, idx, adj, "pr")
    assert O.compare("pr", ref, x)["l1_rel"] < 0.05


def test_cli_tau_calibration_and_cache_file(rmat14, tmp_path):
    p, *_ = rmat14
    out = run(CLI, [p, "--measure", "pr", "--cache", "none"], tmp_path)
    m = re.search(r"fetch rule: tau = ([0-9.]+) \(stream", out)
    assert m, out
    files = list((tmp_path / ".cache" / "excent").glob("*.tau"))
    assert len(files) == 1
    tau, t = open(files[0]).read().split()
    assert abs(float(tau) - float(m.group(1))) < 1e-3
    out2 = run(CLI, [p, "--measure", "pr", "--cache", "none"], tmp_path)
    assert "measured earlier on this machine" in out2


def test_params_tool_reproduces_the_sample_env(tmp_path):
    """bin/excent_params writes the sample graph's given constants: the
    reference's only known answer (datasets/sample/sample.env), and the
    reference's own tool on the same file when it was built."""
    tool = os.path.join(os.path.dirname(CLI), "excent_params")
    out = run(tool, [SAMPLE, str(tmp_path / "s.env")], tmp_path)
    assert re.search(r"^lambda1 = [0-9.]+ after \d+ power iterations", out, re.M), out
    got = read_env(str(tmp_path / "s.env"))
    want = read_env(os.path.join(GOLDEN, "sample.env"))
    assert abs(float(got["LAMBDA"]) - float(want["LAMBDA"])) <= 1e-9 * float(want["LAMBDA"])
    for k in ("ALPHA", "BETA", "EPS_PR", "EPS_KATZ", "EPS_EV"):
        assert got[k] == want[k], (k, got[k], want[k])
    ref_tool = os.path.join(O.REF_DIR, "excent_params")
    if os.path.exists(ref_tool):
        run(ref_tool, [SAMPLE, str(tmp_path / "r.env")], tmp_path)
        ref = read_env(str(tmp_path / "r.env"))
        for k in ("ALPHA", "BETA", "EPS_PR", "EPS_KATZ", "EPS_EV"):
            assert got[k] == ref[k], (k, got[k], ref[k])



@pytest.mark.parametrize("measure", ["pr", "katz", "ev"])
def test_reference_tool_solve_matches_the_golden_fp64(tmp_path, measure):
    """bin/excent_reference's FP64 solve on the GPU against the golden FP64
    solution the reference's own tool wrote for the sample graph."""
    env = read_env(os.path.join(GOLDEN, "sample.env"))
    tool = os.path.join(os.path.dirname(CLI), "excent_reference")
    extra = ["--alpha", env["ALPHA"]] if measure == "katz" else []
    out = run(tool, [SAMPLE, measure, str(tmp_path / "r.bin"), *extra], tmp_path)
    assert out.startswith(f"reference {measure}:"), out
    got = np.fromfile(str(tmp_path / "r.bin"), dtype=np.float64)
    want = np.fromfile(os.path.join(GOLDEN, f"sample_ref_{measure}.f64"), dtype=np.float64)
    assert got.shape == want.shape
    assert np.abs(got - want).max() <= 1e-8 * np.abs(want).max()
