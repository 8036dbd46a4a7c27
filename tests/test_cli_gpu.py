"""The drop-in program bin/mhd2d_glm_gpu on the GPU, against the reference's
own outputs (src/mhd/mhd2d_glm_gpu.cu:353-648 is the program it replaces):

  * the stdout lines the reference's scripts grep (run_baseline_perf_gpu.sh
    :34-36: "Done. Steps:", "Time loop wall time = ... Mcell-steps/s",
    "HLLD->HLL fallbacks = ...") are present and parse, and -- wall time
    apart -- equal the reference CPU program's numbers recorded in
    tests/golden/runs.json (exact build, PMHD_EXACT=1);
  * the .dat file it writes under OUTDIR has the reference's file name and
    data-line md5;
  * the program name selects the precision (_fp64 / _fp32 / _mixed);
  * an OUTDIR that cannot be created or written gives exit code 5 after the
    run (the reference's :604-609);
  * where the reference's own GPU program is built (oracle/_ref), its stdout
    lines parse with the same patterns, field for field.
"""
import hashlib
import json
import os
import re
import subprocess

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BIN = os.path.join(ROOT, "precision-study_b200", "bin", "mhd2d_glm_gpu")
REF_GPU = os.path.join(ROOT, "oracle", "_ref", "mhd2d_glm_gpu_fp64")

# The greps of the reference's perf scripts, plus the fields compared.
PATTERNS = {
    "done": r"Done\. Steps: (\d+), final t = (\S+)",
    "ch": r"c_h\(last\) = (\S+), alpha = (\S+)",
    "wall": r"Time loop wall time = ([0-9.]+) s \(([0-9.]+|inf) Mcell-steps/s\)",
    "evals": r"HLLD flux evaluations = (\d+) \(x=(\d+), y=(\d+)\)",
    "fallbacks": r"HLLD->HLL fallbacks = (\d+) \(degenerate=(\d+), nonphysical=(\d+)\), fraction = (\S+)",
    "divb": r"divB L1 = (\S+), divB Linf = (\S+), psi Linf = (\S+)",
    "saved": r"Saved: (\S+)",
}


def parse(stdout):
    out = {}
    for k, pat in PATTERNS.items():
        m = re.search(pat, stdout)
        out[k] = m.groups() if m else None
    return out


def md5_data(path):
    h = hashlib.md5()
    with open(path, "rb") as f:
        for line in f:
            if not line.startswith(b"#"):
                h.update(line)
    return h.hexdigest()


def golden(prec, nx, ny, t_end, order="muscl", solver="hlld"):
    for r in json.load(open(os.path.join(HERE, "golden", "runs.json")))["runs"]:
        if (r["precision"], r["nx"], r["ny"], r["t_end"], r["order"], r["solver"]) == (prec, nx, ny, t_end, order,
                                                                                      solver):
            return r
    raise KeyError((prec, nx, ny, t_end))


def run_cli(prog, args, outdir, exact=True):
    env = dict(os.environ, OUTDIR=str(outdir))
    if exact:
        env["PMHD_EXACT"] = "1"
    return subprocess.run([prog] + [str(a) for a in args], capture_output=True, text=True, env=env, timeout=300)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_cli_lines_and_dat_match_the_reference(pmhd_lib, tmp_path, prec):
    args = [64, 64, 0.2, 0.25, "muscl", "hlld", 0.18]
    r = run_cli(BIN + "_" + prec, args, tmp_path)
    assert r.returncode == 0, r.stderr
    p = parse(r.stdout)
    g = golden(prec, 64, 64, 0.2)
    assert all(p[k] is not None for k in PATTERNS), p
    assert int(p["done"][0]) == g["steps"]
    assert float(p["ch"][0]) == g["ch_last_printed"]
    assert (int(p["evals"][1]), int(p["evals"][2])) == (g["x_evals"], g["y_evals"])
    assert (int(p["fallbacks"][1]), int(p["fallbacks"][2])) == (g["degenerate"], g["nonphysical"])
    assert int(p["fallbacks"][0]) == g["degenerate"] + g["nonphysical"]
    assert float(p["wall"][0]) >= 0.0
    f = f"orszag_tang_glm_muscl_hlld_{prec}_N64x64.dat"
    assert p["saved"][0] == os.path.join(str(tmp_path), f)
    assert md5_data(os.path.join(str(tmp_path), f)) == g["md5"]
    assert f"Precision: {64 if prec == 'fp64' else 32} bit ({prec})" in r.stdout


def test_cli_mixed_program_name_selects_mixed(pmhd_lib, tmp_path):
    r = run_cli(BIN + "_mixed", [48, 32, 0.05, 0.25, "muscl", "hlld", 0.18], tmp_path, exact=False)
    assert r.returncode == 0, r.stderr
    assert "(mixed)" in r.stdout
    assert os.path.exists(os.path.join(str(tmp_path), "orszag_tang_glm_muscl_hlld_mixed_N48x32.dat"))
    p = parse(r.stdout)
    assert p["done"] is not None and p["fallbacks"] is not None


def test_cli_unwritable_outdir_exits_5(pmhd_lib, tmp_path):
    bad = "/dev/null/pmhd_cannot_create"
    r = run_cli(BIN, [32, 32, 0.02, 0.25, "muscl", "hlld", 0.18], bad)
    assert r.returncode == 5, (r.returncode, r.stderr)
    assert "failed to open output file" in r.stderr
    assert parse(r.stdout)["done"] is not None  # the run itself completed first


@pytest.mark.skipif(not os.path.exists(REF_GPU), reason="reference GPU program not built (oracle/_ref)")
def test_cli_lines_parse_like_the_reference_gpu_program(pmhd_lib, tmp_path):
    args = [64, 64, 0.05, 0.25, "muscl", "hlld", 0.18]
    ours = run_cli(BIN + "_fp64", args, tmp_path / "ours", exact=False)
    ref = run_cli(REF_GPU, args, tmp_path / "ref", exact=False)
    assert ours.returncode == 0 and ref.returncode == 0, (ours.stderr, ref.stderr)
    po, pr = parse(ours.stdout), parse(ref.stdout)
    for k in PATTERNS:
        assert (po[k] is None) == (pr[k] is None), k
    assert po["done"][0] == pr["done"][0]  # same step count
    assert po["evals"] == pr["evals"]
    assert os.path.basename(po["saved"][0]) == os.path.basename(pr["saved"][0])


EULER_BIN = os.path.join(ROOT, "precision-study_b200", "bin", "euler2d_gpu")


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_euler_cli_writes_the_reference_program_data(pmhd_lib, tmp_path, prec):
    """The shock-bubble drop-in (bin/euler2d_gpu_<prec>, replacing
    src/euler/euler2d_cuda.cu): its progress and summary lines, and -- exact
    kernels -- the data lines of gpu_shock_bubble.dat equal those of the
    reference CPU program's cpu_shock_bubble.dat (tests/golden/euler_runs.json)."""
    gold = next(r for r in json.load(open(os.path.join(HERE, "golden", "euler_runs.json")))["shock_bubble"]
                if r["precision"] == prec)
    env = dict(os.environ, OUTDIR=str(tmp_path), PMHD_EXACT="1")
    r = subprocess.run([EULER_BIN + "_" + prec], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stderr
    assert int(re.search(r"Done\. Steps: (\d+)", r.stdout).group(1)) == gold["steps"]
    assert re.search(r"Execution Time: [0-9.]+ ms \([0-9.]+ s\)", r.stdout)
    assert len(re.findall(r"^Step \d+00: t = \S+$", r.stdout, re.M)) == gold["steps"] // 100
    path = os.path.join(str(tmp_path), "gpu_shock_bubble.dat")
    assert f"Saved {path}" in r.stdout
    with open(path, "rb") as f:
        assert f.readline().startswith(b"# Time = ")
    assert md5_data(path) == gold["md5_data"]


RIEMANN_BIN = os.path.join(ROOT, "precision-study_b200", "bin", "riemann2d_gpu")


@pytest.mark.parametrize("n,config,prec", [(64, 3, "fp64"), (64, 6, "fp32"), (100, 3, "fp64")])
def test_riemann_cli_writes_the_reference_program_output(pmhd_lib, tmp_path, n, config, prec):
    """The 2D Riemann drop-in (bin/riemann2d_gpu_<prec> N config, replacing
    src/euler/riemann2d_gpu.cu): step count, file name and -- exact kernels
    -- the .dat file equal the reference CPU program's
    (tests/golden/euler_runs.json)."""
    gold = next(r for r in json.load(open(os.path.join(HERE, "golden", "euler_runs.json")))["runs2d"]
                if (r["n"], r["config"], r["solver"], r["precision"]) == (n, config, "hllc", prec))
    env = dict(os.environ, OUTDIR=str(tmp_path), PMHD_EXACT="1")
    r = subprocess.run([RIEMANN_BIN + "_" + prec, str(n), str(config)], capture_output=True, text=True, env=env,
                       timeout=120)
    assert r.returncode == 0, r.stderr
    assert re.search(r"Done\. Steps: (\d+)   Wall: \S+ s", r.stdout).group(1) == str(gold["steps"])
    name = {3: "cfg3_4shocks", 6: "cfg6_4contacts", 12: "cfg12_2S2C"}[config]
    path = os.path.join(str(tmp_path), f"riemann2d_{name}_hllc_{n}.dat")
    assert f"Saved: {path}" in r.stdout
    with open(path, "rb") as f:
        assert hashlib.md5(f.read()).hexdigest() == gold["md5"]


RIEMANN1D_BIN = os.path.join(ROOT, "precision-study_b200", "bin", "riemann1d_gpu")


@pytest.mark.parametrize("test,solver,prec", [(1, "hllc", "fp64"), (5, "hll", "fp64"), (3, "hllc", "fp32")])
def test_riemann1d_cli_writes_the_reference_program_output(pmhd_lib, tmp_path, test, solver, prec):
    """The 1D Riemann drop-in (bin/riemann1d_gpu_<prec> N test solver,
    replacing src/euler/riemann1d_gpu.cu): step count, file name and -- exact
    kernels -- the .dat file equal the reference CPU program's
    (tests/golden/euler_runs.json)."""
    gold = next(r for r in json.load(open(os.path.join(HERE, "golden", "euler_runs.json")))["runs1d"]
                if (r["n"], r["test"], r["solver"], r["precision"]) == (200, test, solver, prec))
    env = dict(os.environ, OUTDIR=str(tmp_path), PMHD_EXACT="1")
    r = subprocess.run([RIEMANN1D_BIN + "_" + prec, "200", str(test), solver], capture_output=True, text=True,
                       env=env, timeout=120)
    assert r.returncode == 0, r.stderr
    assert int(re.search(r"Done\. Steps: (\d+)", r.stdout).group(1)) == gold["steps"]
    path = os.path.join(str(tmp_path), f"toro{test}_{solver}_{prec}_200.dat")
    assert f"Saved: {path}" in r.stdout
    with open(path, "rb") as f:
        assert hashlib.md5(f.read()).hexdigest() == gold["md5"]
