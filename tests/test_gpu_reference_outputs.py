"""The drop-in against the outputs the reference ships with its examples (summarised into
tests/golden/ by tests/golden/make_golden.py):

* examples/example_dadi/run_980_2.out -- per-bin mean and standard deviation of the normalised SFS
  (n = 1001, population 1) over 50 replicates of the two-population model of
  examples/example_dadi/run.cu:23-117 at L = 2e8, made by the reference on a GTX 980.  The drop-in runs
  the same model with the same replicate seeds (tests/cpp/scenarios.h, scenario_dadi); the model
  starts at mutation-selection equilibrium with gamma = -4, where the reference itself is not
  reproducible run to run, so the comparison is statistical: per bin, z = (mean_mine - mean_ref) /
  sqrt(sd_mine^2 / 50 + sd_ref^2 / 50).
* examples/example_compilation/bfile.dat -- the seed-pinned dump of examples/example_compilation
  (2 inbred populations, 20,000-generation blank-start burn-in, then 1,000 generations from it),
  written on a GTX 780M / 980 with an older CUDA.  The drop-in is bit-exact against the reference
  built here and run on this GPU (its operator<< text is byte-identical); whether the old dump itself
  reproduces is recorded by the test (fast-math code generation differs across GPU generations), and
  the dump is checked statistically against replicates of the drop-in with other seeds.
"""
from __future__ import annotations

import hashlib
import json
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from gfdump import Dump

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"


def read_dadi_table(path: Path, n: int):
    mean, sd = np.zeros(n), np.zeros(n)
    for ln in path.read_text().splitlines():
        f = ln.split("\t")
        if len(f) == 3 and f[0].isdigit():
            i = int(f[0])
            mean[i], sd[i] = float(f[1]), float(f[2])
    return mean[1:], sd[1:]


def test_dadi_model_matches_reference_table(gofish_driver, tmp_path):
    ref = json.loads((GOLDEN / "dadi_reference.json").read_text())["run_980_2.out"]
    bins = np.array(ref["bins"])
    assert bins.shape == (1000, 3) and ref["num_sites"] == 2e8
    reps = 50
    out = tmp_path / "dadi.txt"
    subprocess.run([str(gofish_driver), "dadi", str(out), f"reps={reps}", "L=2e8", "sfs_n=1001"], check=True,
                   capture_output=True)
    mean, sd = read_dadi_table(out, 1001)
    assert np.all(sd > 0)
    z = (mean - bins[:, 1]) / np.sqrt(sd ** 2 / reps + bins[:, 2] ** 2 / reps)
    # neighbouring bins of a projected SFS are strongly correlated, so the checks are on the
    # distribution of z over bins rather than a sum of squares.  Both tables use the same replicate
    # seeds, and the runs differ only where the reference's equilibrium start sums floats in another
    # order (and in the GPU's fast-math code), so the two sets of replicates are strongly correlated and
    # |z| is typically far below the 0.67 median of independent samples; the bounds are one-sided.
    print(f"dadi table: median |z| {np.median(np.abs(z)):.3f}, max |z| {np.abs(z).max():.3f}")
    assert np.median(np.abs(z)) < 1.1, np.median(np.abs(z))
    assert np.abs(z).max() < 5.0, (np.argmax(np.abs(z)) + 1, np.abs(z).max())
    assert abs(z.mean()) < 1.0, z.mean()
    # the normalised SFS sums to the reference's within its own replicate spread
    assert abs(mean.sum() - bins[:, 1].sum()) < 0.01


def compilation_stats(d: Dump) -> dict:
    """Per-sample mutation counts and, per sample and population, the numbers of lost and fixed
    mutations and the mean allele count of the segregating ones."""
    out = {}
    for s, smp in enumerate(d.samples):
        out[f"M{s}"] = smp["M"]
        for p in range(d.P):
            nc = smp["Nc"][p]
            c = np.rint(smp["freq"][p].astype(np.float64) * nc)
            seg = c[(c > 0) & (c < nc)]
            out[f"lost{s}{p}"] = int((c == 0).sum())
            out[f"fixed{s}{p}"] = int((c == nc).sum())
            out[f"mean{s}{p}"] = float(seg.mean()) if seg.size else 0.0
    return out


def golden_compilation_stats(g: dict) -> dict:
    out = {}
    for s, M in enumerate(g["num_mutations"]):
        out[f"M{s}"] = M
        for p in range(g["num_populations"]):
            h = np.array(g["count_histograms"][f"{s},{p}"], dtype=np.float64)
            nc = len(h) - 1
            k = np.arange(nc + 1)
            out[f"lost{s}{p}"] = int(h[0])
            out[f"fixed{s}{p}"] = int(h[nc])
            seg = h[1:nc]
            out[f"mean{s}{p}"] = float((seg * k[1:nc]).sum() / seg.sum())
    return out


def test_example_compilation_against_reference_and_its_committed_dump(gofish_driver, ref_driver, tmp_path):
    g = json.loads((GOLDEN / "example_compilation.json").read_text())
    # 1. the reference's own example, run by both libraries on this GPU: bit for bit, and the same text
    subprocess.run([str(gofish_driver), "compilation", str(tmp_path / "mine.bin"), f"text={tmp_path / 'mine.txt'}"],
                   check=True, capture_output=True)
    mine = Dump(tmp_path / "mine.bin")
    subprocess.run([str(ref_driver), "sim", "compilation", str(tmp_path / "ref.bin"), f"text={tmp_path / 'ref.txt'}"],
                   check=True, capture_output=True)
    ref = Dump(tmp_path / "ref.bin")
    assert [s["generation"] for s in ref.samples] == g["generations"]
    from test_gpu_parity import assert_dumps_equal
    assert_dumps_equal(mine, ref)
    text = (tmp_path / "mine.txt").read_text()
    assert text == (tmp_path / "ref.txt").read_text()
    # 2. the committed dump of the same program: exact reproduction is recorded, not required
    rows = re.findall(r"^\((-?\d+),(-?\d+),(-?\d+),(-?\d+)\):", text, flags=re.M)
    sha = hashlib.sha256("".join(f"{a},{b},{c},{d}\n" for a, b, c, d in rows).encode()).hexdigest()
    exact = sha == g["ids_sha256"] and [s["M"] for s in mine.samples] == g["num_mutations"]
    print(f"committed bfile.dat reproduced exactly on this GPU: {exact}")
    # 3. statistically: the committed dump's summary against replicates of the drop-in with other seeds
    stats = []
    for r in range(10):
        out = tmp_path / f"rep{r}.bin"
        subprocess.run([str(gofish_driver), "compilation", str(out), f"seed1={0x1000 + 7 * r}",
                        f"seed2={0x2000 + 13 * r}"], check=True, capture_output=True)
        stats.append(compilation_stats(Dump(out)))
    want = golden_compilation_stats(g)
    for key, v in want.items():
        xs = np.array([st[key] for st in stats], dtype=np.float64)
        sd = xs.std(ddof=1)
        z = (v - xs.mean()) / (sd * np.sqrt(1 + 1 / len(xs)) if sd > 0 else 1.0)
        assert abs(z) < 4.5, f"{key}: committed {v}, drop-in {xs.mean():.1f} +- {sd:.1f} (z {z:.1f})"
