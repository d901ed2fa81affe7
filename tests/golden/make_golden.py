"""Generate the golden fixtures in this directory from the reference (run in the build container,
where the reference checkout is available; the fixtures are committed, the reference is not needed
afterwards).

  ref_hostrng.bin                 Philox4x32-10 blocks and host-side Poisson draws (the new-mutation
                                  count path) computed by the reference's own RNG::Philox /
                                  RNG::ApproxRandPois1 host code (oracle/_ref/ref_driver hostrng).
  example_compilation.json        Summary of the reference's committed dump
                                  examples/example_compilation/bfile.dat (2 populations, 2 time
                                  samples): mutation counts, per-sample/population allele-count
                                  histograms, a hash of the mutation-ID list and the first rows.
  dadi_reference.json             Per-bin mean and SD of the normalised SFS (n = 1001) over 50
                                  replicates from the reference's committed runs
                                  examples/example_dadi/run_980.out (L = 2e9) and run_980_2.out
                                  (L = 2e8), and the diffusion expectation dadi_example.out.

Usage:  python tests/golden/make_golden.py [--reference <reference checkout>]
        (default: $REF, else a checkout named `reference` beside this repository)
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import re
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]


def hostrng(ref_root: Path) -> None:
    drv = ROOT / "oracle" / "_ref" / "ref_driver"
    if not drv.exists():
        subprocess.run(["bash", str(ROOT / "oracle" / "build_ref.sh")], check=True, env={"REF": str(ref_root),
                                                                                           "PATH": "/usr/bin:/bin"})
    subprocess.run([str(drv), "hostrng", str(HERE / "ref_hostrng.bin")], check=True)


def example_compilation(ref_root: Path) -> None:
    path = ref_root / "examples" / "example_compilation" / "bfile.dat"
    lines = path.read_text().splitlines()
    kv = {}
    rows = []
    in_rows = False
    for ln in lines:
        if ln.startswith("mutation ID"):
            in_rows = True
            continue
        if in_rows:
            if not ln.strip():
                continue
            m = re.match(r"\((-?\d+),(-?\d+),(-?\d+),(-?\d+)\):\t(.*)", ln)
            ids = tuple(int(m.group(i)) for i in range(1, 5))
            freqs = [float(x) for x in m.group(5).split("\t")]
            rows.append((ids, freqs))
        elif "\t" in ln:
            k, *v = ln.split("\t")
            kv[k.rstrip(":")] = v
    P = int(kv["num_populations"][0])
    S = len([x for x in kv["time sample"] if x != ""])
    Nc = [int(x) for x in kv["effective population size (chromosomes)"]]
    gens = [int(x) for x in kv["generation"] if x != ""]
    nmut = [int(x) for x in kv["number of mutations reported"] if x != ""]
    hist = {}
    for s in range(S):
        for p in range(P):
            nc = Nc[s * P + p]
            h = [0] * (nc + 1)
            for (ids, fr) in rows[: nmut[s]]:
                h[int(round(fr[s * P + p] * nc))] += 1
            hist[f"{s},{p}"] = h
    id_text = "".join(f"{a},{b},{c},{d}\n" for (a, b, c, d), _ in rows)
    out = {
        "source": "examples/example_compilation/bfile.dat",
        "seed1": int(kv["seed1"][0]), "seed2": int(kv["seed2"][0]),
        "num_sites": float(kv["num_sites"][0]), "num_populations": P, "compact_interval": int(kv["compact_interval"][0]),
        "generations": gens, "num_mutations": nmut, "Nchrom_e": Nc,
        "count_histograms": hist,
        "ids_sha256": hashlib.sha256(id_text.encode()).hexdigest(),
        "first_rows": [[list(ids), [int(round(f * 1000)) for f in fr]] for ids, fr in rows[:25]],
    }
    (HERE / "example_compilation.json").write_text(json.dumps(out))


def dadi(ref_root: Path) -> None:
    out = {}
    for name, L in (("run_980.out", 2e9), ("run_980_2.out", 2e8)):
        txt = (ref_root / "examples" / "example_dadi" / name).read_text().splitlines()
        table = []
        for ln in txt:
            f = ln.split("\t")
            if len(f) == 4 and f[0].isdigit():
                table.append([int(f[0]), float(f[1]), float(f[2])])
        tail = "\n".join(txt[-6:])
        out[name] = {"num_sites": L, "bins": table,
                     "avg_mutations_sim": float(re.search(r"simulation: ([\d.e+]+)", tail).group(1)),
                     "avg_mutations_sfs": float(re.search(r"SFS: ([\d.e+]+)", tail).group(1)),
                     "time_ms_gtx980": float(re.search(r"\(ms\): ([\d.]+)", tail).group(1))}
    txt = (ref_root / "examples" / "example_dadi" / "dadi_example.out").read_text().splitlines()
    vals = [float(x) for x in txt if re.fullmatch(r"-?\d[\d.e+-]*", x.strip())]
    out["dadi_expectation"] = vals
    (HERE / "dadi_reference.json").write_text(json.dumps(out))


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("REF", str(ROOT.parent / "reference")))
    a = ap.parse_args()
    ref = Path(a.reference)
    hostrng(ref)
    example_compilation(ref)
    dadi(ref)
    print("fixtures written to", HERE)
