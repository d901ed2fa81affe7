"""The engine's host-only planning logic (csrc/gf_plan.h), compiled with the host compiler: the
batched engine's record layout (resident and ring, every record one index, windows contiguous and
inside one slab, lock-step regions), its finishing schedule, and the rules for multi-population
windows."""
from __future__ import annotations

import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_plan_logic(tmp_path):
    exe = tmp_path / "plan_test"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", str(ROOT / "parallelpopgen_b200" / "csrc"),
                    "-I", str(ROOT / "include"), str(ROOT / "tests" / "cpp" / "plan_test.cpp"), "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.strip().endswith("OK"), out.stdout
