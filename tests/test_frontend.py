"""The drop-in C++ front-end (include/3P/) builds with plain g++ and its host-side semantics match the
reference's definitions (template_inline_simulation_functors.cuh, inline_go_fish_data_struct.hpp).
No GPU needed."""
from __future__ import annotations

import math
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
INC = ROOT / "include" / "3P"
F32 = np.float32


@pytest.fixture(scope="module")
def host_values(tmp_path_factory):
    d = tmp_path_factory.mktemp("fe")
    exe = d / "fe"
    subprocess.run(["g++", "-O1", "-std=c++17", "-Wall", "-Wno-unused-parameter", "-I", str(INC),
                    str(ROOT / "tests" / "cpp" / "frontend_host_test.cpp"), "-o", str(exe),
                    "-L", str(ROOT / "parallelpopgen_b200"), "-lgofish_b200",
                    "-Wl,-rpath," + str(ROOT / "parallelpopgen_b200")], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return {k: float(v) for k, v in (ln.split() for ln in out.splitlines())}


def test_scenario_drivers_compile_with_gpp(tmp_path):
    subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-Wno-unused-parameter", "-I", str(INC),
                    "-I", str(ROOT / "tests" / "cpp"), str(ROOT / "tests" / "cpp" / "gofish_driver.cpp")], check=True)


def test_demography_models(host_values):
    v = host_values
    assert v["dem_exp_g105"] == round(F32(10000) * np.exp(F32(0.01) * F32(100)))
    term = np.exp(F32(0.005) * F32(1000))
    assert v["dem_log_g1000"] == round(F32(500000) * F32(10000) * term / (F32(500000) + F32(10000) * (term - F32(1))))
    assert abs(v["dem_log_g5000"] - 500000) <= 1  # saturates at the carrying capacity
    assert v["dem_sine_g50"] == int(F32(1000) * np.sin(F32(0.01) * F32(50)) + F32(20000))
    assert (v["dem_ps_p0"], v["dem_ps_p1"]) == (100, 7)
    assert (v["dem_pw_99"], v["dem_pw_100"]) == (10, 20)


def test_migration_models(host_values):
    v = host_values
    assert v["mig_eq_self"] == float(F32(1) - F32(2) * F32(0.01))
    assert v["mig_eq_other"] == float(F32(0.01))
    assert v["mig_eq1_other"] == 0.0  # a single population has no migrants
    assert v["mig_dir_01"] == 0.5 and v["mig_dir_10"] == float(F32(0.01))
    assert v["mig_pw_9"] == float(F32(0.01)) and v["mig_pw_10"] == 0.5


def test_parameter_and_boolean_models(host_values):
    v = host_values
    assert v["fmh_sine_g3"] == float(F32(0.1) * np.sin(F32(0.5) * F32(3)) + F32(0.2))
    # piecewise with generation_shift 2: switches at inflection 5 + shift 2
    assert (v["fmh_pw_6"], v["fmh_pw_7"]) == (float(F32(0.1)), float(F32(0.9)))
    assert (v["pulse_15"], v["pulse_14"]) == (1, 0)
    assert (v["bpw_2"], v["bpw_3"]) == (0, 1)


def test_selection_models_and_affine_coefficients(host_values):
    v = host_values
    denom = F32(2 * 5000) / F32(1.25)
    assert v["sel_const_s"] == float(F32(-10) / denom)
    assert v["sel_lin_slope"] == float(F32(2) / denom) and v["sel_lin_intercept"] == float(F32(-1) / denom)
    assert v["sel_pw99_slope"] == 0.0 and v["sel_pw99_intercept"] == v["sel_const_s"]
    assert v["sel_pw100_slope"] == v["sel_lin_slope"]
    assert v["sel_ps_p1"] == float(F32(0.02)) and v["sel_ps_p0"] == 0.0
    assert abs(v["sel_sine_g12"] - (0.01 * math.sin(0.1 * 12) + 0.001)) < 1e-7


def test_allele_trajectories_defaults(host_values):
    v = host_values
    assert v["default_seed1"] == float(np.int32(np.uint32(0xBEEFF00D)))
    assert v["default_seed2"] == float(np.int32(np.uint32(0xDECAFBAD)))
    assert v["default_sites"] == 1000 and v["default_compact"] == 35 and v["default_init_mse"] == 1
    assert v["default_prev_sample"] == -1 and v["default_device"] == -1
    assert v["dump_empty_has_no_sim"] == 1


def test_sfs_copies_are_deep(host_values):
    """Spectrum::SFS is copyable as in the reference; here the copies own their arrays."""
    v = host_values
    assert v["sfs_copy_bin3"] == 30.0 and v["sfs_assigned_bin3"] == 30.0
    assert v["sfs_copy_distinct"] == 1 and v["sfs_copy_fields"] == 1
    assert v["sfs_joint_copy_last"] == 11.0
