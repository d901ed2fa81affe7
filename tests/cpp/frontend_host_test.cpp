// Host-only checks of the drop-in C++ front-end (no GPU): Sim_Model functor values, the exact affine
// coefficients extracted from selection models, allele_trajectories semantics and its text dump.
// Prints "name value" lines that tests/test_frontend.py compares with the reference's definitions.
#include <cmath>
#include <cstdio>
#include <sstream>

#include "go_fish.cuh"
#include "spectrum.h"

using namespace Sim_Model;

static void line(const char* name, double v) { std::printf("%s %.17g\n", name, v); }

int main() {
  // demography
  demography_exponential_growth eg(0.01f, 10000, 5);
  line("dem_exp_g105", eg(0, 105));
  demography_logistic_growth lg(0.005f, 10000, 500000);
  line("dem_log_g1000", lg(0, 1000));
  line("dem_log_g5000", lg(0, 5000));
  demography_sine_wave sw(1000.f, 0.01f, 20000);
  line("dem_sine_g50", sw(0, 50));
  demography_population_specific<demography_constant, demography_constant> dps(demography_constant(100),
                                                                              demography_constant(7), 1);
  line("dem_ps_p0", dps(0, 3));
  line("dem_ps_p1", dps(1, 3));
  demography_piecewise<demography_constant, demography_constant> dpw(demography_constant(10), demography_constant(20), 100);
  line("dem_pw_99", dpw(0, 99));
  line("dem_pw_100", dpw(0, 100));
  // migration
  migration_constant_equal me(0.01f, 3);
  line("mig_eq_self", me(1, 1, 0));
  line("mig_eq_other", me(0, 2, 0));
  migration_constant_equal me1(0.01f, 1);
  line("mig_eq1_other", me1(0, 1, 0));
  migration_constant_directional<migration_constant_equal> md(0.5f, 0, 1, me);
  line("mig_dir_01", md(0, 1, 0));
  line("mig_dir_10", md(1, 0, 0));
  migration_piecewise<migration_constant_equal, migration_constant_directional<migration_constant_equal>> mpw(me, md, 10);
  line("mig_pw_9", mpw(0, 1, 9));
  line("mig_pw_10", mpw(0, 1, 10));
  // F / mu / h
  F_mu_h_sine_wave fs(0.1f, 0.5f, 0.2f);
  line("fmh_sine_g3", fs(0, 3));
  F_mu_h_piecewise<F_mu_h_constant, F_mu_h_constant> fpw(F_mu_h_constant(0.1f), F_mu_h_constant(0.9f), 5, 2);
  line("fmh_pw_6", fpw(0, 6));
  line("fmh_pw_7", fpw(0, 7));
  // booleans
  bool_pulse<bool_off, bool_on> pulse(bool_off(), bool_on(), 10, 5);
  line("pulse_15", pulse(15));
  line("pulse_14", pulse(14));
  bool_piecewise<bool_off, bool_on> bpw(bool_off(), bool_on(), 3);
  line("bpw_2", bpw(2));
  line("bpw_3", bpw(3));
  // selection and its affine coefficients
  demography_constant N(5000);
  F_mu_h_constant F(0.25f);
  selection_constant sc(-10.f, N, F);
  line("sel_const_s", sc.s);
  selection_linear_frequency_dependent sl(2.f, -1.f, N, F);
  float a, b;
  gofish_detail::selection_affine(sl, 0, 0, a, b);
  line("sel_lin_slope", a);
  line("sel_lin_intercept", b);
  line("sel_lin_at_03", sl(0, 0, 0.3f));
  selection_piecewise<selection_constant, selection_linear_frequency_dependent> spw(sc, sl, 100);
  gofish_detail::selection_affine(spw, 0, 99, a, b);
  line("sel_pw99_slope", a);
  line("sel_pw99_intercept", b);
  gofish_detail::selection_affine(spw, 0, 100, a, b);
  line("sel_pw100_slope", a);
  selection_population_specific<selection_constant, selection_constant> sps(selection_constant(0.f),
                                                                            selection_constant(0.02f), 1);
  gofish_detail::selection_affine(sps, 1, 7, a, b);
  line("sel_ps_p1", b);
  gofish_detail::selection_affine(sps, 0, 7, a, b);
  line("sel_ps_p0", b);
  // (run_sim takes the sine model's coefficient from the device, gf_selection_sine_values; the host
  // operator() is the plain-C++ evaluation a user may call)
  selection_sine_wave ssw(0.01f, 0.1f, 0.001f);
  line("sel_sine_g12", ssw(0, 12, 0.3f));

  // allele_trajectories: defaults, copy, dump, delete_time_sample
  GO_Fish::allele_trajectories t;
  line("default_seed1", t.sim_input_constants.seed1);
  line("default_seed2", t.sim_input_constants.seed2);
  line("default_sites", t.sim_input_constants.num_sites);
  line("default_compact", t.sim_input_constants.compact_interval);
  line("default_init_mse", t.sim_input_constants.init_mse);
  line("default_prev_sample", t.sim_input_constants.prev_sim_sample);
  line("default_device", t.sim_input_constants.device);
  std::ostringstream empty;
  empty << t;
  line("dump_empty_has_no_sim", empty.str().find("no simulation stored") != std::string::npos);

  // Spectrum::SFS copies (deep: each copy owns its arrays; the program must end without a double free)
  Spectrum::SFS sfs;
  sfs.num_populations = 1;
  sfs.sample_size = new int[1];
  sfs.sample_size[0] = 5;
  sfs.populations = new int[1];
  sfs.populations[0] = 1;
  sfs.frequency_spectrum = new float[5];
  for (int i = 0; i < 5; ++i) sfs.frequency_spectrum[i] = 10.f * i;
  sfs.num_sites = 100.f;
  sfs.num_mutations = 100.f;
  sfs.sampled_generation = 7;
  Spectrum::SFS copy(sfs);
  Spectrum::SFS assigned;
  assigned = sfs;
  sfs.frequency_spectrum[3] = -1.f;
  line("sfs_copy_bin3", copy.frequency_spectrum[3]);
  line("sfs_assigned_bin3", assigned.frequency_spectrum[3]);
  line("sfs_copy_distinct", copy.frequency_spectrum != sfs.frequency_spectrum && assigned.populations != sfs.populations);
  line("sfs_copy_fields", copy.sample_size[0] == 5 && copy.populations[0] == 1 && copy.sampled_generation == 7 &&
                              assigned.num_sites == 100.f);
  Spectrum::SFS joint;
  joint.num_populations = 2;
  joint.sample_size = new int[2];
  joint.sample_size[0] = 2;
  joint.sample_size[1] = 3;
  joint.frequency_spectrum = new float[12];
  for (int i = 0; i < 12; ++i) joint.frequency_spectrum[i] = static_cast<float>(i);
  Spectrum::SFS joint_copy(joint);
  line("sfs_joint_copy_last", joint_copy.frequency_spectrum[11]);
  return 0;
}
