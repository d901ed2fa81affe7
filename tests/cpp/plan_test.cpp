// Host-only checks of the engine's planning logic (gf_plan.h): the batched engine's record layout,
// its lock-step finishing schedule, and the generations a multi-population window may hold.
#include <cstdio>
#include <cstring>
#include <random>
#include <set>
#include <vector>

#include "gf_plan.h"

static int failures = 0;
#define CHECK(cond, ...)                        \
  do {                                          \
    if (!(cond)) {                              \
      std::printf("FAIL %s:%d: ", __FILE__, __LINE__); \
      std::printf(__VA_ARGS__);                 \
      std::printf("\n");                        \
      if (++failures > 20) return;              \
    }                                           \
  } while (0)

static std::vector<gf_replicate> draw(int R, unsigned seed, bool mixed_cadence) {
  std::mt19937 rng(seed);
  std::vector<gf_replicate> reps(R);
  for (int r = 0; r < R; ++r) {
    std::memset(&reps[r], 0, sizeof(gf_replicate));
    reps[r].num_generations = static_cast<int>(rng() % 4000);   // 0 .. 3999 (some empty)
    reps[r].compact_interval = mixed_cadence ? 1 + static_cast<int>(rng() % 60) : 10;
  }
  return reps;
}

static void check_plan(const std::vector<gf_replicate>& reps, long long budget) {
  const int R = static_cast<int>(reps.size());
  const gf::RecordPlan P = gf::plan_records(reps.data(), R, budget, 512);
  long long total = 0;
  for (auto& p : reps) total += p.num_generations;
  CHECK(P.total == total && P.region_base[P.nregions] == total, "total %lld vs %lld", P.total, total);
  if (P.ring_slots > 0) {
    CHECK(P.ring_slots >= 2 && P.ring_slots < P.nregions, "ring of %d slots for %d regions", P.ring_slots, P.nregions);
    CHECK(P.slot_records == P.largest && P.slots == P.ring_slots * P.largest, "ring slot sizes");
    CHECK(total > budget || total >= (1ll << 31), "ring without need");
  } else {
    CHECK(P.slots == total, "resident slots %lld vs %lld", P.slots, total);
  }
  for (int j = 0; j < P.nregions; ++j) CHECK(P.region_base[j + 1] - P.region_base[j] <= P.largest, "region size");
  // every record has one index; within a region (resident: everywhere) indices never collide
  std::vector<std::set<long long>> used(P.ring_slots > 0 ? P.nregions : 1);
  for (int r = 0; r < R; ++r) {
    const int G = reps[r].num_generations;
    CHECK(P.chunk[r] % std::max(reps[r].compact_interval, 1) == 0, "slab not a multiple of the cadence");
    for (int g = 0; g < G; ++g) {
      const long long i = P.record_index(r, g);
      CHECK(i >= 0 && i < P.slots, "replicate %d generation %d: index %lld of %lld", r, g, i, P.slots);
      auto& u = used[P.ring_slots > 0 ? g / P.chunk[r] : 0];
      CHECK(u.insert(i).second, "replicate %d generation %d: index %lld used twice", r, g, i);
    }
    // windows of its cadence are contiguous and inside one slab
    const int c = std::max(reps[r].compact_interval, 1);
    for (int g = 0; g < G; g += c) {
      const int n = std::min(c, G - g);
      CHECK(g / P.chunk[r] == (g + n - 1) / P.chunk[r], "replicate %d window at %d straddles slabs", r, g);
      CHECK(P.record_index(r, g + n - 1) - P.record_index(r, g) == n - 1, "window records not contiguous");
      // lock-step: super-step g / c is in region (g / c) / slab_windows for every replicate
      CHECK(g / P.chunk[r] == (g / c) / P.slab_windows, "replicate %d not in lock-step at %d", r, g);
    }
  }
  // finishing schedule: every replicate with generations once, at its last window
  const auto fin = gf::plan_finish_steps(reps.data(), R);
  std::vector<int> seen(R, 0);
  for (size_t k = 0; k < fin.size(); ++k)
    for (int r : fin[k]) {
      ++seen[r];
      const int c = std::max(reps[r].compact_interval, 1);
      CHECK(static_cast<long long>(k) * c < reps[r].num_generations &&
                (static_cast<long long>(k) + 1) * c >= reps[r].num_generations,
            "replicate %d finishes at step %zu", r, k);
    }
  for (int r = 0; r < R; ++r) CHECK(seen[r] == (reps[r].num_generations > 0 ? 1 : 0), "replicate %d listed %d times", r, seen[r]);
}

static void check_window_rules() {
  gf_generation g;
  std::memset(&g, 0, sizeof(g));
  for (int p = 0; p < 3; ++p) {
    g.pop[p].drift = 1;
    g.pop[p].Nchrom_e = 1000;
  }
  CHECK(gf::mp_window_generation_ok(g, 3, 0x7, 4), "all drifted");
  CHECK(!gf::mp_window_generation_ok(g, 1, 0x1, 4), "one population is not a multi-population window");
  CHECK(!gf::mp_window_generation_ok(g, 5, 0x1f, 4), "more populations than the kernel holds");
  g.pop[2].drift = 0;
  g.pop[2].Nchrom_e = 0;
  CHECK(gf::mp_window_generation_ok(g, 3, 0x3, 4), "unfounded population with zero rows");
  CHECK(!gf::mp_window_generation_ok(g, 3, 0x7, 4), "undrifted population whose rows may be nonzero");
  g.pop[2].drift = 1;
  CHECK(!gf::mp_window_generation_ok(g, 3, 0x7, 4), "extinction generation (drifted with Nchrom_e 0)");
  CHECK(gf::drifted_populations(g, 3) == 0x7, "drift mask");
}

int main() {
  for (unsigned seed = 1; seed <= 6 && failures == 0; ++seed) {
    const auto reps = draw(seed % 2 ? 200 : 57, seed, seed > 3);
    check_plan(reps, 1ll << 26);   // resident
    const gf::RecordPlan full = gf::plan_records(reps.data(), static_cast<int>(reps.size()), 1ll << 26, 512);
    check_plan(reps, 3 * full.largest);   // ring of three regions
    check_plan(reps, 10);                 // ring of two
    const int ring3 = gf::plan_records(reps.data(), static_cast<int>(reps.size()), 3 * full.largest, 512).ring_slots;
    if (ring3 != (full.nregions > 3 ? 3 : 0)) {
      std::printf("FAIL: ring of %d slots for a three-region budget (%d regions)\n", ring3, full.nregions);
      ++failures;
    }
  }
  check_window_rules();
  std::printf(failures ? "FAILED %d\n" : "OK\n", failures);
  return failures ? 1 : 0;
}
