// Host-only planning logic of the engine, free of CUDA so that it compiles and is tested with a plain
// C++ compiler: the layout of the batched engine's generation records (regions of slabs, resident or
// cycling through a ring of slots), the lock-step finishing schedule of its replicates, and which
// generations a multi-population window may hold.
#pragma once

#include <algorithm>
#include <cstdint>
#include <vector>

#include "../../include/gofish_b200.h"

namespace gf {

// Generation records of a batch.  Slab j of replicate r is its generations (j * chunk_r,
// (j + 1) * chunk_r] with chunk_r = slab_windows * c_r (c_r its cadence): every replicate advances one
// window per super-step, so all of them enter slab j at super-step j * slab_windows, and no window
// straddles two slabs.  Region j holds slab j of every replicate that runs that long, in replicate
// order.  Resident layout: the regions one after another (region_base); ring layout: region j in slot
// j % ring_slots of slot_records records each.
struct RecordPlan {
  int slab_windows = 1;
  int nregions = 0;
  std::vector<int> chunk;               // [r] generations per slab
  std::vector<long long> region_base;   // [j] first record of region j, resident layout (nregions + 1)
  std::vector<long long> region_jobs;   // [j] slabs in region j
  std::vector<int> region_off;          // [r * nregions + j] offset of replicate r's slab in region j, or -1
  long long total = 0;                  // records of the batch
  long long largest = 0;                // records of the largest region
  int ring_slots = 0;                   // 0: resident; K >= 2: ring of K slots
  long long slot_records = 0;
  long long slots = 0;                  // records the buffers hold

  long long slot_base(int j) const {
    return ring_slots > 0 ? static_cast<long long>(j % ring_slots) * slot_records : region_base[j];
  }
  // Index of replicate r's record of generation g + 1 (g generations done), or -1.
  long long record_index(int r, int g) const {
    const int j = g / chunk[r];
    if (j >= nregions) return -1;
    const int off = region_off[static_cast<size_t>(r) * nregions + j];
    if (off < 0) return -1;
    return slot_base(j) + off + (g - static_cast<long long>(j) * chunk[r]);
  }
};

// Plan the records of `R` replicates for a record budget: resident when the total fits it (and
// record indices stay within int32), else a ring of as many whole regions as fit (at least two).
inline RecordPlan plan_records(const gf_replicate* reps, int R, long long budget, int slab_target) {
  RecordPlan P;
  int cmax = 1;
  for (int r = 0; r < R; ++r) {
    P.total += std::max(reps[r].num_generations, 0);
    cmax = std::max(cmax, reps[r].compact_interval);
  }
  P.slab_windows = std::max(1, (slab_target + cmax - 1) / cmax);
  P.chunk.resize(R);
  for (int r = 0; r < R; ++r) {
    P.chunk[r] = P.slab_windows * std::max(reps[r].compact_interval, 1);
    P.nregions = std::max(P.nregions, (std::max(reps[r].num_generations, 0) + P.chunk[r] - 1) / P.chunk[r]);
  }
  const int nreg = P.nregions;
  P.region_off.assign(static_cast<size_t>(R) * nreg, -1);
  P.region_base.assign(nreg + 1, 0);
  P.region_jobs.assign(nreg, 0);
  long long off = 0;
  for (int j = 0; j < nreg; ++j) {
    P.region_base[j] = off;
    for (int r = 0; r < R; ++r) {
      const int G = reps[r].num_generations;
      const int g0 = j * P.chunk[r];
      if (g0 >= G) continue;
      P.region_off[static_cast<size_t>(r) * nreg + j] = static_cast<int>(off - P.region_base[j]);
      off += std::min(G, g0 + P.chunk[r]) - g0;
      P.region_jobs[j] += 1;
    }
    P.largest = std::max(P.largest, off - P.region_base[j]);
  }
  P.region_base[nreg] = off;
  P.slots = P.total;
  if ((P.total > budget || P.total >= (1ll << 31)) && nreg > 2) {
    const long long K = std::min<long long>(nreg, std::max<long long>(2, budget / std::max<long long>(P.largest, 1)));
    if (K < nreg) {
      P.ring_slots = static_cast<int>(K);
      P.slot_records = P.largest;
      P.slots = K * P.largest;
    }
  }
  return P;
}

// [k]: the replicates whose last window is super-step k (ceil(G / c) windows; none for G = 0).
inline std::vector<std::vector<int>> plan_finish_steps(const gf_replicate* reps, int R) {
  std::vector<std::vector<int>> at;
  for (int r = 0; r < R; ++r) {
    const int G = reps[r].num_generations;
    if (G <= 0) continue;
    const int c = std::max(reps[r].compact_interval, 1);
    const int last = (G + c - 1) / c - 1;
    if (static_cast<int>(at.size()) <= last) at.resize(last + 1);
    at[last].push_back(r);
  }
  return at;
}

// May a multi-population window (2 <= P <= max_pops) hold this generation?  Every population must be
// drifted with Nchrom_e > 0, or not drifted with its rows zero in both state buffers (`live_rows`:
// bit p set when population p's rows may hold a nonzero value).
inline bool mp_window_generation_ok(const gf_generation& g, int P, int live_rows, int max_pops) {
  if (P < 2 || P > max_pops) return false;
  for (int p = 0; p < P; ++p) {
    const gf_population_params& pp = g.pop[p];
    if (pp.drift) {
      if (pp.Nchrom_e <= 0) return false;
    } else if ((live_rows >> p) & 1) {
      return false;
    }
  }
  return true;
}

inline int drifted_populations(const gf_generation& g, int P) {
  int m = 0;
  for (int p = 0; p < P; ++p)
    if (g.pop[p].drift) m |= 1 << p;
  return m;
}

}  // namespace gf
