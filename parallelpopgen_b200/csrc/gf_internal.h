// Internal declarations shared by the engine's translation units.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <deque>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/gofish_b200.h"
#include "gf_plan.h"

namespace gf {

constexpr int kMaxPops = GF_MAX_POPULATIONS;
// One drift thread owns one quad of mutations (4 consecutive slots) -- the reference's counter layout
// draws one Philox block per quad.  A tile is the 1024 slots of one 256-thread block, and is also
// the unit of the compaction scan.
constexpr int kDriftThreads = 256;
constexpr int kTileSlots = kDriftThreads * 4;
// Row stride granularity of the device arrays, in slots: keeps every row 128-byte aligned so quad
// loads and stores are 16-byte aligned and whole tiles map to whole 32-bit flag words.
constexpr int kSlotAlign = kTileSlots;

// Device status word codes (bounded waits and range checks report here instead of trapping).
enum DeviceFault : int {
  kFaultNone = 0,
  kFaultCapacity = 1,  // a kernel was asked to write beyond the allocated rows
  kFaultScanTimeout = 2,
  kFaultRecords = 3,   // a batched replicate's window has no generation records (a planning error)
};

// Per-generation kernel arguments (passed by value; ~1.3 KB).
struct GenArgs {
  int generation;
  int num_pops;
  int seed1, seed2;
  int new_total;                 // new mutations appended this generation, all populations
  int new_offset[kMaxPops + 1];  // exclusive prefix of the per-population new counts
  float new_freq[kMaxPops];      // 1.f / Nchrom_e, computed on the host as the reference does
  int Nc[kMaxPops];              // Nchrom_e used by the drift of each population
  float F[kMaxPops], h[kMaxPops];
  float sel_a[kMaxPops], sel_b[kMaxPops];
  int drift_mask;                // bit p: population p is drifted this generation
  int alive_mask;                // bit p: demography(p, generation) > 0 (compaction flag)
  int flag;                      // 1: write compaction flags and tile counts for this generation
  int check_preserved;           // 1: some mutation may carry the preserved mark
  float mig[kMaxPops * kMaxPops];  // [from * num_pops + to]
  // per-slot selection coefficients s(pop, generation, x_mig) written by the caller before this
  // generation ([P][sel_stride], slots below the generation's starting count); null: affine (sel_a, sel_b)
  const float* sel_table;
  long long sel_stride;
};

// One generation of one single-population replicate, as the window kernel reads it (36 B).
struct WinGen {
  int generation;
  int Nc;          // Nchrom_e of the drift (0: extinction generation, the row is cleared)
  int new_count;   // new mutations appended after the drift (host draw)
  float new_freq;  // 1.f / Nchrom_e, computed on the host
  float F, h, sel_a, sel_b;
  int alive;       // demography(pop, generation) > 0 (compaction flag of the window's last generation)
};

// One replicate's window in a window launch (56 B).  A replicate owns the arena slots
// [base, base + capacity) of every per-slot array; base is a multiple of 1024.
struct WinRep {
  long long base;
  long long capacity;
  int rec;              // first WinGen record of the window
  int ngen;             // generations in the window (>= 1)
  int tile0;            // first launch tile of the replicate
  int ntiles;           // launch tiles of the replicate (covers its end-of-window count)
  int seed1, seed2;
  int check_preserved;  // some slot may carry the preserved mark
  int compact;          // flags after the last generation; compaction follows
  int preserve;         // the compaction marks survivors preserved
  int rep;              // index into the per-replicate count arrays
  long long births;     // new mutations over the window: tiles at or beyond M0 + births hold nothing
};

// Which table entries a batched launch visits: by default all nreps in order; a batch with
// precomputed records passes the list of its unfinished replicates, built on the device each
// super-step (their table indices, first tiles and count), so that finished ones cost nothing.
struct RepList {
  const int* rep = nullptr;     // [i] table index of the i-th listed replicate (null: i)
  const int* tile0 = nullptr;   // [i] its first tile (null: the table's tile0 of entry i)
  const int* count = nullptr;   // how many are listed, on the device (null: nreps)
};

// Pointers and sizes of one window launch plus its optional compaction.
struct WindowLaunch {
  const float* A;          // state at the window start
  float* B;                // state at the window end
  int* id_gp_cur;          // IDs (new mutations are written here)
  int* id_tid_cur;
  int* id_gp_next;         // compaction output of the IDs
  int* id_tid_next;
  unsigned* flags;
  unsigned* tile_count;
  unsigned* tile_offset;
  const int* M_in;         // [rep] counts at the window start
  int* M_end;              // [rep] counts at the window end (before compaction)
  int* M_next;             // [rep] counts for the next window when not compacting (may alias nothing)
  int* M_out;              // [rep] counts after compaction
  const WinRep* reps;      // device
  int nreps;
  const WinGen* recs;      // device
  int total_tiles;         // launch tiles (an upper bound when total_tiles_dev is set)
  const int* total_tiles_dev = nullptr;   // device-side tile count (tiles assigned on the device)
  bool any_compact;
  unsigned long long* stats;
  int* fault;
  int* sched = nullptr;    // two zeroed device words: next tile to hand out, blocks finished (the
                           // launch's last block sets both back to zero)
  // one replicate (the plain engine): its seeds, from which the launch passes the Philox round keys
  // as kernel parameters
  bool uniform_key = false;
  int seed1 = 0, seed2 = 0;
  RepList list{};
};

// Words of the engine's device counter block (d_count) and the first of the window scheduler's two.
constexpr int kCountWords = 8;
constexpr int kSchedWord = 4;

// Longest window (generations per window launch).
constexpr int kMaxWindowGenerations = 128;

// One multi-population window launch of the plain engine (window_mp.cu): generations
// table[0 .. ngen) from state A into state B, counts in d_count[slot_in] -> d_count[slot_out] (and
// d_count[3]), compaction flags and tile counts after the last generation when `compact`.
struct WindowMpLaunch {
  int P;
  const float* A;
  float* B;
  long long stride;          // row stride of A and B in slots (= the capacity)
  int* id_gp;
  int* id_tid;
  unsigned* flags;
  unsigned* tile_count;
  int* d_count;
  int slot_in, slot_out;
  const GenArgs* table;      // device
  int ngen;
  long long births;          // new mutations over the window (host draws)
  int compact;
  int check_preserved;
  int seed1, seed2;
  unsigned long long* stats;
  int tiles_bound;           // launch tiles (an upper bound of the end-of-window tiles)
};

// What a batched super-step derives each replicate's window from on the device (precomputed records):
// super-step k runs generations (k c, min(G, (k + 1) c)] of a replicate with cadence c and G
// generations, from record slab j = k / slab_windows.
struct StepRep {
  int cadence;
  int gens;
  int chunk;   // generations per slab
  int pad;
};
struct BatchStepPlan {
  int slab_windows;
  int nregions;
  int ring_slots;          // 0: every region resident at region_base[j]; else region j in slot j % ring_slots
  int pad;
  long long slot_records;  // records per ring slot
};

// Host record of one replicate of a batch.
struct BatchRep {
  gf_replicate p;
  long long base = 0;       // arena offset (multiple of 1024)
  long long capacity = 0;   // arena slots
  int generation = 0;       // last generation run
  int next_compact = 0;
  int M = 0;                // count after the last read-back
  int id_buf = 0;           // ID buffer holding its state
  int m_slot = 0;           // count array (d_M[m_slot]) holding its latest count
  int chunk = 0;            // generations per record slab (a multiple of its compaction cadence)
  bool done = false;
};

struct Batch {
  int R = 0;
  std::vector<BatchRep> reps;
  long long arena = 0;
  float* freq[2] = {nullptr, nullptr};
  int* id_gp[2] = {nullptr, nullptr};
  int* id_tid[2] = {nullptr, nullptr};
  unsigned* flags = nullptr;
  unsigned* tile_count = nullptr;
  unsigned* tile_offset = nullptr;
  int* d_M[2] = {nullptr, nullptr};
  int* d_Mend = nullptr;
  int* h_M = nullptr;        // pinned read-back of the counts
  int mslot = 0;
  int id_cur = 0;
  WinGen* d_recs = nullptr;
  WinGen* h_recs = nullptr;
  size_t recs_cap = 0;
  WinRep* d_reps = nullptr;
  WinRep* h_reps = nullptr;
  size_t reps_cap = 0;
  long long super_steps = 0;
  long long generations = 0;
  // generation records of every replicate, computed once at begin (when they fit the budget)
  bool precomputed = false;
  WinGen* d_all_recs = nullptr;
  bool counts_stale = false;          // counts on the device are newer than reps[].M
  int* d_total_tiles = nullptr;       // tiles of the current super-step, assigned on the device
  // generation records, drawn by host threads region by region (region j holds slab j -- the
  // generations (j * chunk, (j + 1) * chunk] -- of every replicate that runs that long) while the GPU
  // runs the super-steps; a region is uploaded once all of its slabs are drawn (batch.cu)
  RecordPlan plan;                            // layout of the records (gf_plan.h)
  int uploaded = 0;                           // regions uploaded so far
  int upload_done = 0;                        // regions whose upload has finished (ring mode)
  std::vector<cudaEvent_t> slot_upload;       // ring mode: the last upload from each staging slot
  std::unique_ptr<std::atomic<long long>[]> region_done;   // slabs drawn per region
  std::atomic<long long> next_job{0};         // producers' job counter (region-major over replicates)
  std::atomic<int> producible{0};             // producers may draw regions below this
  std::atomic<bool> cancel{false};
  std::vector<std::thread> producers;
  double record_wait_ms = 0.0;                // host time the super-steps waited for records
  // Every replicate advances one window of its cadence per super-step from generation 0, so after k
  // super-steps an unfinished replicate is at generation k * c_r and in record region k / slab_windows.
  // The host keeps only the list of unfinished replicates and the replicates finishing at each step;
  // their per-replicate fields are brought up to date when a run returns (sync_progress).
  std::vector<int> active;                    // unfinished replicates, in index order
  bool active_dirty = true;
  long long active_cadence_sum = 0;           // sum of their cadences (generations per super-step)
  std::vector<std::vector<int>> finish_at;    // [k]: replicates whose last window is super-step k
  // precomputed records: a replicate table of all R replicates in index order, whose per-window fields
  // (records, generations, tiles, births; none once finished) a kernel derives from the super-step
  // counter on the device, so a super-step needs no host table and no upload
  WinRep* d_table = nullptr;
  StepRep* d_steprep = nullptr;
  int* d_region_off = nullptr;                // [r * nregions + j]
  long long* d_region_base = nullptr;         // [j], resident layout
  int* d_step = nullptr;                      // super-steps launched (advanced by the step kernel)
  int* d_list_rep = nullptr;                  // the step's unfinished replicates (RepList), built by the
  int* d_list_tile0 = nullptr;                // step kernel
  int* d_list_count = nullptr;
  BatchStepPlan step_plan{};
  long long all_tiles = 0;                    // segment tiles of all replicates (the launch bound)
  // one record slab's super-steps as a CUDA graph, per starting buffer parity, and the draw tuning
  // it was captured with
  cudaGraphExec_t slab_graph[2] = {nullptr, nullptr};
  bool graphs_off = false;                    // the stream could not be captured: step by step
  int graph_draw[2] = {-1, -1};
  int graph_blocks[2] = {-1, -1};
  cudaEvent_t* step_ev = nullptr;             // 64 (the engine's batch_ahead[0..63])
  cudaEvent_t* slab_ev = nullptr;             // 2 (batch_ahead[64..65])
  long long steps_enqueued = 0, slabs_enqueued = 0;
};

struct PendingCount {
  cudaEvent_t event;
  int slot;           // index into the pinned readback array
  long long added;    // new mutations appended after this compaction
};

struct Engine {
  int device = 0;
  int num_sms = 148;
  int draw_strategy = 0;   // DrawStrategy of the drift and window kernels
  int blocks_per_sm = 0;   // drift grid limit per SM (0: occupancy maximum)
  long long batch_record_budget = 64ll << 20;   // batches up to this many records are precomputed
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  // stream-ordered pool for the mutation arrays and per-run scratch; it keeps freed memory, so a new
  // simulation on the same engine reuses the previous one's buffers without driver allocations
  cudaMemPool_t pool = nullptr;
  std::string last_error;

  // simulation constants
  bool active = false;
  int P = 1;
  int seed1 = 0, seed2 = 0;
  float num_sites = 0.f;
  int compact_interval = 0;
  bool any_preserved = false;
  int live_rows = 0;         // bit p: row p may hold a nonzero value in either state buffer
  long long step_index = 0;  // generations run since begin
  int count_slot = 0;        // d_count slot holding the current mutation count

  // device arrays; capacity = row stride in slots
  long long capacity = 0;
  float* freq[2] = {nullptr, nullptr};      // [P][capacity]
  int* id_gp[2] = {nullptr, nullptr};       // origin generation | origin population << 24
  int* id_tid[2] = {nullptr, nullptr};      // origin threadID; negative = preserved
  int id_cur = 0;                           // ID buffer of the current generation (swaps on compaction)
  unsigned* flags = nullptr;                // compaction bitmask, 1 bit per slot
  unsigned* tile_count = nullptr;           // survivors per tile
  unsigned* tile_offset = nullptr;          // exclusive prefix of tile_count
  int cur = 0;                              // buffer holding the current generation
  int* d_count = nullptr;                   // [0],[1]: mutation count ping-pong; [2]: device status;
                                            // [3]: slots at the end of a launch; [4],[5]: window tile
                                            // scheduler (kSchedWord); kCountWords words in all
  int* h_pinned = nullptr;                  // pinned readback slots
  int pinned_slots = 64;
  int next_slot = 0;

  // host tracking of the mutation count
  long long M_upper = 0;   // upper bound on the current count (exact when nothing is pending)
  bool M_exact = true;
  // an asynchronous time sample (gf_sim_sample_begin / _wait): the state packed into device scratch on
  // the engine's stream, copied to the caller's arrays on a second stream
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t sample_packed = nullptr, sample_done = nullptr;
  void* sample_scratch = nullptr;
  size_t sample_scratch_bytes = 0;
  int* h_sample_count = nullptr;   // page-locked: the sample's count
  bool sample_in_flight = false;
  float* sample_freq_out = nullptr;   // the in-flight sample's destination arrays
  int32_t* sample_ids_out = nullptr;
  long long sample_bound = 0;         // slots its scratch was laid out for
  int sample_P = 0;                   // populations of the sampled state
  bool sample_to_stage = false;       // the wait copies into the engine's staging
  float* h_sample_stage = nullptr;    // page-locked staging of a sample's rows
  size_t sample_stage_cap = 0;        // in floats
  std::deque<PendingCount> pending;
  std::vector<cudaEvent_t> free_events;

  // per-generation parameter tables (double-buffered: the host fills one while the GPU reads the other)
  GenArgs* d_table[2] = {nullptr, nullptr};
  GenArgs* h_table[2] = {nullptr, nullptr};
  size_t table_cap[2] = {0, 0};
  cudaEvent_t table_done[2] = {nullptr, nullptr};
  int table_next = 0;
  // window records of the single-population path (same double-buffering as the tables above)
  WinGen* d_wgen[2] = {nullptr, nullptr};
  WinGen* h_wgen[2] = {nullptr, nullptr};
  WinRep* d_wrep[2] = {nullptr, nullptr};
  WinRep* h_wrep[2] = {nullptr, nullptr};
  size_t wtable_cap[2] = {0, 0};
  bool use_windows = true;   // single-population runs use the window kernel
  // per-slot selection table of generations whose selection model is evaluated by the caller on the
  // device (gf_sim_selection_view): [P][sel_table_stride] floats, grown with the state's capacity
  float* sel_table = nullptr;
  long long sel_table_stride = 0;

  // batched replicates (gf_batch_*)
  Batch* batch = nullptr;

  // measurement
  unsigned long long* d_stats = nullptr;  // [0] sum of drift slots, [1] generations
  long long compactions = 0;
  long long kernel_launches = 0;
  bool profiling = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof_drift, prof_compact;
  std::vector<cudaEvent_t> prof_pool;

  // spectrum scratch
  // page-locked staging of batched generation records, kept across batches (grown on demand)
  WinGen* h_rec_stage = nullptr;
  size_t h_rec_stage_cap = 0;
  // the batched engine's page-locked count read-back, kept across batches (grown on demand): pinning
  // and freeing it per batch cost up to hundreds of milliseconds on a busy host
  int* batch_h_M = nullptr;
  size_t batch_h_M_cap = 0;
  // events that keep the batched engine's host at most 64 super-steps (or two graph-replayed slabs)
  // ahead of the GPU, so record uploads are not queued far behind the launches that precede them
  cudaEvent_t batch_ahead[66] = {};
  // the batched engine's device arena (state, IDs, flags, tile counts) and generation records, also
  // kept across batches and grown on demand: carving a new batch's gigabytes out of the stream-ordered
  // pool after its small temporaries fragmented it could map fresh memory (~0.5 s) every other batch
  void* batch_arena_mem = nullptr;
  size_t batch_arena_bytes = 0;
  void* batch_recs_mem = nullptr;
  size_t batch_recs_bytes = 0;
  void* batch_plan_mem = nullptr;             // the replicate table and the record plan on the device
  size_t batch_plan_bytes = 0;
  void* spec_scratch = nullptr;
  size_t spec_scratch_bytes = 0;
  float* spec_in = nullptr;
  size_t spec_in_bytes = 0;
  float* spec_out = nullptr;
  size_t spec_out_bytes = 0;
};

// Error helpers: record a message on the engine and return the status.
gf_status fail(Engine* e, gf_status st, const char* fmt, ...);
gf_status cuda_fail(Engine* e, cudaError_t err, const char* what);

#define GF_CUDA(e, call)                                      \
  do {                                                        \
    cudaError_t _err = (call);                                \
    if (_err != cudaSuccess) return ::gf::cuda_fail((e), _err, #call); \
  } while (0)

gf_status pool_alloc(Engine* e, void** ptr, size_t bytes);
gf_status ensure_scratch(Engine* e, void** ptr, size_t* have, size_t need);

// Window launch (+ segmented compaction into compact_dst), window.cu.
void assign_batch_tiles(Engine* e, WinRep* d_reps, int nreps, const int* M_in, const WinGen* recs,
                        int* total_out);
// Super-step *d_step of a batch with precomputed records: every replicate's window fields and tiles
// in d_table (all R replicates; finished ones get none), then *d_step + 1.
void batch_step_tiles(Engine* e, WinRep* d_table, int R, const int* M_in, const WinGen* recs, int* total_out,
                      int* d_step, const BatchStepPlan& plan, const int* region_off, const long long* region_base,
                      const StepRep* steprep, int* fault, int* list_rep, int* list_tile0, int* list_count);
// after_window, before_compaction (either may be null): recorded on the stream between the window
// kernel and its compaction (two events, so that each timing pair owns its own)
gf_status window_run(Engine* e, const WindowLaunch& w, float* compact_dst, cudaEvent_t after_window = nullptr,
                     cudaEvent_t before_compaction = nullptr);
// Multi-population window launch (window_mp.cu); P in [2, 4].
gf_status window_mp_run(Engine* e, const WindowMpLaunch& w);
constexpr int kMaxWindowPops = 4;

// Host draw of one population's new-mutation count (engine.cu).
int host_new_mutation_count(int seed1, int seed2, float mu, int Nchrom_e, float num_sites, int generation, int pop);

// Releases the batch of an engine (batch.cu).
void release_batch(Engine* e);

}  // namespace gf

// The opaque handle of the C ABI.
struct gf_engine {
  gf::Engine impl;
};

#include <new>
#include <exception>

namespace gf {
// No host exception crosses the C ABI: a failed host allocation or thread start inside an entry
// point becomes a status (with the message on the engine).
template <typename F>
gf_status guard_host(gf_engine* g, F&& body) {
  try {
    return body();
  } catch (const std::bad_alloc&) {
    return g ? fail(&g->impl, GF_ERR_OUT_OF_MEMORY, "host allocation failed") : GF_ERR_OUT_OF_MEMORY;
  } catch (const std::exception& ex) {
    return g ? fail(&g->impl, GF_ERR_STATE, "host error: %s", ex.what()) : GF_ERR_STATE;
  }
}
}  // namespace gf
