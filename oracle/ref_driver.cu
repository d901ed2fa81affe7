// Oracle driver for the reference itself (test infrastructure only).
//
// Built by oracle/build_ref.sh against the unmodified ParallelPopGen 3P sources (3P/_internal/*.cu
// and its headers), with the reference's own flags (-O3 --use_fast_math), into oracle/_ref/.  It
// runs the reference on the GPU so that the engine can be compared with it bit for bit:
//   ref_driver sim <scenario> <out.bin> key=value ...   scenarios of tests/cpp/scenarios.h
//   ref_driver drift1 <in.bin> <out.bin> key=value ...  one call of the reference's
//        migration_selection_drift kernel (go_fish_impl.cuh:93-124) on a given frequency row
//   ref_driver draws <in.bin> <out.bin>                 RNG::ApproxRandBinom1 / ApproxRandPois1
//        (shared.cuh:251-267) evaluated on the device for a list of inputs
//   ref_driver hostrng <out.bin>                         RNG::Philox and ApproxRandPois1 evaluated
//        on the host (golden vectors for the CPU oracle; needs no GPU)
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../tests/cpp/scenarios.h"  // includes the reference's go_fish.cuh and spectrum.h

static std::vector<char> slurp(const char* path) {
  FILE* f = std::fopen(path, "rb");
  if (!f) { std::perror(path); std::exit(2); }
  std::fseek(f, 0, SEEK_END);
  const long n = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  std::vector<char> buf(n);
  if (n && std::fread(buf.data(), 1, n, f) != static_cast<size_t>(n)) { std::perror(path); std::exit(2); }
  std::fclose(f);
  return buf;
}

static void spit(const char* path, const void* data, size_t bytes) {
  FILE* f = std::fopen(path, "wb");
  if (!f) { std::perror(path); std::exit(2); }
  std::fwrite(data, 1, bytes, f);
  std::fclose(f);
}

#define CK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { std::fprintf(stderr, "CUDA %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, __LINE__); std::exit(3); } } while (0)

// drift1 input: int32 M, then float freq[M]; params: N F h s gen seed1 seed2
static int mode_drift1(const char* in, const char* out, const scn::Args& args) {
  std::vector<char> buf = slurp(in);
  int M;
  std::memcpy(&M, buf.data(), 4);
  const float* h_in = reinterpret_cast<const float*>(buf.data() + 4);
  const int array_length = (M + 31) / 32 * 32;
  float *d_prev, *d_next;
  int4* d_id;
  CK(cudaMalloc(&d_prev, sizeof(float) * array_length));
  CK(cudaMalloc(&d_next, sizeof(float) * array_length));
  CK(cudaMalloc(&d_id, sizeof(int4) * array_length));
  CK(cudaMemset(d_prev, 0, sizeof(float) * array_length));
  CK(cudaMemcpy(d_prev, h_in, sizeof(float) * M, cudaMemcpyHostToDevice));
  const int N = static_cast<int>(args.integer("N", 20000));
  const float F = static_cast<float>(args.num("F", 0));
  const float h = static_cast<float>(args.num("h", 0.5));
  const float s = static_cast<float>(args.num("s", 0));
  const float slope = static_cast<float>(args.num("slope", 0));
  const int gen = static_cast<int>(args.integer("gen", 1));
  int2 seed;
  seed.x = static_cast<int>(args.integer("seed1", 0xbeef));
  seed.y = static_cast<int>(args.integer("seed2", 0xdecaf));
  Sim_Model::migration_constant_equal mig;
  if (slope != 0.f) {
    Sim_Model::selection_linear_frequency_dependent sel(slope, s);
    go_fish_details::migration_selection_drift<<<600, 128>>>(d_next, d_prev, d_id, M, array_length, N, mig, sel, F, h,
                                                             seed, 0, 1, gen);
  } else {
    Sim_Model::selection_constant sel(s);
    go_fish_details::migration_selection_drift<<<600, 128>>>(d_next, d_prev, d_id, M, array_length, N, mig, sel, F, h,
                                                             seed, 0, 1, gen);
  }
  CK(cudaGetLastError());
  std::vector<float> h_out(M);
  CK(cudaMemcpy(h_out.data(), d_next, sizeof(float) * M, cudaMemcpyDeviceToHost));
  spit(out, h_out.data(), sizeof(float) * M);
  return 0;
}

// draws input: int32 n, then n records {int32 kind (0 binom1, 1 pois1), float mean, float var, float N,
// int32 seed1, int32 seed2, int32 k, int32 step, int32 pop}; output int32 per record
struct DrawRec { int kind; float mean, var, N; int seed1, seed2, k, step, pop; };

__global__ void draws_kernel(const DrawRec* recs, int n, int* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const DrawRec r = recs[i];
  int2 seed;
  seed.x = r.seed1;
  seed.y = r.seed2;
  if (r.kind == 0) out[i] = RNG::ApproxRandBinom1(r.mean, r.var, r.mean / r.N, r.N, seed, r.k, r.step, r.pop);
  else out[i] = RNG::ApproxRandPois1(r.mean, r.var, 0.f, r.N, seed, r.k, r.step, r.pop);
}

static int mode_draws(const char* in, const char* out) {
  std::vector<char> buf = slurp(in);
  int n;
  std::memcpy(&n, buf.data(), 4);
  DrawRec* d_recs;
  int* d_out;
  CK(cudaMalloc(&d_recs, sizeof(DrawRec) * std::max(n, 1)));
  CK(cudaMalloc(&d_out, sizeof(int) * std::max(n, 1)));
  CK(cudaMemcpy(d_recs, buf.data() + 4, sizeof(DrawRec) * n, cudaMemcpyHostToDevice));
  draws_kernel<<<(n + 255) / 256, 256>>>(d_recs, n, d_out);
  CK(cudaGetLastError());
  std::vector<int> h(n);
  CK(cudaMemcpy(h.data(), d_out, sizeof(int) * n, cudaMemcpyDeviceToHost));
  spit(out, h.data(), sizeof(int) * n);
  return 0;
}

// hostrng output: records of Philox blocks and host Poisson draws over a fixed grid of inputs
static int mode_hostrng(const char* out) {
  std::vector<int32_t> o;
  const int seeds[3][2] = {{0xbeef, 0xdecaf}, {static_cast<int>(0xbeeff00d), static_cast<int>(0xdecafbad)}, {0, 0}};
  // Philox: k, step, pop, round grid
  for (auto& sd : seeds) {
    int2 seed;
    seed.x = sd[0];
    seed.y = sd[1];
    for (int k = 0; k < 6; ++k)
      for (int step = 0; step < 4; ++step)
        for (int pop = 0; pop < 3; ++pop) {
          const int kk = k == 5 ? 123456789 : k;
          const int ss = step == 3 ? 20000 : step;
          const uint4 r = RNG::Philox(seed, kk, ss, pop, 0);
          o.insert(o.end(), {sd[0], sd[1], kk, ss, pop, 0, (int32_t)r.x, (int32_t)r.y, (int32_t)r.z, (int32_t)r.w});
        }
  }
  const size_t n_philox = o.size() / 10;
  // host ApproxRandPois1: the new-mutation count path (mean = mu Nc L)
  std::vector<int32_t> p;
  const float means[] = {0.f, 0.5f, 1.f, 2.5f, 5.99f, 6.f, 6.5f, 40.f, 400.f, 4000.f, 200000.f, 1e6f};
  for (auto& sd : seeds) {
    int2 seed;
    seed.x = sd[0];
    seed.y = sd[1];
    for (float mean : means)
      for (int gen = 1; gen <= 40; ++gen)
        for (int pop = 0; pop < 2; ++pop) {
          const int c = RNG::ApproxRandPois1(mean, mean, 0.f, 1e12f, seed, 1, gen, pop);
          int32_t mbits;
          std::memcpy(&mbits, &mean, 4);
          p.insert(p.end(), {sd[0], sd[1], mbits, gen, pop, c});
        }
  }
  FILE* f = std::fopen(out, "wb");
  int32_t hdr[2] = {static_cast<int32_t>(n_philox), static_cast<int32_t>(p.size() / 6)};
  std::fwrite(hdr, 4, 2, f);
  std::fwrite(o.data(), 4, o.size(), f);
  std::fwrite(p.data(), 4, p.size(), f);
  std::fclose(f);
  return 0;
}

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: ref_driver sim <scenario> <out> k=v... | drift1 <in> <out> k=v... | draws <in> <out> | hostrng <out>\n");
    return 2;
  }
  const std::string mode = argv[1];
  if (mode == "hostrng") return mode_hostrng(argv[2]);
  if (mode == "draws" && argc >= 4) return mode_draws(argv[2], argv[3]);
  if (mode == "drift1" && argc >= 4) return mode_drift1(argv[2], argv[3], scn::Args(argc, argv, 4));
  if (mode == "dadi") {  // ref_driver dadi <out.txt> key=value...
    scn::dadi_table(scn::Args(argc, argv, 3), argv[2]);
    return 0;
  }
  if (mode == "sim" && argc >= 4) {
    scn::Args args(argc, argv, 4);
    GO_Fish::allele_trajectories a;
    const auto t0 = std::chrono::steady_clock::now();
    if (!scn::run_scenario(argv[2], a, args)) {
      std::fprintf(stderr, "unknown scenario %s\n", argv[2]);
      return 2;
    }
    cudaDeviceSynchronize();
    const auto t1 = std::chrono::steady_clock::now();
    std::printf("sim_ms %.3f\n", std::chrono::duration<double, std::milli>(t1 - t0).count());
    scn::dump_results(a, args, argv[3]);
    return 0;
  }
  std::fprintf(stderr, "bad arguments\n");
  return 2;
}
