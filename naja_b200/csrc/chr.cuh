// Host-visible description of one CHR launch and the launcher entry point.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace naja {

enum StepKind : int { kCoord = 0, kPair = 1, kKSparse = 2 };

// Everything the step kernel needs, passed by value.  Matrices are
// column-major with a padded leading dimension `lda` (a multiple of 32
// elements, so every column starts on a 128-byte boundary).
struct ChrArgs {
  const float* A32;   // FP32 copy of A (FP32 tier hot path)
  const double* A64;  // FP64 A (FP64 tier hot path; init and recompute)
  int lda;
  const double* b;    // m
  int m, d;
  const double* X0;   // d x nchains, leading dimension ldx (column = local chain)
  int ldx;
  double* X_final;    // nullable, same layout as X0
  void* samples;      // (nspc * out_nchains) x d row-major, row = s*out_nchains + chain_base + chain
  int out_f64;        // 1: samples are double, 0: float
  int out_nchains;
  int chain_base;     // global index of this launch's chain 0 (RNG key and output row)
  int nspc, thinning;
  long long step_offset;  // Philox step counter offset (continuation of a chain)
  unsigned long long seed;
  double pair_prob, ksparse_prob;
  int ksparse_k, pair_mode;
  const int* pair_i;
  const int* pair_j;
  const double* pair_c;
  const double* pair_s;
  int n_pairs;
  int resync;  // FP64 slack recompute every `resync` steps (t = 0 included), 0 = never
  int rng;     // 0 = Philox4x32-10, 1 = cuRAND MRG32k3a in the reference's draw order
  void* rng_state;  // nullable: curandStateMRG32k3a[nchains] loaded at start, stored at exit
  int* err;         // device error word
  unsigned long long timeout_ns;
  // Nullable instrumentation, 4 words per chain: consumer cycles waiting for
  // staged columns, producer cycles waiting for free slots, consumer cycles
  // in the step loop, producer cycles in its loop.
  unsigned long long* wait_cycles;
  // Nullable: receives each chain's slack b - A x after its last step
  // (nchains x m values of the tier's type, chain-major).
  void* slack_final;
  // Step range of this launch within the chains' run: steps t_first ..
  // t_first + steps - 1 (steps 0: nspc * thinning steps from t_first 0).
  // Saved samples (every thinning-th global step, output row = global step /
  // thinning), Philox steps (step_offset + global step) and the resync
  // schedule (global multiples of resync) follow the global step index.
  long long t_first, steps;
  // Nullable: each chain's slack at step t_first (the tier's type,
  // chain-major, nchains x m), read instead of the initial FP64 recompute.
  const void* slack_in;
};

struct ChrLaunchConfig {
  int threads;    // consumer threads per CTA (multiple of 32)
  int rows;       // row chunks held per consumer warp (template capacity)
  int slots;      // staged-column ring depth (0 = read columns straight from L2/HBM)
  size_t smem;    // dynamic shared memory bytes
  int cluster;    // CTAs per chain (thread-block cluster); 1 = one CTA per chain
  int slice_lda;  // rows a CTA's column slot holds (cluster > 1), padded to 32
  int max_col;    // sparse-column kernel: entries of the longest compressed column
  int pair_scatter;  // sparse-column kernel: 1 = pair steps through a scratch column, 0 = by search
  int uniform;       // dense single-CTA kernel: 1 = every warp runs `rows` chunks, the rows past m
                     // repeating the last V rows (needs m % V == 0); 0 = chunks as rows allow
};

// Compressed columns of A for the sparse-column kernel, in the tier's
// precision: column j's entries (value, row) are cols[col_start[j],
// col_start[j + 1]), rows ascending, padded with (0, m) entries to a
// 16-byte multiple and to at least one 16-byte group.  row_ent holds the
// FP64 A by rows for the FP64 slack recompute: row r's (value, column)
// entries (16 bytes each, columns ascending) are row_ent[row_start[r],
// row_start[r + 1]), padded with (0, 0) entries to a multiple of
// kSpRowGroup.
struct SpArgs {
  const void* cols;
  const int* col_start;
  const int* row_start;
  const void* row_ent;
};
constexpr int kSpRowGroup = 16;

// Entry sizes of the compressed columns: (float value, int row) and
// (double value, int row, padding).
constexpr int kSpEntryBytes32 = 8;
constexpr int kSpEntryBytes64 = 16;

// Plans the sparse-column kernel: `tpb` consumer threads per chain (32, 64,
// 128, 256 or 512; <= 0 = automatic from the mean column length `mean_col`),
// `max_col` entries per staged column.  Returns 0 or a naja status code
// (NAJA_ERR_UNSUPPORTED when the chain's state does not fit on chip).
int chr_sparse_plan(int precision, int m, int d, int max_col, double mean_col, int tpb, int max_slots,
                    ChrLaunchConfig* out);
int chr_sparse_launch(int precision, const ChrArgs& args, const SpArgs& sp, int nchains, const ChrLaunchConfig& cfg,
                      cudaStream_t stream);

// Picks a launch configuration.  `tpb` > 0 forces the consumer thread count
// (one of the reference's 32, 64, 128, 256, 512, 1024; 1024 runs as 992 consumer
// threads plus the producer warp); `max_slots` > 0 caps the ring.
// Returns 0 or a naja status code.
// `cluster`: CTAs per chain, 0 = automatic (one CTA per chain), 1 = one CTA
// per chain, 2..8 = a thread-block cluster of that many CTAs per chain;
// `nchains` and `sms` are the launch's chains and the device's SMs.
int chr_plan(int precision, int m, int d, int lda, int tpb, int max_slots, int nchains, int cluster, int sms,
             ChrLaunchConfig* out);

// Launches nchains independent chains (one CTA each) on `stream`.
int chr_launch(int precision, const ChrArgs& args, int nchains, const ChrLaunchConfig& cfg, cudaStream_t stream);

// Runs the same chains as one chr_launch with args.resync = K > 0, as
// segments of K steps: before each segment one kernel over the whole GPU
// recomputes every chain's slack b - A64 x in FP64 (each row's fma chain
// over the columns in order, as the step kernel's recompute), and the
// segment's step kernel starts from it (slack_in) with no recompute of its
// own.  Samples, final positions, final slack and RNG streams are those of
// the single launch, bit for bit; the recompute, which the step kernel
// does on the chain's one SM, reads A64 on every SM instead.  Returns the
// number of kernel launches through `launches` (nullable).  `sp` non-null:
// the segments run the compressed-column kernel (chr_sparse_launch) with
// those columns; its own recompute skips the zero terms of a row, which can
// change only the sign of a zero sum, so against the dense recompute here it
// can differ at most in the sign of a zero slack (where b is -0).
int chr_run_segmented(int precision, const ChrArgs& args, int nchains, const ChrLaunchConfig& cfg,
                      cudaStream_t stream, long long* launches, const SpArgs* sp = nullptr);

// Steps of one launch (host side of the kernels' launch_steps).
inline long long launch_steps_host(const ChrArgs& a) {
  return a.steps > 0 ? a.steps : static_cast<long long>(a.nspc) * a.thinning;
}

// True where chr_run_segmented pays for its per-segment launches: a
// single-CTA run (either step kernel) with a recompute interval shorter than
// the run and an A64 large enough (m d >= kSegmentMinCells) that
// recomputing from one SM costs more than a segment boundary.
constexpr long long kSegmentMinCells = 1LL << 19;
inline bool chr_use_segments(long long m, long long d, int resync, long long total_steps, int cluster,
                             bool instrumented) {
  return resync > 0 && total_steps > resync && cluster <= 1 && !instrumented && m * d >= kSegmentMinCells;
}

// Records the first `count` uniforms of curand_init(seed, chain_base + c, 0)
// MRG32k3a states, c < nchains, into tape[c * count + i] (device memory).
int mrg_tape(unsigned long long seed, int chain_base, int nchains, long count, double* tape, cudaStream_t stream);

// ---------------------------------------------------------------- batches
// One model of a batched run: its polytope (padded column-major A, b), start
// points and outputs.  Every model of a batch shares d and the step settings
// of the launch's ChrArgs; chains of a model are numbered 0..nchains-1 and
// draw the streams a standalone run of that model with `seed` draws.
struct ModelDesc {
  const float* A32;
  const double* A64;
  int lda;
  int m;
  const double* b;
  const double* X0;  // d x nchains, leading dimension ldx
  int ldx;
  void* samples;     // (nspc * nchains) x d
  double* X_final;   // nullable
  unsigned long long seed;
  SpArgs sp;         // compressed columns (FP32 tier) for the compressed-column batch
};

struct BatchConfig {
  int threads;      // consumer threads per chain
  int rows;         // row chunks per consumer warp (template capacity)
  int slots;        // ring depth, 0 = direct column reads
  int slack_smem;   // 1: slack in shared memory, 0: in registers
  int ctas_per_sm;  // requested resident chains per SM (0 = as many as fit)
  int lda_max;      // dense: largest padded leading dimension; compressed: largest m
  size_t smem;
  int sparse;       // 1: the compressed-column kernel (threads 64, 128 or 256)
  int max_col;      // compressed: entries of the longest column of any model
};

// Chunk-per-warp capacities instantiated for the batched kernel, per
// (consumer threads, slack store), ascending; 0 ends a list.
inline const int* batch_chunk_capacities(int threads, bool slack_smem) {
  static const int k512s[] = {4, 8, 0}, k512r[] = {4, 8, 0};
  static const int k256s[] = {4, 8, 16, 0}, k256r[] = {6, 8, 12, 0};
  static const int k128s[] = {12, 16, 0}, k128r[] = {12, 16, 0};
  if (threads == 512) return slack_smem ? k512s : k512r;
  if (threads == 256) return slack_smem ? k256s : k256r;
  if (threads == 128) return slack_smem ? k128s : k128r;
  return nullptr;
}

// Validates a batch configuration for models of at most m_max rows and fills
// rows / smem.  Returns 0 or a naja status code.
int chr_batch_plan(int m_max, int d, int lda_max, BatchConfig* cfg);
// The same for the compressed-column kernel (cfg->sparse = 1, cfg->max_col
// set), with its dispatch.
int chr_sparse_batch_plan(int m_max, int d, BatchConfig* cfg);
int chr_sparse_batch_dispatch(const ChrArgs* base, const ModelDesc* models, const int* im, const int* ic, int nitems,
                              const BatchConfig& cfg, cudaStream_t stream, int* occ_out);
// Resident CTAs per SM the configuration allows (occupancy calculator).
int chr_batch_occupancy(const BatchConfig& cfg, int* ctas_per_sm);
// Persistent launch over nitems (model, chain) work items (device arrays).
int chr_batch_launch(const ChrArgs& base, const ModelDesc* models, const int* item_model, const int* item_chain,
                     int nitems, const BatchConfig& cfg, cudaStream_t stream);

// Seeds nchains MRG32k3a states with curand_init(seed, chain_base + c, 0).
int mrg_init_states(unsigned long long seed, int chain_base, int nchains, void* states, cudaStream_t stream);

// Size in bytes of one chain's MRG32k3a state (for rng_state buffers).
size_t mrg_state_bytes();

}  // namespace naja
