/*
 * naja_chr.h -- C ABI of the B200-native coordinate hit-and-run (CHR)
 * sampler (libnaja_b200.so).
 *
 * Plain C: pointers, sizes, POD structs, an integer status and a
 * thread-local last-error string.  Every pointer argument may be host or
 * device memory (the library inspects it); device pointers must live on the
 * device the call runs on (device memory of another GPU is rejected with
 * NAJA_ERR_INVALID_ARGUMENT; managed memory is accepted).  Calls are
 * asynchronous on the given stream
 * unless a host pointer forces a synchronous copy back.  Matrices are
 * column-major with an explicit leading dimension, as in the reference
 * (IDX2C(i,j,ld) = j*ld + i, src/gpu/helper.h:9 of quothbonney/naja).
 *
 * The sample matrix layout is the reference's: sample s of chain c is
 * column c + s*nchains of a d x (nchains*nspc) column-major matrix
 * (src/gpu/chr.cu:284,460), which is byte-identical to the row-major
 * (nchains*nspc, d) array that `samples.npy` stores (src/npy.h:96-141).
 */
#ifndef NAJA_CHR_H
#define NAJA_CHR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ statuses */
#define NAJA_OK 0
#define NAJA_ERR_INVALID_ARGUMENT 1 /* reference: std::invalid_argument */
#define NAJA_ERR_RUNTIME 2          /* reference: std::runtime_error    */
#define NAJA_ERR_CUDA 3             /* a CUDA runtime call failed         */
#define NAJA_ERR_NO_MEMORY 4
#define NAJA_ERR_UNSUPPORTED 5      /* shape outside what the kernels take */
#define NAJA_ERR_DEVICE 6           /* the kernel reported an error word  */

/* ------------------------------------------------------------- options */
#define NAJA_PREC_FP32 0 /* FP32 A and slack, FP64 x, FP64 recompute every K */
#define NAJA_PREC_FP64 1 /* FP64 throughout (the reference's arithmetic)      */

#define NAJA_RNG_PHILOX 0  /* counter-based Philox4x32-10 keyed (seed, chain, step) */
#define NAJA_RNG_REF_MRG 1 /* cuRAND MRG32k3a, curand_init(seed, chain, 0), reference draw order */

#define NAJA_DTYPE_F32 0
#define NAJA_DTYPE_F64 1

#define NAJA_SPARSE_AUTO 0    /* compressed columns when A is at most 1/4 nonzero and they fit */
#define NAJA_SPARSE_DENSE 1   /* every row of A every step                                     */
#define NAJA_SPARSE_COLUMNS 2 /* only the nonzero rows of the step's column(s)                 */

#define NAJA_BACKMAP_FP64 0    /* FP64 SIMT GEMM (reference arithmetic)          */
#define NAJA_BACKMAP_BF16X3 1  /* split-BF16 on tcgen05, FP32 accumulate          */
#define NAJA_BACKMAP_TF32X3 2  /* 3xTF32 on tcgen05, FP32 accumulate              */

typedef struct naja_polytope naja_polytope; /* device-resident A (FP64 + FP32), b */

/* Sampling parameters.  Field meanings follow the reference's
 * CoordinateHitAndRun arguments (src/gpu/gpusamplers.h:30-46). */
typedef struct naja_chr_params {
    int nspc;              /* samples per chain                                  */
    int thinning;          /* steps between saved samples (> 0)                  */
    int nchains;           /* chains in this call                                */
    int tpb;               /* consumer threads per chain; <= 0 = automatic        */
    unsigned long long seed;
    double pair_prob;      /* probability of a pair direction                    */
    int resync_interval;   /* slack = b - A x recomputed in FP64 every K steps   */
    double ksparse_prob;
    int ksparse_k;
    int pair_mode;         /* 1 = (e_i - e_j)/sqrt 2, 2 = Jacobi schedule         */
    const int* pair_i;     /* pair schedule (pair_mode 2), n_pairs entries each  */
    const int* pair_j;
    const double* pair_c;
    const double* pair_s;
    int n_pairs;
    int precision;         /* NAJA_PREC_*                                        */
    int rng;               /* NAJA_RNG_*                                         */
    int out_dtype;         /* NAJA_DTYPE_* of the samples buffer                 */
    int chain_base;        /* global index of chain 0 (RNG stream, output row)   */
    int out_nchains;       /* chains per output row block (>= chain_base+nchains); 0 = nchains */
    long long step_offset; /* Philox: continue chains from this step             */
    int max_slots;         /* staged-column ring depth cap; 0 = automatic        */
    void* rng_state;       /* nullable MRG32k3a states (naja_mrg_state_bytes each), in/out */
    unsigned long long* wait_cycles; /* nullable device buffer, 4 per chain: consumer wait for columns,
                                        producer wait for slots, consumer loop, producer loop (SM cycles) */
    int cluster;           /* CTAs per chain: 0 = automatic (one CTA per chain), 1 = one CTA per
                              chain, 2..8 = a chain's rows split over a thread-block cluster of that
                              many CTAs (128 or 256 threads each); results are identical for every value */
    int sparse;            /* NAJA_SPARSE_*: which step kernel walks A.  The compressed-column kernel
                              takes ksparse_prob = 0 and cluster <= 1, and tpb 0 (automatic), 32, 64,
                              128, 256 or 512 when forced (automatic selection needs tpb 0); results
                              are identical for every value */
    void* slack_final;     /* nullable, host or device: each chain's slack b - A x after its last step,
                              nchains x m values (FP32 tier: float, FP64 tier: double), chain-major;
                              one CTA per chain only.  The FP32 tier's drift from the exact slack is
                              this minus b - A x_final in FP64 (the reference's resync hook,
                              src/gpu/chr.cu:384-395, bounds it every resync_interval steps) */
} naja_chr_params;

/* Fills `p` with the reference's defaults (gpusamplers.h:30-46): tpb auto,
 * seed 0, pair_prob 0, resync 0, ksparse_prob 0, ksparse_k 8, pair_mode 1,
 * FP32 tier, Philox, float output. */
void naja_chr_params_default(naja_chr_params* p);

/* ------------------------------------------------------------ polytope */

/* Uploads the polytope A y <= b (A m x d column-major, leading dimension
 * lda >= m) to `device`, keeping an FP64 copy and an FP32 copy, each with
 * a leading dimension padded to a multiple of 32.  Replaces the DMatrix /
 * DVector uploads of src/engine/job_sampling.cu:258-259 (quothbonney/naja). */
int naja_polytope_create(int device, int m, int d, const double* A, int lda, const double* b,
                         naja_polytope** out);
int naja_polytope_destroy(naja_polytope* P);
int naja_polytope_shape(const naja_polytope* P, int* m, int* d);
/* Waits for all work on the polytope's device and reports (then clears)
 * an error word a kernel set since the last check: a bounded wait that
 * expired, or a pair index outside [0, d).  Calls whose buffers are all on
 * the device return before the kernel ends; this is how their device-side
 * errors surface.  Calls with a host buffer check it themselves. */
int naja_polytope_check(const naja_polytope* P);

/* ------------------------------------------------------------ sampling */

/* Runs params->nchains chains from X0 (d x nchains, leading dimension ldx)
 * and writes params->nspc samples per chain into `samples`, laid out as
 * described at the top of this file (rows of d values of out_dtype).
 * X_final (nullable) receives the last state of every chain (the
 * reference's persist_state, src/gpu/chr.cu:485-489).  Replaces
 * naja::gpu::CoordinateHitAndRun (src/gpu/chr.cu:13-70) and
 * launchChrKernel (src/gpu/chr.cu:498-553). */
int naja_chr_run(const naja_polytope* P, const naja_chr_params* params, const double* X0, int ldx,
                 void* samples, double* X_final, void* stream);

/* The step kernel naja_chr_run would launch for these parameters:
 * *sparse_kernel = 1 for the compressed-column kernel (only the nonzero rows
 * of each step's column), 0 for the dense one; its consumer threads per
 * chain, staged-column slots and dynamic shared memory.  Any output pointer
 * may be null.  The first call for a polytope that may take the compressed
 * columns builds them (device memory held until naja_polytope_destroy).  No
 * counterpart in the reference (its launchChrKernel, src/gpu/chr.cu:498-553,
 * has one kernel). */
int naja_chr_kernel_choice(const naja_polytope* P, const naja_chr_params* params, int* sparse_kernel,
                           int* threads, int* slots, size_t* smem);

/* ------------------------------------------------------------- batches */

/* Launch shape of a batched run (chosen by the autotuner in
 * naja_b200/autotune.py, or by hand). */
typedef struct naja_batch_config {
    int threads;      /* consumer threads per chain: 128, 256 or 512            */
    int slots;        /* staged-column ring depth 2..8, 0 = direct column reads */
    int slack_smem;   /* 1: slack in shared memory (several chains per SM)      */
    int ctas_per_sm;  /* resident chains per SM, 0 = as many as fit             */
    int sparse;       /* 1: compressed-column kernel (threads 64, 128 or 256 consumer
                         threads, slots 3..8, slack_smem ignored); same samples       */
} naja_batch_config;

/* Runs params->nchains chains of each of `nmodels` polytopes (the same d)
 * in ONE persistent launch.  Model k uses seed params->seed + k*seed_stride
 * and its chains are numbered 0..nchains-1, so it draws exactly the streams a
 * standalone naja_chr_run of that model with that seed draws.  X0s[k]
 * (d x nchains, leading dimension ldx) and samples[k] ((nspc*nchains) x d,
 * params->out_dtype) are device pointers; X_finals (nullable array, entries
 * nullable) receives each model's last states like naja_chr_run's X_final, so
 * a later launch with params->step_offset continues the chains.  FP32 tier.
 * This replaces the reference's model-by-model bulk loop
 * (src/engine/job_bulk.cpp:115-189), which launches one small
 * CoordinateHitAndRun per model. */
int naja_chr_run_batched(int nmodels, const naja_polytope* const* models, const naja_chr_params* params,
                         const double* const* X0s, int ldx, void* const* samples, double* const* X_finals,
                         unsigned long long seed_stride, const naja_batch_config* config, void* stream);
/* Resident chains per SM that `config` allows for these models (0 if none). */
int naja_batch_occupancy(int nmodels, const naja_polytope* const* models, const naja_batch_config* config,
                         int* ctas_per_sm);
/* The same batched launch captured once into a CUDA graph (*graph receives
 * an opaque handle that keeps the launch's descriptors alive); replay it
 * with naja_graph_launch, check it with naja_graph_check, release it with
 * naja_graph_destroy. */
int naja_chr_capture_batched(int nmodels, const naja_polytope* const* models, const naja_chr_params* params,
                             const double* const* X0s, int ldx, void* const* samples, double* const* X_finals,
                             unsigned long long seed_stride, const naja_batch_config* config, void** graph);
int naja_graph_launch(void* graph, void* stream);
int naja_graph_check(void* graph);
int naja_graph_destroy(void* graph);

/* ------------------------------------------------------------- backmap */

/* V = T * Y + shift * 1^T.  T is n x d column-major (leading dimension ldt),
 * Y holds N samples of d values (row-major N x d, y_dtype), V receives N
 * rows of n values (v_dtype).  Replaces backmap_into
 * (src/gpu/backmap.cu:20-48). */
int naja_backmap(int n, int d, long long N, const double* T, int ldt, const double* shift,
                 const void* Y, int y_dtype, void* V, int v_dtype, int mode, void* stream);

/* The same tensor-core backmap (modes NAJA_BACKMAP_BF16X3 / TF32X3 only)
 * without allocating device memory: for callers that must not allocate at
 * the point of the call, such as a service that reserves its device-memory
 * budget up front and forbids allocations on its request path, or a host
 * framework whose allocator owns the device.  No counterpart in the
 * reference.  T, shift, Y and V must be device memory.  The split operands
 * use a 64 MiB array that every device loading the library holds until
 * process exit; a call needing more (about 1 KiB + 2 * N * dp * e +
 * 2 * n * dp * e bytes, dp = d rounded up to 64, e = 2 for BF16X3 and 4
 * for TF32X3) is rejected with NAJA_ERR_INVALID_ARGUMENT: split N across
 * calls.  The first call on a device does the set-up: it looks the array's
 * device address up with that device current and caches it; make that first
 * call before any stream capture, and do not call this entry point again on
 * a device after cudaDeviceReset of it.  All calls on a device share the
 * array: calls whose work overlaps on the GPU (other streams, other host
 * threads) race, so the caller serialises them.  Synchronises `stream` to
 * read its error word. */
int naja_backmap_noalloc(int n, int d, long long N, const double* T, int ldt, const double* shift,
                         const void* Y, int y_dtype, void* V, int v_dtype, int mode, void* stream);

/* ------------------------------------------------------------ pipeline */

/* naja_chr_run followed by naja_backmap as one job, overlapped: the chains
 * run in chunks of chunk_nspc samples (<= 0: automatic, whole
 * lcm(resync_interval, thinning) periods of about 65,536 steps) on one
 * stream while the previous chunk's backmap V = T y + shift and the copies of
 * its rows run on another.  V receives nspc*nchains rows of n values
 * (v_dtype) in the sample order of naja_chr_run; `samples` (nullable) also
 * receives the samples themselves (params->out_dtype).  V, samples, X0,
 * X_final, T and shift may be host or device memory; pinned host memory
 * lets the copies overlap the sampling.  Chunking needs the Philox streams
 * and resync_interval > 0 (a chunk starts where one run recomputes the slack
 * anyway, so the samples are those of one naja_chr_run, bit for bit);
 * otherwise the job runs as one chunk.  chain_base must be 0 and out_nchains
 * 0 or nchains.  Synchronises `stream` and reports device-side errors before
 * returning.  Replaces the sample-then-backmap-then-copy sequence of
 * run_sampling_job (src/engine/job_sampling.cu:300-385) around
 * CoordinateHitAndRunBackmap (src/gpu/chr.cu:72-99). */
int naja_chr_run_backmapped(const naja_polytope* P, const naja_chr_params* params, const double* X0, int ldx,
                            int n, const double* T, int ldt, const double* shift, int mode, void* V, int v_dtype,
                            void* samples, double* X_final, int chunk_nspc, void* stream);

/* ------------------------------------------------------------ validate */

/* Geyer ESS per (dim, chain) and split-R-hat per dim of an (N, dim)
 * row-major float32 sample matrix (src/validate/mcmc.cpp:91-194).
 * layout 0 = the reference's windows (chain c = rows [c*spc, (c+1)*spc)),
 * layout 1 = chains interleaved as the sampler writes them (row r belongs
 * to chain r % nchains).  ess: dim*nchains values (dim-major), rhat: dim;
 * either may be null (that metric is skipped).  ESS takes at most 49,152
 * samples per chain (a series is held on chip); R-hat has no such limit. */
int naja_validate(const float* samples, long long N, int dim, int nchains, int layout, double* ess,
                  double* rhat, void* stream);

/* --------------------------------------------------------------- misc */

/* Thread-local description of the last failure on this thread. */
const char* naja_last_error(void);
/* Size of one MRG32k3a state for naja_chr_params.rng_state. */
size_t naja_mrg_state_bytes(void);
/* Seeds `nchains` MRG32k3a states (device buffer, naja_mrg_state_bytes()
 * each) with curand_init(seed, chain_base + c, 0), the reference's seeding
 * (src/gpu/chr.cu:555-560).  A run given them in rng_state continues each
 * stream and stores it back, as the reference's streamed mode carries its
 * PRNGState across chunks (src/gpu/chr.cu:154-201). */
int naja_mrg_init_states(int device, unsigned long long seed, int chain_base, int nchains, void* states);
/* Test hook: the first `count` uniforms that cuRAND's curand_uniform_double
 * returns for curand_init(seed, chain_base + c, 0), c < nchains, written to
 * tape[c*count + i].  This is the reference's per-chain stream
 * (src/gpu/chr.cu:555-560). */
int naja_mrg_tape(int device, unsigned long long seed, int chain_base, int nchains, long long count, double* tape);
const char* naja_version(void);

#ifdef __cplusplus
}
#endif
#endif /* NAJA_CHR_H */
