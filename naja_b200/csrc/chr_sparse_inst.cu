// Planning and launch of the sparse-column CHR step kernel (chr_sparse.cuh).
#include "chr_sparse.cuh"

namespace naja {
using namespace chr_detail;

int chr_sparse_plan(int precision, int m, int d, int max_col, double mean_col, int tpb, int max_slots,
                    ChrLaunchConfig* out) {
  if (max_col <= 0) return NAJA_ERR_UNSUPPORTED;
  int threads;
  if (tpb > 0) {
    if (tpb != 32 && tpb != 64 && tpb != 128 && tpb != 256 && tpb != 512) return NAJA_ERR_UNSUPPORTED;
    threads = tpb;
  } else {
    // at most two entries of a mean column per consumer thread: a step's
    // latency is a chain of shared-memory loads, divisions and barriers, and
    // spreading the entries wider shortens it (m = 5200, 416 entries per
    // column, 16 chains: 1.45 us per step with 256 threads, 2.0 us with 128)
    threads = 32;
    while (threads < 512 && mean_col > 2.0 * threads) threads *= 2;
  }
  const bool f64 = precision == NAJA_PREC_FP64;
  const int elt = f64 ? 8 : 4, eb = f64 ? kSpEntryBytes64 : kSpEntryBytes32;
  const int nw = threads / 32;
  // Pair steps through a scratch column where it fits (fewer instructions per
  // step); otherwise by search (no scratch column, m values less).
  int slots = 0;
  bool scatter = true;
  Layout L;
  for (int sc = 1; sc >= 0 && slots == 0; --sc) {
    int s = kMaxSlots;
    if (max_slots > 0 && max_slots < s) s = max_slots;
    L = make_sparse_layout(d, m, elt, eb, max_col, nw, s, sc != 0);
    while (s > 3 && L.total > kSmemBudget) {
      --s;
      L = make_sparse_layout(d, m, elt, eb, max_col, nw, s, sc != 0);
    }
    if (s >= 3 && L.total <= kSmemBudget) {
      slots = s;
      scatter = sc != 0;
    }
  }
  if (slots == 0) return NAJA_ERR_UNSUPPORTED;
  out->threads = threads;
  out->rows = 0;
  out->slots = slots;
  out->smem = L.total;
  out->cluster = 1;
  out->slice_lda = 0;
  out->max_col = max_col;
  out->pair_scatter = scatter ? 1 : 0;
  out->uniform = 0;
  return NAJA_OK;
}

int chr_sparse_launch(int precision, const ChrArgs& a, const SpArgs& sp, int nchains, const ChrLaunchConfig& cfg,
                      cudaStream_t stream) {
  if (precision == NAJA_PREC_FP64) return launch_sparse_nw<double>(a, sp, nchains, cfg, stream);
  return launch_sparse_nw<float>(a, sp, nchains, cfg, stream);
}

int chr_sparse_batch_plan(int m_max, int d, BatchConfig* cfg) {
  const int nt = cfg->threads;
  if (nt != 64 && nt != 128 && nt != 256) return NAJA_ERR_INVALID_ARGUMENT;
  if (cfg->slots < 3 || cfg->slots > kMaxSlots) return NAJA_ERR_INVALID_ARGUMENT;
  if (cfg->max_col <= 0) return NAJA_ERR_UNSUPPORTED;
  const Layout L = make_sparse_layout(d, m_max, 4, kSpEntryBytes32, cfg->max_col, nt / 32, cfg->slots);
  // the kernel also holds one ChrArgs and one SpArgs in static shared memory
  if (L.total + align_up(sizeof(ChrArgs) + sizeof(SpArgs), 128) > kSmemBudget) return NAJA_ERR_UNSUPPORTED;
  cfg->rows = 0;
  cfg->lda_max = m_max;
  cfg->smem = L.total;
  return NAJA_OK;
}

int chr_sparse_batch_dispatch(const ChrArgs* base, const ModelDesc* models, const int* im, const int* ic, int nitems,
                              const BatchConfig& cfg, cudaStream_t stream, int* occ_out) {
  switch (cfg.threads) {
    case 64: return batch_sparse_one<2>(base, models, im, ic, nitems, cfg, stream, occ_out);
    case 128: return batch_sparse_one<4>(base, models, im, ic, nitems, cfg, stream, occ_out);
    case 256: return batch_sparse_one<8>(base, models, im, ic, nitems, cfg, stream, occ_out);
    default: return NAJA_ERR_UNSUPPORTED;
  }
}
}  // namespace naja
