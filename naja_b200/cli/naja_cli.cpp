// `naja` command line: the sampling and validate commands of quothbonney/naja
// over this project's C ABI (include/naja_chr.h).
//
//   naja sample run --model-dir DIR --out-root DIR --n-chains K --n-samples S [flags]
//       src/cli/sample/cmd_run.cpp:44-237 (flags, checks, phase lines) and
//       src/engine/job_sampling.cu:82-445 (the job): model-directory contract
//       (src/pipeline/model_contract.cpp:56-84), run directory
//       <out-root>/<model>_<YYYYMMDD>_<NNN> (model_contract.cpp:217-230),
//       config_generated.txt, run_manifest.json (src/pipeline/run_manifest.cpp:
//       74-143), samples.npy as (n_samples, dim) float32 C order with the
//       reference's header padding (src/npy.h:96-141), profile.json
//       (src/engine/profile.h:28-66), config_used.txt (job_sampling.cu:34-60).
//       Thinning defaults to max(d/6, 1) and the seed to the reference's hash
//       of model name, model directory and GPU (job_sampling.cu:237-254).
//       Rounding inputs (src/rounding/plan.cpp:12-62): --pair-schedule FILE
//       (i,j,c,s CSV) or --iter-rounding-passes P --iter-rounding-warmup W (a
//       warm-up estimate, src/rounding/runtime_warmup.cpp:16-108) select
//       Jacobi-rotated pair steps; --affine-hull-tol samples the affine hull of
//       the rows tight at the start (job_sampling.cu:196-235, T and shift
//       composed as in :299-303); --extra-constraint-eps / --constraint-eps
//       relax rows as job_sampling.cu:138-146 does.
//   naja sample bulk --models-root DIR --model-list FILE --out-root DIR --name RUN --gpus 0,1,...
//       src/cli/sample/cmd_bulk.cpp:20-163 and src/engine/job_bulk.cpp:115-267:
//       every listed model sampled as `sample run` would, one host thread per
//       GPU id, --skip-existing / --resume-from, bulk_summary.csv.
//   naja sample calibrate-rounding --models-root DIR --model-list FILE --out F.csv
//       src/cli/sample/cmd_calibrate_rounding.cpp:24-195: one pair schedule
//       from warm-up moments pooled over a list of models.
//   naja validate --samples F.npy [--model-dir DIR] [--n-chains 4]
//       src/cli/validate_cli.cpp:49-296: ESS / split-R-hat (naja_validate, the
//       reference's chain windows), bounds compliance of v = T y + shift
//       against the GEM bounds (src/validate/bounds_check.cpp:8-39), the
//       one-line status to stderr and the JSON report to stdout.
//
// The one flag value the reference accepts for a feature this project leaves
// out (--start-policy cube_center, a Gurobi LP) is rejected with a usage
// error instead of being ignored.
#include <dirent.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <charconv>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/naja/rounding.hpp"
#include "../../include/naja_chr.h"

namespace {

// ------------------------------------------------------------------ files
bool path_exists(const std::string& p) {
  struct stat st;
  return stat(p.c_str(), &st) == 0;
}
bool is_directory(const std::string& p) {
  struct stat st;
  return stat(p.c_str(), &st) == 0 && S_ISDIR(st.st_mode);
}
void ensure_dir(const std::string& p) {
  if (p.empty() || is_directory(p)) return;
  const auto slash = p.find_last_of('/');
  if (slash != std::string::npos && slash > 0) ensure_dir(p.substr(0, slash));
  if (mkdir(p.c_str(), 0755) != 0 && !is_directory(p)) throw std::runtime_error("cannot create directory: " + p);
}
std::string absolute(const std::string& p) {
  if (p.empty()) return p;
  char buf[4096];
  if (realpath(p.c_str(), buf)) return buf;
  if (p[0] == '/') return p;
  if (getcwd(buf, sizeof(buf))) return std::string(buf) + "/" + p;
  return p;
}
std::string stamp(const char* fmt) {
  const std::time_t now = std::time(nullptr);
  char b[64];
  std::strftime(b, sizeof(b), fmt, std::localtime(&now));
  return b;
}
std::string self_path() {
  char buf[4096];
  const ssize_t n = readlink("/proc/self/exe", buf, sizeof(buf) - 1);
  if (n <= 0) return "naja";
  buf[n] = 0;
  return buf;
}

// CSV of numbers; rows separated by newlines, values by commas.  The text is
// split into line-aligned blocks parsed in parallel (std::from_chars), one
// thread per block -- the reference parses cell by cell with std::stod on one
// thread (src/csv_loader.h:12-49), which dominates loading at genome scale.
struct Csv {
  int rows = 0, cols = 0;
  std::vector<double> v;  // row-major
};
namespace csv_detail {
struct Block {
  std::vector<double> v;
  std::vector<int> row_cols;
  std::string error;
};
inline bool blank(char ch) { return ch == ' ' || ch == '\t' || ch == '\r'; }
void parse_block(const char* p, const char* end, Block& out) {
  while (p < end) {
    const char* eol = static_cast<const char*>(std::memchr(p, '\n', end - p));
    if (!eol) eol = end;
    const char* q = p;
    while (q < eol && (blank(*q) || *q == '\f' || *q == '\v')) ++q;
    if (q < eol) {
      int cols = 0;
      while (q < eol) {
        if (*q == '+') ++q;
        double x = 0.0;
        const auto r = std::from_chars(q, eol, x);
        if (r.ec != std::errc() || r.ptr == q) {
          out.error = "bad number";
          return;
        }
        out.v.push_back(x);
        ++cols;
        q = r.ptr;
        while (q < eol && blank(*q)) ++q;
        if (q < eol && *q == ',') ++q;
        while (q < eol && blank(*q)) ++q;
      }
      out.row_cols.push_back(cols);
    }
    p = eol + 1;
  }
}
}  // namespace csv_detail
Csv load_csv(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f.is_open()) throw std::runtime_error("cannot open file: " + path);
  std::string text((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
  const char* beg = text.data();
  const char* end = beg + text.size();
  const size_t hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t nblk = std::max<size_t>(1, std::min<size_t>(hw, text.size() / (1 << 20)));
  std::vector<const char*> cut(nblk + 1, end);
  cut[0] = beg;
  for (size_t k = 1; k < nblk; ++k) {
    const char* at = beg + text.size() * k / nblk;
    const char* nl = static_cast<const char*>(std::memchr(at, '\n', end - at));
    cut[k] = nl ? nl + 1 : end;
    if (cut[k] < cut[k - 1]) cut[k] = cut[k - 1];
  }
  std::vector<csv_detail::Block> blocks(nblk);
  std::vector<std::thread> pool;
  for (size_t k = 1; k < nblk; ++k)
    pool.emplace_back([&, k] { csv_detail::parse_block(cut[k], cut[k + 1], blocks[k]); });
  csv_detail::parse_block(cut[0], cut[1], blocks[0]);
  for (auto& t : pool) t.join();
  Csv c;
  size_t total = 0;
  for (const auto& b : blocks) total += b.v.size();
  c.v.reserve(total);
  for (const auto& b : blocks) {
    if (!b.error.empty())
      throw std::runtime_error(b.error + " in " + path + " near row " + std::to_string(c.rows + b.row_cols.size() + 1));
    for (int cols : b.row_cols) {
      if (c.rows == 0) c.cols = cols;
      else if (cols != c.cols) throw std::runtime_error("ragged csv: " + path);
      ++c.rows;
    }
    c.v.insert(c.v.end(), b.v.begin(), b.v.end());
  }
  if (c.rows == 0) throw std::runtime_error("empty csv: " + path);
  return c;
}
// Column-major copy (rows x cols, ld = rows).
std::vector<double> colmajor(const Csv& c) {
  std::vector<double> out(static_cast<size_t>(c.rows) * c.cols);
  for (int r = 0; r < c.rows; ++r)
    for (int k = 0; k < c.cols; ++k) out[static_cast<size_t>(k) * c.rows + r] = c.v[static_cast<size_t>(r) * c.cols + k];
  return out;
}

// One npy array, header padded as src/npy.h:56-79 / 96-141 pad it: the
// header text is padded with spaces so that magic + version + length + text
// reach a multiple of 64 bytes, then a newline.
void save_npy_raw(const std::string& path, const char* descr, const std::string& shape, const void* data,
                  size_t nbytes) {
  std::ofstream f(path, std::ios::binary);
  if (!f.is_open()) throw std::runtime_error("Cannot write file: " + path);
  f.write("\x93NUMPY", 6);
  f.put(0x01);
  f.put(0x00);
  std::string hs = std::string("{'descr': '") + descr + "', 'fortran_order': False, 'shape': (" + shape + "), }";
  const size_t total = 6 + 2 + 2 + hs.size();
  hs.append((64 - total % 64) % 64, ' ');
  hs.push_back('\n');
  const uint16_t len = static_cast<uint16_t>(hs.size());
  f.write(reinterpret_cast<const char*>(&len), 2);
  f.write(hs.data(), len);
  f.write(reinterpret_cast<const char*>(data), static_cast<std::streamsize>(nbytes));
}

// (rows, cols) float32 C order (src/npy.h:96-141).
void save_npy_f32(const std::string& path, const float* data, long long rows, long long cols) {
  save_npy_raw(path, "<f4", std::to_string(rows) + ", " + std::to_string(cols), data,
               static_cast<size_t>(rows * cols) * sizeof(float));
}

// 1-D uint8 (src/npy.h:56-79).
void save_npy_u8(const std::string& path, const std::vector<uint8_t>& v) {
  save_npy_raw(path, "|u1", std::to_string(v.size()) + ",", v.data(), v.size());
}

// Loads an npy of '<f4' or '<f8' as float32 (rows, cols) C order.
std::vector<float> load_npy(const std::string& path, long long* rows, long long* cols) {
  std::ifstream f(path, std::ios::binary);
  if (!f.is_open()) throw std::runtime_error("cannot open: " + path);
  char magic[6];
  f.read(magic, 6);
  if (std::memcmp(magic, "\x93NUMPY", 6) != 0) throw std::runtime_error("not an npy file: " + path);
  char ver[2];
  f.read(ver, 2);
  uint32_t hlen = 0;
  if (ver[0] == 1) {
    uint16_t h16;
    f.read(reinterpret_cast<char*>(&h16), 2);
    hlen = h16;
  } else {
    f.read(reinterpret_cast<char*>(&hlen), 4);
  }
  std::string header(hlen, ' ');
  f.read(&header[0], hlen);
  const bool f32 = header.find("'<f4'") != std::string::npos, f64 = header.find("'<f8'") != std::string::npos;
  if (!f32 && !f64) throw std::runtime_error("unsupported dtype in " + path);
  if (header.find("'fortran_order': True") != std::string::npos) throw std::runtime_error("fortran order npy: " + path);
  const auto sp = header.find("'shape':"), p1 = header.find('(', sp), p2 = header.find(')', p1);
  std::string s = header.substr(p1 + 1, p2 - p1 - 1);
  std::replace(s.begin(), s.end(), ',', ' ');
  std::stringstream ss(s);
  ss >> *rows >> *cols;
  const size_t n = static_cast<size_t>(*rows) * static_cast<size_t>(*cols);
  std::vector<float> out(n);
  if (f32) {
    f.read(reinterpret_cast<char*>(out.data()), static_cast<std::streamsize>(n * 4));
  } else {
    std::vector<double> b(n);
    f.read(reinterpret_cast<char*>(b.data()), static_cast<std::streamsize>(n * 8));
    for (size_t i = 0; i < n; ++i) out[i] = static_cast<float>(b[i]);
  }
  if (!f) throw std::runtime_error("truncated npy: " + path);
  return out;
}

// SHA-256 (FIPS 180-4) of a file, for the run manifest.
std::string sha256_file(const std::string& path) {
  static const uint32_t K[64] = {
      0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5, 0xd807aa98,
      0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174, 0xe49b69c1, 0xefbe4786,
      0x0fc19dc6, 0x240ca1cc, 0x2de92c6f, 0x4a7484aa, 0x5cb0a9dc, 0x76f988da, 0x983e5152, 0xa831c66d, 0xb00327c8,
      0xbf597fc7, 0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967, 0x27b70a85, 0x2e1b2138, 0x4d2c6dfc, 0x53380d13,
      0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85, 0xa2bfe8a1, 0xa81a664b, 0xc24b8b70, 0xc76c51a3, 0xd192e819,
      0xd6990624, 0xf40e3585, 0x106aa070, 0x19a4c116, 0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a,
      0x5b9cca4f, 0x682e6ff3, 0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7,
      0xc67178f2};
  uint32_t H[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a, 0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};
  std::ifstream f(path, std::ios::binary);
  if (!f.is_open()) return "";
  std::string data((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
  const uint64_t bits = static_cast<uint64_t>(data.size()) * 8;
  data.push_back(static_cast<char>(0x80));
  while (data.size() % 64 != 56) data.push_back(0);
  for (int i = 7; i >= 0; --i) data.push_back(static_cast<char>((bits >> (8 * i)) & 0xff));
  auto rotr = [](uint32_t x, int n) { return (x >> n) | (x << (32 - n)); };
  for (size_t off = 0; off < data.size(); off += 64) {
    uint32_t w[64];
    for (int i = 0; i < 16; ++i) {
      const unsigned char* p = reinterpret_cast<const unsigned char*>(data.data() + off + 4 * i);
      w[i] = (uint32_t(p[0]) << 24) | (uint32_t(p[1]) << 16) | (uint32_t(p[2]) << 8) | uint32_t(p[3]);
    }
    for (int i = 16; i < 64; ++i) {
      const uint32_t s0 = rotr(w[i - 15], 7) ^ rotr(w[i - 15], 18) ^ (w[i - 15] >> 3);
      const uint32_t s1 = rotr(w[i - 2], 17) ^ rotr(w[i - 2], 19) ^ (w[i - 2] >> 10);
      w[i] = w[i - 16] + s0 + w[i - 7] + s1;
    }
    uint32_t a = H[0], b = H[1], c = H[2], d = H[3], e = H[4], fv = H[5], g = H[6], h = H[7];
    for (int i = 0; i < 64; ++i) {
      const uint32_t S1 = rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25);
      const uint32_t ch = (e & fv) ^ (~e & g);
      const uint32_t t1 = h + S1 + ch + K[i] + w[i];
      const uint32_t S0 = rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22);
      const uint32_t mj = (a & b) ^ (a & c) ^ (b & c);
      const uint32_t t2 = S0 + mj;
      h = g;
      g = fv;
      fv = e;
      e = d + t1;
      d = c;
      c = b;
      b = a;
      a = t1 + t2;
    }
    H[0] += a;
    H[1] += b;
    H[2] += c;
    H[3] += d;
    H[4] += e;
    H[5] += fv;
    H[6] += g;
    H[7] += h;
  }
  std::ostringstream o;
  for (uint32_t x : H) o << std::hex << std::setw(8) << std::setfill('0') << x;
  return o.str();
}

void json_string(std::ostream& o, const std::string& s) {
  o << '"';
  for (char c : s) {
    if (c == '"' || c == '\\') o << '\\' << c;
    else if (c == '\n') o << "\\n";
    else o << c;
  }
  o << '"';
}

void phase(bool on, const std::string& what) {
  if (on) std::cout << "> " << what << std::endl;
}
void kv(bool on, const std::string& k, const std::string& v) {
  if (on) std::cout << "  " << std::left << std::setw(16) << k << v << std::endl;
}

void check(int st) {
  if (st != NAJA_OK) throw std::runtime_error(naja_last_error());
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// ------------------------------------------------------------ sample run
[[noreturn]] void die_usage(const std::string& msg) {
  std::cerr << "error: " << msg << "\n\nusage:\n"
            << "  naja sample run --model-dir <dir> --out-root <dir> --n-chains K --n-samples S\n"
            << "      [--gpu 0] [--tpb 128] [--thinning T] [--pair-prob p] [--resync-interval K]\n"
            << "      [--ksparse-prob p] [--ksparse-k k] [--extra-constraints auto|ignore|require]\n"
            << "      [--backmap] [--write-npy] [--bounds-policy ignore|filter] [--bounds-eps e]\n"
            << "      [--write-samples-valid] [--precision fp32|fp64] [--rng philox|mrg]\n"
            << "      [--backmap-mode fp64|tf32x3|bf16x3] [--verbose] [--quiet] [--dry-run] [--print-config]\n"
            << "      [--pair-schedule FILE] [--iter-rounding-passes P] [--iter-rounding-warmup W]\n"
            << "      [--affine-hull-tol t] [--extra-constraint-eps e] [--constraint-eps e]\n"
            << "  naja sample bulk --models-root <dir> --model-list <file> --out-root <dir> --name <run>\n"
            << "      --gpus <csv> --n-chains K --n-samples S [--skip-existing] [--resume-from <run_dir>]\n"
            << "      [the per-job flags of sample run]\n"
            << "  naja sample calibrate-rounding --models-root <dir> --model-list <file> --out <csv>\n"
            << "      [--warmup 2000] [--passes 2] [--pair-prob 0.3] [--extra-constraint-eps 0] [--seed 1]\n"
            << "      [--max-models 0]\n";
  std::exit(2);
}

std::string next_arg(int& i, int argc, char** argv, const std::string& flag) {
  if (i + 1 >= argc) die_usage("missing value for " + flag);
  return argv[++i];
}

struct RunConfig {
  std::string model_dir, model_name, rounding_dir, gem_dir, data_dir, out_dir;
  int gpu = 0, n_chains = -1, n_samples = -1, tpb = 128, thinning = 0, resync_interval = 0, ksparse_k = 8;
  double pair_prob = 0.0, ksparse_prob = 0.0, bounds_eps = 1e-6;
  int iter_rounding_passes = 0, iter_rounding_warmup = 0;
  double affine_hull_tol = 0.0, extra_constraint_eps = 0.0, constraint_eps = 0.0;
  std::string pair_schedule;
  std::string extra_constraints = "auto", bounds_policy = "ignore", precision = "fp32", rng = "philox",
              backmap_mode = "fp64";
  bool backmap = false, write_npy = false, verbose = false, quiet = false, dry_run = false, print_config = false,
       write_samples_valid = false;
  bool tpb_set = false;  // --tpb given: run that thread count; otherwise the library picks the kernel
  std::string file(const std::string& what) const { return rounding_dir + "/" + model_name + "_rounding_" + what + ".csv"; }
};

void require_nonempty(const std::string& path, const std::string& what) {
  struct stat st;
  if (!path_exists(path)) throw std::runtime_error("missing " + what + ": " + path);
  if (stat(path.c_str(), &st) != 0) throw std::runtime_error("cannot stat " + what + ": " + path);
  if (st.st_size == 0) throw std::runtime_error("empty " + what + ": " + path);
}

void validate_contract(const RunConfig& c) {
  if (!is_directory(c.rounding_dir)) throw std::runtime_error("missing rounding/ dir: " + c.rounding_dir);
  require_nonempty(c.file("A"), "rounding_A");
  require_nonempty(c.file("b"), "rounding_b");
  require_nonempty(c.file("start"), "rounding_start");
  if (c.backmap) {
    require_nonempty(c.file("T"), "rounding_T");
    require_nonempty(c.file("shift"), "rounding_shift");
  }
  const bool ha = path_exists(c.file("extra_A")), hb = path_exists(c.file("extra_b"));
  if (ha != hb)
    throw std::runtime_error("extra constraints must be both-present or both-absent: " + c.file("extra_A") + " / " +
                             c.file("extra_b"));
  if (ha) {
    require_nonempty(c.file("extra_A"), "extra_A");
    require_nonempty(c.file("extra_b"), "extra_b");
  }
}

std::string allocate_run_dir(const std::string& out_root, const std::string& name) {
  ensure_dir(out_root);
  const std::string date = stamp("%Y%m%d");
  for (int idx = 1; idx < 1000000; ++idx) {
    std::ostringstream o;
    o << out_root << "/" << name << "_" << date << "_" << std::setw(3) << std::setfill('0') << idx;
    if (!path_exists(o.str())) {
      ensure_dir(o.str());
      return o.str();
    }
  }
  throw std::runtime_error("could not allocate run directory under " + out_root);
}

void write_generated_config(const std::string& path, const RunConfig& c) {
  std::ofstream f(path);
  if (!f.is_open()) throw std::runtime_error("cannot write generated config: " + path);
  f << "DATA_DIR=" << c.data_dir << "\n"
    << "MODEL_NAME=" << c.model_name << "\n"
    << "OUT_DIR=" << c.out_dir << "\n"
    << "N_CHAINS=" << c.n_chains << "\n"
    << "N_SAMPLES=" << c.n_samples << "\n"
    << "TPB_SS=" << c.tpb << "\n"
    << "GPU_DEVICE=" << c.gpu << "\n"
    << "THINNING=" << c.thinning << "\n"
    << "PAIR_PROB=" << std::setprecision(17) << c.pair_prob << "\n"
    << "RESYNC_INTERVAL=" << c.resync_interval << "\n"
    << "KSPARSE_PROB=" << c.ksparse_prob << "\n"
    << "KSPARSE_K=" << c.ksparse_k << "\n"
    << "EXTRA_CONSTRAINTS=" << c.extra_constraints << "\n"
    << "BACK_TRANSFORM=" << (c.backmap ? 1 : 0) << "\n"
    << "WRITE_DATA=" << (c.write_npy ? 1 : 0) << "\n"
    << "BOUNDS_FILTER=" << (c.bounds_policy == "filter" ? 1 : 0) << "\n"
    << "BOUNDS_EPS=" << c.bounds_eps << "\n"
    << "WRITE_SAMPLES_VALID=" << (c.write_samples_valid ? 1 : 0) << "\n"
    << "PRECISION=" << c.precision << "\n"
    << "RNG=" << c.rng << "\n"
    << "BACKMAP_MODE=" << c.backmap_mode << "\n"
    << "ITER_ROUNDING_PASSES=" << c.iter_rounding_passes << "\n"
    << "ITER_ROUNDING_WARMUP=" << c.iter_rounding_warmup << "\n"
    << "PAIR_SCHEDULE=" << c.pair_schedule << "\n"
    << "AFFINE_HULL_TOL=" << c.affine_hull_tol << "\n"
    << "EXTRA_CONSTRAINT_EPS=" << c.extra_constraint_eps << "\n"
    << "CONSTRAINT_EPS=" << c.constraint_eps << "\n";
}

void write_run_manifest(const RunConfig& c, const std::vector<std::string>& argv_full,
                        const std::string& name = "run_manifest.json") {
  const std::string exe = self_path();
  struct stat st {};
  stat(exe.c_str(), &st);
  std::ofstream f(c.out_dir + "/" + name);
  if (!f.is_open()) throw std::runtime_error("cannot write run manifest: " + c.out_dir + "/" + name);
  f << "{\n  \"argv\": [";
  for (size_t i = 0; i < argv_full.size(); ++i) {
    if (i) f << ", ";
    json_string(f, argv_full[i]);
  }
  f << "],\n  \"model_dir\": ";
  json_string(f, absolute(c.model_dir));
  f << ",\n  \"engine\": {\n    \"path\": ";
  json_string(f, absolute(exe));
  f << ",\n    \"sha256\": ";
  json_string(f, sha256_file(exe));
  f << ",\n    \"size\": " << static_cast<long long>(st.st_size) << ",\n    \"library\": ";
  json_string(f, naja_version());
  f << "\n  },\n  \"config\": {\n"
    << "    \"gpu_device\": " << c.gpu << ",\n"
    << "    \"n_chains\": " << c.n_chains << ",\n"
    << "    \"n_samples\": " << c.n_samples << ",\n"
    << "    \"tpb_ss\": " << c.tpb << ",\n"
    << "    \"back_transform\": " << (c.backmap ? "true" : "false") << ",\n"
    << "    \"write_data\": " << (c.write_npy ? "true" : "false") << ",\n"
    << "    \"bounds_policy\": ";
  json_string(f, c.bounds_policy);
  f << ",\n    \"bounds_eps\": " << std::setprecision(12) << c.bounds_eps << ",\n"
    << "    \"write_samples_valid\": " << (c.write_samples_valid ? "true" : "false") << "\n  },\n"
    << "  \"resolved_paths\": {\n    \"model_dir\": ";
  json_string(f, absolute(c.model_dir));
  const char* keys[] = {"A", "b", "start", "T", "shift", "extra_A", "extra_b"};
  for (const char* k : keys) {
    f << ",\n    \"" << k << "\": ";
    json_string(f, absolute(c.file(k)));
  }
  f << "\n  }\n}\n";
}

struct Profile {
  double load = 0, upload = 0, sampling = 0, download = 0, backtransform = 0, write = 0, total = 0, throughput = 0;
  int n_chains = 0, n_samples = 0, reduced_dim = 0, original_dim = 0, constraints = 0, thinning = 0;
};

void write_profile(const std::string& path, const Profile& p, const RunConfig& c) {
  std::ofstream f(path);
  if (!f.is_open()) throw std::runtime_error("cannot write profile: " + path);
  f << "{\n  \"timestamp\": \"" << stamp("%Y-%m-%d %H:%M:%S") << "\",\n  \"config\": {\n"
    << "    \"n_chains\": " << p.n_chains << ",\n    \"n_samples\": " << p.n_samples << ",\n"
    << "    \"reduced_dim\": " << p.reduced_dim << ",\n    \"original_dim\": " << p.original_dim << ",\n"
    << "    \"constraints\": " << p.constraints << ",\n    \"thinning\": " << p.thinning << ",\n"
    << "    \"tpb_ss\": " << c.tpb << ",\n    \"gpu_device\": " << c.gpu << ",\n"
    << "    \"back_transform\": " << (c.backmap ? "true" : "false") << "\n  },\n  \"timing\": {\n"
    << std::fixed << std::setprecision(4) << "    \"load_polytope_s\": " << p.load << ",\n"
    << "    \"upload_to_gpu_s\": " << p.upload << ",\n    \"gpu_sampling_s\": " << p.sampling << ",\n"
    << "    \"download_from_gpu_s\": " << p.download << ",\n    \"backtransform_s\": " << p.backtransform << ",\n"
    << "    \"write_output_s\": " << p.write << ",\n    \"total_s\": " << p.total << "\n  },\n"
    << "  \"performance\": {\n    \"total_samples\": " << static_cast<long long>(p.n_chains) * p.n_samples << ",\n"
    << "    \"throughput_samples_per_sec\": " << std::setprecision(1) << p.throughput << ",\n"
    << "    \"sampling_fraction\": " << std::setprecision(3) << (p.total > 0 ? p.sampling / p.total : 0.0) << "\n"
    << "  }\n}\n";
}

void write_config_used(const RunConfig& c, const std::string& gen) {
  std::ofstream dst(c.out_dir + "/config_used.txt");
  std::ifstream src(gen);
  if (!dst.is_open() || !src.is_open()) throw std::runtime_error("cannot write config snapshot: " + c.out_dir);
  dst << "# Source config: " << absolute(gen) << "\n# Captured at: " << stamp("%Y-%m-%d %H:%M:%S") << "\n"
      << "# Output directory: " << absolute(c.out_dir) << "\n\n"
      << src.rdbuf() << "\n# Derived metadata\nMODEL_NAME=" << c.model_name << "\n"
      << "DATA_DIR_ABS=" << absolute(c.data_dir) << "\nMODEL_DIR_ABS=" << absolute(c.model_dir) << "\n"
      << "A_FILE=" << absolute(c.file("A")) << "\nB_FILE=" << absolute(c.file("b")) << "\n";
}

// GEM-bounds filter of the backmapped samples (src/engine/bounds_filter.cpp:
// 65-180): sample j is valid when max over reactions i of
// max((lb_i - x) - eps, (x - ub_i) - eps) is <= 0, x the float32 sample
// widened to double.  Writes valid_mask.npy (uint8), valid_fraction.txt,
// bounds_report.json (mean / p99 / max of the per-sample worst violation,
// the ten reactions with the largest violation) and, if asked,
// samples_valid.npy.  Samples are split over the host's cores; each thread
// keeps its own per-reaction maxima, merged after the join (maxima, so the
// result does not depend on the split).
long long bounds_filter_and_write(const RunConfig& c, const std::vector<float>& out, long long N, long long dim) {
  const std::string ids_path = c.gem_dir + "/reaction_ids.txt";
  const std::string lb_path = c.gem_dir + "/l_bounds.csv", ub_path = c.gem_dir + "/u_bounds.csv";
  require_nonempty(ids_path, "gem/reaction_ids.txt");
  require_nonempty(lb_path, "gem/l_bounds.csv");
  require_nonempty(ub_path, "gem/u_bounds.csv");
  std::vector<std::string> ids;
  {
    std::ifstream f(ids_path);
    for (std::string line; std::getline(f, line);) {
      const size_t a = line.find_first_not_of(" \t\r\n"), z = line.find_last_not_of(" \t\r\n");
      if (a != std::string::npos) ids.push_back(line.substr(a, z - a + 1));
    }
  }
  const Csv l = load_csv(lb_path), u = load_csv(ub_path);
  if (static_cast<long long>(ids.size()) != dim)
    throw std::runtime_error("reaction_ids length mismatch: expected " + std::to_string(dim) + " got " +
                             std::to_string(ids.size()));
  if (static_cast<long long>(l.v.size()) != dim || static_cast<long long>(u.v.size()) != dim)
    throw std::runtime_error("bounds length mismatch: expected " + std::to_string(dim) + " got lb=" +
                             std::to_string(l.v.size()) + " ub=" + std::to_string(u.v.size()));
  const double eps = c.bounds_eps;
  std::vector<uint8_t> mask(static_cast<size_t>(N), 1);
  std::vector<double> per_sample(static_cast<size_t>(N), 0.0);
  const int nt = static_cast<int>(std::max<long long>(1, std::min<long long>(
                     std::max(1u, std::thread::hardware_concurrency()), (N + 4095) / 4096)));
  std::vector<std::vector<double>> worst_rxn(nt, std::vector<double>(static_cast<size_t>(dim), 0.0));
  std::vector<double> worst_all(nt, 0.0);
  std::vector<std::thread> pool;
  for (int t = 0; t < nt; ++t)
    pool.emplace_back([&, t] {
      const long long j0 = N * t / nt, j1 = N * (t + 1) / nt;
      double* wr = worst_rxn[t].data();
      double wa = 0.0;
      for (long long j = j0; j < j1; ++j) {
        const float* x = out.data() + j * dim;
        double worst = 0.0;
        bool ok = true;
        for (long long i = 0; i < dim; ++i) {
          const double xi = x[i];
          const double lo = (l.v[i] - xi) - eps, hi = (xi - u.v[i]) - eps;
          const double v = lo > hi ? lo : hi;
          if (v > 0.0) {
            ok = false;
            if (v > wa) wa = v;
            if (v > wr[i]) wr[i] = v;
            if (v > worst) worst = v;
          }
        }
        mask[j] = ok ? 1 : 0;
        per_sample[j] = worst;
      }
      worst_all[t] = wa;
    });
  for (auto& th : pool) th.join();
  double max_violation = 0.0;
  std::vector<double> by_rxn(static_cast<size_t>(dim), 0.0);
  for (int t = 0; t < nt; ++t) {
    max_violation = std::max(max_violation, worst_all[t]);
    for (long long i = 0; i < dim; ++i) by_rxn[i] = std::max(by_rxn[i], worst_rxn[t][i]);
  }
  long long n_valid = 0;
  for (uint8_t m : mask) n_valid += m != 0;
  save_npy_u8(c.out_dir + "/valid_mask.npy", mask);
  {
    std::ofstream vf(c.out_dir + "/valid_fraction.txt");
    if (!vf.is_open()) throw std::runtime_error("cannot write valid_fraction.txt");
    vf << std::setprecision(12) << (N ? static_cast<double>(n_valid) / static_cast<double>(N) : 0.0) << "\n";
  }
  if (c.write_samples_valid) {
    std::vector<float> valid;
    valid.reserve(static_cast<size_t>(n_valid * dim));
    for (long long j = 0; j < N; ++j)
      if (mask[j]) valid.insert(valid.end(), out.data() + j * dim, out.data() + (j + 1) * dim);
    save_npy_f32(c.out_dir + "/samples_valid.npy", valid.data(), n_valid, dim);
  }
  double mean_v = 0.0;
  for (double v : per_sample) mean_v += v;
  mean_v = N ? mean_v / static_cast<double>(N) : 0.0;
  double p99 = 0.0;
  if (N > 0) {
    const size_t k = static_cast<size_t>((99 * (N - 1)) / 100);
    std::nth_element(per_sample.begin(), per_sample.begin() + static_cast<std::ptrdiff_t>(k), per_sample.end());
    p99 = per_sample[k];
  }
  std::vector<std::pair<long long, double>> top;
  for (long long i = 0; i < dim; ++i) top.emplace_back(i, by_rxn[i]);
  const size_t k_top = static_cast<size_t>(std::min<long long>(dim, 10));
  std::partial_sort(top.begin(), top.begin() + static_cast<std::ptrdiff_t>(k_top), top.end(),
                    [](const auto& a, const auto& b) { return a.second > b.second; });
  top.resize(k_top);
  while (!top.empty() && top.back().second <= 0.0) top.pop_back();
  std::ofstream f(c.out_dir + "/bounds_report.json");
  if (!f.is_open()) throw std::runtime_error("Cannot write bounds report: " + c.out_dir + "/bounds_report.json");
  f << std::setprecision(12) << "{\n  \"model\": ";
  json_string(f, c.model_name);
  f << ",\n  \"model_dir\": ";
  json_string(f, absolute(c.model_dir));
  f << ",\n  \"run_dir\": ";
  json_string(f, absolute(c.out_dir));
  f << ",\n  \"eps\": " << eps << ",\n  \"n_total\": " << N << ",\n  \"n_valid\": " << n_valid
    << ",\n  \"n_invalid\": " << (N - n_valid) << ",\n  \"invalid_fraction\": "
    << (N ? static_cast<double>(N - n_valid) / static_cast<double>(N) : 0.0) << ",\n  \"mean_violation\": " << mean_v
    << ",\n  \"p99_violation\": " << p99 << ",\n  \"max_violation\": " << max_violation
    << ",\n  \"outputs\": {\n    \"valid_mask\": ";
  json_string(f, absolute(c.out_dir + "/valid_mask.npy"));
  f << ",\n    \"samples_valid\": ";
  if (c.write_samples_valid) json_string(f, absolute(c.out_dir + "/samples_valid.npy"));
  else f << "null";
  f << "\n  },\n  \"top_violations\": [\n";
  for (size_t i = 0; i < top.size(); ++i) {
    f << "    {\"index\": " << top[i].first << ", \"reaction\": ";
    json_string(f, ids[static_cast<size_t>(top[i].first)]);
    f << ", \"worst_violation\": " << top[i].second << "}" << (i + 1 != top.size() ? "," : "") << "\n";
  }
  f << "  ]\n}\n";
  return n_valid;
}

int run_sampling(const RunConfig& c) {
  const auto t_total = std::chrono::steady_clock::now();
  Profile prof;
  const bool st = !c.quiet;
  phase(st, "loading polytope");
  auto t0 = std::chrono::steady_clock::now();
  Csv A = load_csv(c.file("A")), b = load_csv(c.file("b")), x0 = load_csv(c.file("start"));
  const bool have_extra = path_exists(c.file("extra_A"));
  if (c.extra_constraints == "require" && !have_extra)
    throw std::runtime_error("--extra-constraints require: missing " + c.file("extra_A"));
  if (have_extra && c.extra_constraints != "ignore") {
    // append extra rows (src/pipeline/extra_constraints.cpp:17-58)
    Csv eA = load_csv(c.file("extra_A")), eb = load_csv(c.file("extra_b"));
    if (eA.cols != A.cols) throw std::runtime_error("extra_A has " + std::to_string(eA.cols) + " columns, A has " + std::to_string(A.cols));
    if (eb.rows * eb.cols != eA.rows) throw std::runtime_error("extra_b length does not match extra_A rows");
    for (double& v : eb.v) v += c.extra_constraint_eps;  // extra_constraints.cpp: b_extra + eps
    A.v.insert(A.v.end(), eA.v.begin(), eA.v.end());
    A.rows += eA.rows;
    b.v.insert(b.v.end(), eb.v.begin(), eb.v.end());
    b.rows += eb.rows * eb.cols;
  }
  if (c.constraint_eps > 0.0)
    for (double& v : b.v) v += c.constraint_eps;  // global relaxation A x <= b + eps (job_sampling.cu:142-146)
  int m = A.rows, d = A.cols;
  const int d_file = d;
  if (static_cast<int>(b.v.size()) != m) throw std::runtime_error("dimension mismatch: rhs vector size (" + std::to_string(b.v.size()) + ") != rows (" + std::to_string(m) + ")");
  if (static_cast<int>(x0.v.size()) != d) throw std::runtime_error("start point has " + std::to_string(x0.v.size()) + " values, A has " + std::to_string(d) + " columns");
  // feasible start (src/validate/feasibility.h:12-35): max(A x0 - b) <= 1e-9
  double worst = -1e300;
  for (int r = 0; r < m; ++r) {
    double s = 0;
    for (int k = 0; k < d; ++k) s += A.v[static_cast<size_t>(r) * d + k] * x0.v[k];
    worst = std::max(worst, s - b.v[r]);
  }
  if (worst > 1e-9) throw std::runtime_error("infeasible start point: max(A x0 - b) = " + std::to_string(worst));
  // Affine hull of the rows tight at the start (job_sampling.cu:196-235):
  // sample z in {z : (A B) z <= b - A x0}, y = B z + x0.
  std::vector<double> hull_basis, hull_shift;
  if (c.affine_hull_tol > 0.0) {
    int dd = d, n_tight = 0;
    if (naja::rounding::affine_hull_basis(A.v, b.v, x0.v, m, d, c.affine_hull_tol, hull_basis, &dd, &n_tight)) {
      Csv Ar;
      Ar.rows = m;
      Ar.cols = dd;
      Ar.v.assign(static_cast<size_t>(m) * dd, 0.0);
      std::vector<double> slack0(m);
      for (int r = 0; r < m; ++r) {
        double sx = 0.0;
        const double* ar = &A.v[static_cast<size_t>(r) * d];
        for (int k = 0; k < d; ++k) sx += ar[k] * x0.v[k];
        slack0[r] = b.v[r] - sx;
        double* o = &Ar.v[static_cast<size_t>(r) * dd];
        // a tight row lies in the span the basis is orthogonal to: its reduced
        // coefficients are zero (rounding leaves ~1e-16 that, over a zero
        // slack, would block every chord)
        if (slack0[r] <= c.affine_hull_tol) continue;
        for (int k = 0; k < d; ++k) {
          const double a = ar[k];
          if (a == 0.0) continue;
          const double* brow = &hull_basis[static_cast<size_t>(k) * dd];
          for (int q = 0; q < dd; ++q) o[q] += a * brow[q];
        }
      }
      hull_shift = x0.v;
      A = std::move(Ar);
      b.v = std::move(slack0);
      x0.v.assign(dd, 0.0);
      d = dd;
      if (c.verbose) {
        std::cout << "  affine_hull_tol  " << std::setprecision(12) << c.affine_hull_tol << "\n"
                  << "  affine_hull_rows " << n_tight << "\n  affine_hull_dim  " << dd << " (from " << d_file << ")\n";
      }
      for (int r = 0; r < m; ++r)
        if (-b.v[r] > 1e-9) throw std::runtime_error("infeasible start point after the affine-hull reduction");
    } else if (c.verbose) {
      std::cout << "  affine_hull_tol  " << std::setprecision(12) << c.affine_hull_tol << " (no reduction; "
                << n_tight << " tight rows)\n";
    }
  }
  const int thinning = c.thinning > 0 ? c.thinning : std::max(d / 6, 1);
  prof.load = seconds_since(t0);
  prof.n_chains = c.n_chains;
  prof.n_samples = c.n_samples;
  prof.reduced_dim = d;
  prof.constraints = m;
  prof.thinning = thinning;
  if (c.verbose) {
    std::cout << "  constraints     " << m << "\n  reduced_dim     " << d << "\n  thinning        " << thinning
              << "\n  time            " << std::fixed << std::setprecision(3) << prof.load << "s\n\n";
  }
  std::hash<std::string> h;
  int seed = static_cast<int>(h(c.model_name) ^ (h(c.model_dir) << 1) ^
                              static_cast<uint64_t>(c.gpu * 0x9e3779b9));
  if (seed == 0) seed = 1;

  phase(st, "uploading to gpu");
  t0 = std::chrono::steady_clock::now();
  const std::vector<double> Acm = colmajor(A);
  naja_polytope* P = nullptr;
  check(naja_polytope_create(c.gpu, m, d, Acm.data(), m, b.v.data(), &P));
  std::vector<double> X0(static_cast<size_t>(d) * c.n_chains);
  for (int k = 0; k < c.n_chains; ++k) std::copy(x0.v.begin(), x0.v.end(), X0.begin() + static_cast<size_t>(k) * d);
  prof.upload = seconds_since(t0);

  naja_chr_params p;
  naja_chr_params_default(&p);
  p.nspc = c.n_samples;
  p.thinning = thinning;
  p.nchains = c.n_chains;
  p.tpb = c.tpb_set ? c.tpb : 0;
  p.seed = static_cast<unsigned long long>(static_cast<long long>(seed));
  p.pair_prob = c.pair_prob;
  p.resync_interval = c.resync_interval;
  p.ksparse_prob = c.ksparse_prob;
  p.ksparse_k = c.ksparse_k;
  p.precision = c.precision == "fp64" ? NAJA_PREC_FP64 : NAJA_PREC_FP32;
  p.rng = c.rng == "mrg" ? NAJA_RNG_REF_MRG : NAJA_RNG_PHILOX;
  p.out_dtype = NAJA_DTYPE_F32;
  // Rounding plan (src/rounding/plan.cpp:12-62): a schedule file, else a warm-up estimate.
  naja::rounding::PairSchedule sched;
  if (!c.pair_schedule.empty()) {
    phase(st, "loading pair schedule");
    sched = naja::rounding::load_pair_schedule_csv(c.pair_schedule);
  } else if (c.iter_rounding_passes > 0 && c.iter_rounding_warmup > 0 && d >= 2) {
    phase(st, "iterative rounding-lite (warmup)");
    sched = naja::rounding::estimate_runtime_pair_schedule(P, x0.v, seed, c.iter_rounding_passes,
                                                           c.iter_rounding_warmup, c.pair_prob, p);
    if (c.verbose)
      std::cout << "  iter_rounding_passes " << c.iter_rounding_passes << "\n  iter_rounding_warmup "
                << c.iter_rounding_warmup << "\n  iter_rounding_pairs  " << sched.size() << "\n";
  }
  if (sched.size() > 0) {
    p.pair_mode = 2;
    p.pair_i = sched.i.data();
    p.pair_j = sched.j.data();
    p.pair_c = sched.c.data();
    p.pair_s = sched.s.data();
    p.n_pairs = sched.size();
  }
  const long long N = static_cast<long long>(c.n_samples) * c.n_chains;
  std::vector<float> out;
  long long dim = d;
  std::vector<double> Tcm, shift, lb, ub;
  if (c.backmap) {
    phase(st, "loading transform");
    Csv T = load_csv(c.file("T")), sh = load_csv(c.file("shift"));
    if (T.cols != d_file)
      throw std::runtime_error("dimension mismatch: transform matrix cols (" + std::to_string(T.cols) +
                               ") != reduced dim (" + std::to_string(d_file) + ")");
    shift = sh.v;
    if (!hull_basis.empty()) {
      // T <- T0 B, shift <- T0 x0 + shift (job_sampling.cu:299-303)
      Csv Tr;
      Tr.rows = T.rows;
      Tr.cols = d;
      Tr.v.assign(static_cast<size_t>(T.rows) * d, 0.0);
      for (int i = 0; i < T.rows; ++i) {
        const double* tr = &T.v[static_cast<size_t>(i) * d_file];
        double* o = &Tr.v[static_cast<size_t>(i) * d];
        for (int k = 0; k < d_file; ++k) {
          shift[i] += tr[k] * hull_shift[k];
          if (tr[k] == 0.0) continue;
          const double* brow = &hull_basis[static_cast<size_t>(k) * d];
          for (int q = 0; q < d; ++q) o[q] += tr[k] * brow[q];
        }
      }
      T = std::move(Tr);
    }
    Tcm = colmajor(T);
    dim = T.rows;
    prof.original_dim = T.rows;
    out.resize(static_cast<size_t>(N) * dim);
    const int mode = c.backmap_mode == "tf32x3" ? NAJA_BACKMAP_TF32X3
                     : c.backmap_mode == "bf16x3" ? NAJA_BACKMAP_BF16X3 : NAJA_BACKMAP_FP64;
    // Sampling and the backmap of each chunk overlapped in one call; the
    // reference times the backmap inside the sampling call too
    // (job_sampling.cu:313-336).
    phase(st, "gpu sampling+backmap");
    t0 = std::chrono::steady_clock::now();
    int rc = naja_chr_run_backmapped(P, &p, X0.data(), d, T.rows, Tcm.data(), T.rows, shift.data(), mode, out.data(),
                                     NAJA_DTYPE_F32, nullptr, nullptr, 0, nullptr);
    prof.sampling = seconds_since(t0);
    naja_polytope_destroy(P);
    check(rc);
  } else {
    out.resize(static_cast<size_t>(N) * d);
    phase(st, "gpu sampling");
    t0 = std::chrono::steady_clock::now();
    int rc = naja_chr_run(P, &p, X0.data(), d, out.data(), nullptr, nullptr);
    prof.sampling = seconds_since(t0);
    naja_polytope_destroy(P);
    check(rc);
  }
  prof.throughput = prof.sampling > 0 ? static_cast<double>(N) / prof.sampling : 0.0;
  if (st) std::cout << "> done: " << std::fixed << std::setprecision(1) << prof.sampling << "s, " << std::setprecision(0)
                    << prof.throughput << " samples/s" << std::endl;
  if (c.write_npy) {
    phase(st, "writing npy");
    t0 = std::chrono::steady_clock::now();
    save_npy_f32(c.out_dir + "/samples.npy", out.data(), N, dim);
    prof.write = seconds_since(t0);
  }
  if (c.bounds_policy == "filter") {
    phase(st, "bounds filter (GEM validity)");
    const long long n_ok = bounds_filter_and_write(c, out, N, dim);
    kv(st, "bounds_valid", std::to_string(n_ok) + "/" + std::to_string(N));
  }
  prof.total = seconds_since(t_total);
  write_profile(c.out_dir + "/profile.json", prof, c);
  write_config_used(c, c.out_dir + "/config_generated.txt");
  if (c.verbose) std::cout << "output      :: " << absolute(c.out_dir) << std::endl;
  return 0;
}

// The per-job flags shared by `sample run` and `sample bulk`
// (src/cli/sample/cmd_run.cpp:44-120, cmd_bulk.cpp:41-64).  Returns false
// for a flag that is not one of them.
bool parse_job_flag(RunConfig& c, const std::string& a, int& i, int argc, char** argv) {
  if (a == "--n-chains") c.n_chains = std::stoi(next_arg(i, argc, argv, a));
  else if (a == "--n-samples") c.n_samples = std::stoi(next_arg(i, argc, argv, a));
  else if (a == "--tpb") {
    c.tpb = std::stoi(next_arg(i, argc, argv, a));
    c.tpb_set = true;
  }
  else if (a == "--thinning") c.thinning = std::stoi(next_arg(i, argc, argv, a));
  else if (a == "--pair-prob") c.pair_prob = std::stod(next_arg(i, argc, argv, a));
  else if (a == "--resync-interval") c.resync_interval = std::stoi(next_arg(i, argc, argv, a));
  else if (a == "--ksparse-prob") c.ksparse_prob = std::stod(next_arg(i, argc, argv, a));
  else if (a == "--ksparse-k") c.ksparse_k = std::stoi(next_arg(i, argc, argv, a));
  else if (a == "--extra-constraints") c.extra_constraints = next_arg(i, argc, argv, a);
  else if (a == "--backmap") c.backmap = true;
  else if (a == "--write-npy") c.write_npy = true;
  else if (a == "--verbose") c.verbose = true;
  else if (a == "--bounds-policy") c.bounds_policy = next_arg(i, argc, argv, a);
  else if (a == "--bounds-eps") c.bounds_eps = std::stod(next_arg(i, argc, argv, a));
  else if (a == "--write-samples-valid") c.write_samples_valid = true;
  else if (a == "--quiet") c.quiet = true;
  else if (a == "--dry-run") c.dry_run = true;
  else if (a == "--print-config") c.print_config = true;
  else if (a == "--precision") c.precision = next_arg(i, argc, argv, a);
  else if (a == "--rng") c.rng = next_arg(i, argc, argv, a);
  else if (a == "--backmap-mode") c.backmap_mode = next_arg(i, argc, argv, a);
  else if (a == "--start-policy") {
    if (next_arg(i, argc, argv, a) != "file") die_usage("invalid --start-policy (only 'file' is supported)");
  } else if (a == "--iter-rounding-passes") c.iter_rounding_passes = std::stoi(next_arg(i, argc, argv, a));
  else if (a == "--iter-rounding-warmup") c.iter_rounding_warmup = std::stoi(next_arg(i, argc, argv, a));
  else if (a == "--pair-schedule" || a == "--pair-schedule-file") c.pair_schedule = next_arg(i, argc, argv, a);
  else if (a == "--affine-hull-tol") c.affine_hull_tol = std::stod(next_arg(i, argc, argv, a));
  else if (a == "--extra-constraint-eps") c.extra_constraint_eps = std::stod(next_arg(i, argc, argv, a));
  else if (a == "--constraint-eps") c.constraint_eps = std::stod(next_arg(i, argc, argv, a));
  else return false;
  return true;
}

void check_job_flags(const RunConfig& c) {
  if (c.n_chains <= 0) die_usage("invalid --n-chains");
  if (c.n_samples <= 0) die_usage("invalid --n-samples");
  if (c.pair_prob < 0.0 || c.pair_prob > 1.0) die_usage("invalid --pair-prob (must be in [0,1])");
  if (c.resync_interval < 0) die_usage("invalid --resync-interval (must be >=0)");
  if (c.ksparse_prob < 0.0 || c.ksparse_prob > 1.0) die_usage("invalid --ksparse-prob (must be in [0,1])");
  if (c.ksparse_k <= 0) die_usage("invalid --ksparse-k (must be >0)");
  if (c.iter_rounding_passes < 0) die_usage("--iter-rounding-passes must be >= 0");
  if (c.iter_rounding_warmup < 0) die_usage("--iter-rounding-warmup must be >= 0");
  if (c.extra_constraint_eps < 0.0) die_usage("invalid --extra-constraint-eps (must be >=0)");
  if (c.constraint_eps < 0.0) die_usage("invalid --constraint-eps (must be >=0)");
  if (c.affine_hull_tol < 0.0) die_usage("invalid --affine-hull-tol (must be >=0)");
  if (c.extra_constraints != "auto" && c.extra_constraints != "ignore" && c.extra_constraints != "require")
    die_usage("invalid --extra-constraints (auto|ignore|require)");
  if (c.bounds_policy != "ignore" && c.bounds_policy != "filter") die_usage("invalid --bounds-policy: " + c.bounds_policy);
  if (c.precision != "fp32" && c.precision != "fp64") die_usage("invalid --precision (fp32|fp64)");
  if (c.rng != "philox" && c.rng != "mrg") die_usage("invalid --rng (philox|mrg)");
  if (c.backmap_mode != "fp64" && c.backmap_mode != "tf32x3" && c.backmap_mode != "bf16x3")
    die_usage("invalid --backmap-mode (fp64|tf32x3|bf16x3)");
  if (c.bounds_policy == "filter" && !c.backmap) throw std::runtime_error("bounds-policy=filter requires --backmap");
}

// Model name and contract paths of a model directory (model_contract.cpp:56-84).
void set_model(RunConfig& c, std::string md) {
  if (!md.empty() && md.back() == '/') md.pop_back();
  if (!is_directory(md)) throw std::runtime_error("model-dir is not a directory: " + md);
  const auto slash = md.find_last_of('/');
  c.model_dir = md;
  c.model_name = slash == std::string::npos ? md : md.substr(slash + 1);
  c.rounding_dir = md + "/rounding";
  c.gem_dir = md + "/gem";
  c.data_dir = slash == std::string::npos ? "." : md.substr(0, slash);
}

int cmd_sample_run(int argc, char** argv) {
  RunConfig c;
  std::string out_root;
  for (int i = 0; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "--model-dir") c.model_dir = next_arg(i, argc, argv, a);
    else if (a == "--out-root") out_root = next_arg(i, argc, argv, a);
    else if (a == "--gpu") c.gpu = std::stoi(next_arg(i, argc, argv, a));
    else if (!parse_job_flag(c, a, i, argc, argv)) die_usage("unknown flag: " + a);
  }
  if (c.model_dir.empty()) die_usage("missing --model-dir");
  if (out_root.empty()) die_usage("missing --out-root");
  check_job_flags(c);
  set_model(c, c.model_dir);
  validate_contract(c);
  c.out_dir = allocate_run_dir(out_root, c.model_name);
  const bool st = !c.quiet;
  phase(st, "validate model contract");
  phase(st, "write generated config");
  const std::string gen = c.out_dir + "/config_generated.txt";
  write_generated_config(gen, c);
  if (c.print_config) {
    std::cout << "config_generated    :: " << absolute(gen) << "\n---\n";
    std::ifstream f(gen);
    std::cout << f.rdbuf() << "---\n";
  }
  std::vector<std::string> full = {"naja", "sample", "run"};
  for (int i = 0; i < argc; ++i) full.push_back(argv[i]);
  write_run_manifest(c, full);
  kv(st, "model", c.model_name);
  kv(st, "output", absolute(c.out_dir));
  kv(st, "bounds", c.bounds_policy);
  if (c.bounds_policy == "filter") kv(st, "bounds_eps", std::to_string(c.bounds_eps));
  if (c.dry_run) {
    phase(st, "dry-run: not executing sampling");
    return 0;
  }
  phase(st, "sampling");
  return run_sampling(c);
}

// ------------------------------------------------- calibrate-rounding
// One pair schedule for a list of models (src/cli/sample/cmd_calibrate_rounding.cpp:24-195):
// pairs from a shuffle seeded with --seed, then per pass one warm-up chain
// per model (--warmup samples, thinning 1, Jacobi pairs of the schedule so
// far, seed ^ model index ^ (pass + 1)), the pairs' population moments
// averaged over models, and the Jacobi rotation of the averages.
std::vector<std::string> load_model_list(const std::string& path) {
  require_nonempty(path, "model list");
  std::ifstream f(path);
  if (!f.is_open()) throw std::runtime_error("cannot open model list: " + path);
  std::vector<std::string> out;
  for (std::string line; std::getline(f, line);) {
    const size_t a = line.find_first_not_of(" \t\r\n"), z = line.find_last_not_of(" \t\r\n");
    if (a == std::string::npos) continue;
    line = line.substr(a, z - a + 1);
    if (line[0] == '#') continue;
    out.push_back(line);
  }
  if (out.empty()) throw std::runtime_error("no models in list: " + path);
  return out;
}

int cmd_calibrate_rounding(int argc, char** argv) {
  std::string models_root, model_list, out_csv;
  int warmup = 2000, passes = 2, seed = 1, max_models = 0, gpu = 0;
  double pair_prob = 0.3, extra_eps = 0.0;
  std::string precision = "fp64", rng = "mrg";
  for (int i = 0; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "--models-root") models_root = next_arg(i, argc, argv, a);
    else if (a == "--model-list") model_list = next_arg(i, argc, argv, a);
    else if (a == "--out") out_csv = next_arg(i, argc, argv, a);
    else if (a == "--warmup") warmup = std::stoi(next_arg(i, argc, argv, a));
    else if (a == "--passes") passes = std::stoi(next_arg(i, argc, argv, a));
    else if (a == "--pair-prob") pair_prob = std::stod(next_arg(i, argc, argv, a));
    else if (a == "--extra-constraint-eps") extra_eps = std::stod(next_arg(i, argc, argv, a));
    else if (a == "--seed") seed = std::stoi(next_arg(i, argc, argv, a));
    else if (a == "--max-models") max_models = std::stoi(next_arg(i, argc, argv, a));
    else if (a == "--gpu") gpu = std::stoi(next_arg(i, argc, argv, a));
    else if (a == "--precision") precision = next_arg(i, argc, argv, a);
    else if (a == "--rng") rng = next_arg(i, argc, argv, a);
    else die_usage("unknown flag: " + a);
  }
  if (models_root.empty()) die_usage("missing --models-root");
  if (model_list.empty()) die_usage("missing --model-list");
  if (out_csv.empty()) die_usage("missing --out");
  if (warmup <= 0) die_usage("invalid --warmup");
  if (passes <= 0) die_usage("invalid --passes");
  if (!(pair_prob > 0.0 && pair_prob <= 1.0)) die_usage("invalid --pair-prob (0,1]");
  if (extra_eps < 0.0) die_usage("invalid --extra-constraint-eps (must be >=0)");
  if (max_models < 0) die_usage("invalid --max-models (must be >=0)");
  if (precision != "fp32" && precision != "fp64") die_usage("invalid --precision (fp32|fp64)");
  if (rng != "philox" && rng != "mrg") die_usage("invalid --rng (philox|mrg)");
  if (seed == 0) seed = 1;
  std::vector<std::string> names = load_model_list(model_list);
  if (max_models > 0 && static_cast<int>(names.size()) > max_models) names.resize(max_models);
  struct Model {
    naja_polytope* P = nullptr;
    std::vector<double> x0;
  };
  std::vector<Model> models;
  int d = -1;
  for (const std::string& nm : names) {
    RunConfig c;
    c.model_dir = absolute(models_root + "/" + nm);
    c.model_name = nm.substr(nm.find_last_of('/') == std::string::npos ? 0 : nm.find_last_of('/') + 1);
    c.rounding_dir = c.model_dir + "/rounding";
    validate_contract(c);
    Csv A = load_csv(c.file("A")), b = load_csv(c.file("b")), x0 = load_csv(c.file("start"));
    if (path_exists(c.file("extra_A")) && path_exists(c.file("extra_b"))) {
      Csv eA = load_csv(c.file("extra_A")), eb = load_csv(c.file("extra_b"));
      if (eA.cols != A.cols) throw std::runtime_error("extra_A columns differ from A: " + c.file("extra_A"));
      for (double& v : eb.v) v += extra_eps;
      A.v.insert(A.v.end(), eA.v.begin(), eA.v.end());
      A.rows += eA.rows;
      b.v.insert(b.v.end(), eb.v.begin(), eb.v.end());
    }
    if (d < 0) d = A.cols;
    if (A.cols != d) throw std::runtime_error("model " + nm + " has reduced dim " + std::to_string(A.cols) + ", expected " + std::to_string(d));
    if (d < 2) throw std::runtime_error("calibrate-rounding requires reduced_dim >= 2");
    Model mdl;
    const std::vector<double> Acm = colmajor(A);
    check(naja_polytope_create(gpu, A.rows, d, Acm.data(), A.rows, b.v.data(), &mdl.P));
    mdl.x0 = x0.v;
    models.push_back(std::move(mdl));
  }
  naja::rounding::PairSchedule sched = naja::rounding::random_pairing(d, static_cast<uint64_t>(seed));
  const int np = sched.size();
  std::vector<double> W(static_cast<size_t>(warmup) * d);
  for (int pass = 0; pass < passes; ++pass) {
    std::vector<double> svi(np, 0.0), svj(np, 0.0), scov(np, 0.0);
    for (size_t mi = 0; mi < models.size(); ++mi) {
      naja_chr_params p;
      naja_chr_params_default(&p);
      p.nspc = warmup;
      p.thinning = 1;
      p.nchains = 1;
      p.tpb = 0;
      p.seed = static_cast<unsigned long long>(static_cast<long long>(seed ^ static_cast<int>(mi) ^ (pass + 1)));
      p.pair_prob = pair_prob;
      p.pair_mode = 2;
      p.pair_i = sched.i.data();
      p.pair_j = sched.j.data();
      p.pair_c = sched.c.data();
      p.pair_s = sched.s.data();
      p.n_pairs = np;
      p.precision = precision == "fp64" ? NAJA_PREC_FP64 : NAJA_PREC_FP32;
      p.rng = rng == "mrg" ? NAJA_RNG_REF_MRG : NAJA_RNG_PHILOX;
      p.out_dtype = NAJA_DTYPE_F64;
      check(naja_chr_run(models[mi].P, &p, models[mi].x0.data(), d, W.data(), nullptr, nullptr));
      check(naja_polytope_check(models[mi].P));
      for (int k = 0; k < np; ++k) {
        const int ii = sched.i[k], jj = sched.j[k];
        double mi_ = 0.0, mj_ = 0.0;
        for (int t = 0; t < warmup; ++t) {
          mi_ += W[static_cast<size_t>(t) * d + ii];
          mj_ += W[static_cast<size_t>(t) * d + jj];
        }
        mi_ /= warmup;
        mj_ /= warmup;
        double vi = 0.0, vj = 0.0, cv = 0.0;
        for (int t = 0; t < warmup; ++t) {
          const double a = W[static_cast<size_t>(t) * d + ii] - mi_, bb = W[static_cast<size_t>(t) * d + jj] - mj_;
          vi += a * a;
          vj += bb * bb;
          cv += a * bb;
        }
        svi[k] += vi / warmup;
        svj[k] += vj / warmup;
        scov[k] += cv / warmup;
      }
    }
    const double w = static_cast<double>(models.size());
    for (int k = 0; k < np; ++k) {
      const auto cs = naja::rounding::jacobi_rotation_cs(svi[k] / w, svj[k] / w, scov[k] / w);
      sched.c[k] = cs.first;
      sched.s[k] = cs.second;
    }
  }
  for (auto& mdl : models) naja_polytope_destroy(mdl.P);
  naja::rounding::write_pair_schedule_csv(out_csv, sched);
  std::cout << "OK\n"
            << "out              :: " << absolute(out_csv) << "\n"
            << "models           :: " << names.size() << "\n"
            << "reduced_dim      :: " << d << "\n"
            << "pairs            :: " << np << "\n"
            << "passes           :: " << passes << "\n"
            << "warmup           :: " << warmup << "\n"
            << "pair_prob        :: " << pair_prob << "\n"
            << "extra_eps        :: " << extra_eps << "\n";
  return 0;
}

// ------------------------------------------------------------ sample bulk
// Every model of a list sampled into one run directory
// (src/cli/sample/cmd_bulk.cpp:20-163, src/engine/job_bulk.cpp:115-267):
// one host thread per entry of --gpus, all pulling the next model index
// from one atomic counter; each job gets <run>/<model>/<model>_<date>_<NNN>
// and runs exactly as `sample run` would (same flags, seed from model name,
// model directory and GPU).  --skip-existing takes a model as done when a
// job directory of it holds a non-empty samples.npy and profile.json (and,
// with the bounds filter, valid_mask.npy, valid_fraction.txt and
// bounds_report.json); --resume-from reuses a run directory.  The run ends
// with bulk_summary.csv (model,status,elapsed_s,device_id,message,
// output_dir,inherited_from_base) and fails when any job failed.
struct BulkResult {
  std::string model, status, message, output_dir;
  double elapsed = 0.0;
  int device = 0;
};

bool file_nonempty(const std::string& path) {
  struct stat st;
  return stat(path.c_str(), &st) == 0 && st.st_size > 0;
}

std::vector<int> parse_gpu_list(const std::string& s) {
  std::vector<int> ids;
  std::stringstream ss(s);
  for (std::string tok; std::getline(ss, tok, ',');) {
    const size_t a = tok.find_first_not_of(" \t"), z = tok.find_last_not_of(" \t");
    if (a == std::string::npos) continue;
    const std::string t = tok.substr(a, z - a + 1);
    int id = -1;
    const auto [end, ec] = std::from_chars(t.data(), t.data() + t.size(), id);
    if (ec != std::errc() || end != t.data() + t.size() || id < 0) die_usage("invalid --gpus entry: " + t);
    ids.push_back(id);
  }
  if (ids.empty()) die_usage("invalid --gpus: " + s);
  return ids;
}

// The newest job directory of `model` under the run directory with complete
// outputs (job_bulk.cpp:86-111), or "".
std::string find_completed_job_dir(const std::string& run_dir, const std::string& model, bool filter) {
  const std::string root = run_dir + "/" + model;
  DIR* d = opendir(root.c_str());
  if (!d) return {};
  std::string best;
  time_t best_mtime = 0;
  for (dirent* e; (e = readdir(d)) != nullptr;) {
    const std::string name = e->d_name;
    if (name == "." || name == "..") continue;
    const std::string dir = root + "/" + name;
    struct stat st;
    if (stat(dir.c_str(), &st) != 0 || !S_ISDIR(st.st_mode)) continue;
    if (!file_nonempty(dir + "/samples.npy") || !file_nonempty(dir + "/profile.json")) continue;
    if (filter && (!file_nonempty(dir + "/valid_mask.npy") || !file_nonempty(dir + "/valid_fraction.txt") ||
                   !file_nonempty(dir + "/bounds_report.json")))
      continue;
    if (best.empty() || st.st_mtime > best_mtime) {
      best = dir;
      best_mtime = st.st_mtime;
    }
  }
  closedir(d);
  return best;
}

// <root>/<model>_<YYYYMMDD>_<NNN>, claimed by mkdir itself so that two
// workers given the same model never share a directory.
std::string claim_job_dir(const std::string& root, const std::string& model) {
  ensure_dir(root);
  const std::string date = stamp("%Y%m%d");
  for (int idx = 1; idx < 1000000; ++idx) {
    std::ostringstream o;
    o << root << "/" << model << "_" << date << "_" << std::setw(3) << std::setfill('0') << idx;
    if (mkdir(o.str().c_str(), 0755) == 0) return o.str();
    if (errno != EEXIST) throw std::runtime_error("cannot create directory: " + o.str());
  }
  throw std::runtime_error("could not allocate job directory under " + root);
}

std::string inherited_from_base(const std::string& models_root, const std::string& model) {
  std::ifstream f(models_root + "/" + model + "/rounding/INHERITED_FROM.txt");
  for (std::string line; std::getline(f, line);) {
    const size_t a = line.find_first_not_of(" \t\r\n"), z = line.find_last_not_of(" \t\r\n");
    if (a == std::string::npos) continue;
    line = line.substr(a, z - a + 1);
    if (line.rfind("base_model_dir=", 0) == 0) return line.substr(15);
  }
  return {};
}

int cmd_sample_bulk(int argc, char** argv) {
  RunConfig base;
  std::string models_root, model_list, out_root, resume_from, name, gpus;
  bool skip_existing = false;
  for (int i = 0; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "--models-root") models_root = next_arg(i, argc, argv, a);
    else if (a == "--model-list") model_list = next_arg(i, argc, argv, a);
    else if (a == "--out-root") out_root = next_arg(i, argc, argv, a);
    else if (a == "--resume-from") resume_from = next_arg(i, argc, argv, a);
    else if (a == "--name") name = next_arg(i, argc, argv, a);
    else if (a == "--gpus") gpus = next_arg(i, argc, argv, a);
    else if (a == "--skip-existing") skip_existing = true;
    else if (!parse_job_flag(base, a, i, argc, argv)) die_usage("unknown flag: " + a);
  }
  if (models_root.empty()) die_usage("missing --models-root");
  if (model_list.empty()) die_usage("missing --model-list");
  if (name.empty()) die_usage("missing --name");
  if (gpus.empty()) die_usage("missing --gpus");
  check_job_flags(base);
  const std::vector<int> gpu_ids = parse_gpu_list(gpus);
  if (!is_directory(models_root)) throw std::runtime_error("models-root is not a directory: " + models_root);
  const std::vector<std::string> models = load_model_list(model_list);
  std::vector<RunConfig> jobs;
  for (const auto& m : models) {
    RunConfig jc = base;
    set_model(jc, models_root + "/" + m);
    validate_contract(jc);
    jobs.push_back(std::move(jc));
  }
  RunConfig run = base;
  run.model_dir = models_root;
  run.data_dir = models_root;
  run.model_name = name;
  if (!resume_from.empty()) {
    if (!is_directory(resume_from)) throw std::runtime_error("resume-from is not a directory: " + resume_from);
    run.out_dir = resume_from;
  } else {
    if (out_root.empty()) die_usage("missing --out-root (or use --resume-from)");
    run.out_dir = allocate_run_dir(out_root, name);
  }
  const bool st = !base.quiet;
  phase(st, "validate model contracts");
  phase(st, "write generated bulk config");
  const std::string gen = run.out_dir + "/bulk_config_generated.txt";
  write_generated_config(gen, run);
  {
    std::ofstream f(gen, std::ios::app);
    f << "GPU_LIST=" << gpus << "\nBULK_MODEL_LIST=" << model_list << "\nSKIP_EXISTING=" << (skip_existing ? 1 : 0)
      << "\n";
  }
  if (base.print_config) {
    std::cout << "config_generated    :: " << absolute(gen) << "\n---\n";
    std::ifstream f(gen);
    std::cout << f.rdbuf() << "---\n";
  }
  std::vector<std::string> full = {"naja", "sample", "bulk"};
  for (int i = 0; i < argc; ++i) full.push_back(argv[i]);
  const bool resumed = !resume_from.empty() && path_exists(run.out_dir + "/run_manifest.json");
  write_run_manifest(run, full, resumed ? "run_manifest_resume.json" : "run_manifest.json");
  kv(st, "bulk_name", name);
  kv(st, "jobs", std::to_string(jobs.size()));
  kv(st, "gpus", gpus);
  kv(st, "output", absolute(run.out_dir));
  kv(st, "bounds", base.bounds_policy);
  if (base.bounds_policy == "filter") kv(st, "bounds_eps", std::to_string(base.bounds_eps));
  if (skip_existing) kv(st, "skip_existing", "true");
  if (base.dry_run) {
    phase(st, "dry-run: not executing bulk sampling");
    return 0;
  }
  phase(st, "bulk sampling");
  std::cout << "bulk sampling :: " << jobs.size() << " jobs across " << gpu_ids.size() << " gpu(s)\n"
            << "output root   :: " << absolute(run.out_dir) << "\n" << std::endl;

  std::atomic<size_t> next{0};
  std::mutex mu;
  std::vector<BulkResult> results;
  const bool filter = base.bounds_policy == "filter";
  auto worker = [&](int device) {
    for (;;) {
      const size_t k = next.fetch_add(1);
      if (k >= jobs.size()) return;
      RunConfig jc = jobs[k];
      jc.gpu = device;
      jc.quiet = true;
      jc.print_config = false;
      BulkResult r;
      r.model = jc.model_name;
      r.device = device;
      const auto t0 = std::chrono::steady_clock::now();
      std::string done = skip_existing ? find_completed_job_dir(run.out_dir, jc.model_name, filter) : std::string();
      if (!done.empty()) {
        r.status = "SKIP";
        r.message = "SKIP";
        r.output_dir = done;
      } else {
        try {
          jc.out_dir = claim_job_dir(run.out_dir + "/" + jc.model_name, jc.model_name);
          r.output_dir = jc.out_dir;
          write_generated_config(jc.out_dir + "/config_generated.txt", jc);
          const int rc = run_sampling(jc);
          r.status = rc == 0 ? "OK" : "FAIL";
          if (rc != 0) r.message = "return code " + std::to_string(rc);
        } catch (const std::exception& e) {
          r.status = "FAIL";
          r.message = e.what();
        }
        r.elapsed = seconds_since(t0);
      }
      std::lock_guard<std::mutex> lock(mu);
      std::cout << "[gpu " << device << "] " << r.model << " -> " << r.status;
      if (r.status != "SKIP") {
        std::cout << " (" << std::fixed << std::setprecision(2) << r.elapsed << "s";
        if (r.status == "FAIL" && !r.message.empty()) std::cout << ", " << r.message;
        std::cout << ")";
      }
      std::cout << std::endl;
      results.push_back(std::move(r));
    }
  };
  std::vector<std::thread> pool;
  for (int id : gpu_ids) pool.emplace_back(worker, id);
  for (auto& t : pool) t.join();

  size_t ok = 0;
  for (const auto& r : results) ok += r.status != "FAIL";
  std::cout << "\nsummary\n  completed : " << ok << " / " << jobs.size() << "\n" << std::endl;
  const std::string summary = run.out_dir + "/bulk_summary.csv";
  std::ofstream f(summary);
  if (!f.is_open()) throw std::runtime_error("cannot write bulk summary: " + summary);
  f << "model,status,elapsed_s,device_id,message,output_dir,inherited_from_base\n";
  for (const auto& r : results) {
    std::string msg = r.message;
    std::replace(msg.begin(), msg.end(), '\n', ' ');
    f << r.model << "," << r.status << "," << std::fixed << std::setprecision(2) << r.elapsed << "," << r.device
      << "," << msg << "," << r.output_dir << "," << inherited_from_base(models_root, r.model) << "\n";
  }
  f.close();
  std::cout << "  wrote summary :: " << summary << std::endl;
  if (ok != jobs.size()) throw std::runtime_error("bulk sampling failed with return code 2");
  return 0;
}


// ------------------------------------------------------------ validate
float percentile(std::vector<float> v, float q) {
  if (v.empty()) return 0.0f;
  std::sort(v.begin(), v.end());
  const float pos = q * static_cast<float>(v.size() - 1);
  const int lo = static_cast<int>(std::floor(pos)), hi = static_cast<int>(std::ceil(pos));
  if (lo == hi) return v[lo];
  const float t = pos - static_cast<float>(lo);
  return v[lo] * (1.0f - t) + v[hi] * t;
}

[[noreturn]] void die_validate(const std::string& msg) {
  std::cerr << "error: " << msg << "\n\nusage:\n  naja validate --samples <file.npy> [--model-dir <dir>] [--n-chains 4]\n";
  std::exit(2);
}

int cmd_validate(int argc, char** argv) {
  std::string samples_path, model_dir;
  int n_chains = 4, gpu = 0;
  for (int i = 0; i < argc; ++i) {
    const std::string a = argv[i];
    auto nxt = [&]() -> std::string {
      if (i + 1 >= argc) die_validate("missing value for " + a);
      return argv[++i];
    };
    if (a == "--samples") samples_path = nxt();
    else if (a == "--model-dir") model_dir = nxt();
    else if (a == "--n-chains") n_chains = std::stoi(nxt());
    else if (a == "--gpu") gpu = std::stoi(nxt());
    else die_validate("unknown flag: " + a);
  }
  (void)gpu;
  if (samples_path.empty()) die_validate("missing --samples");
  if (n_chains < 1) die_validate("--n-chains must be >= 1");
  std::cerr << "loading " << samples_path << "..." << std::endl;
  long long rows = 0, cols = 0;
  std::vector<float> raw = load_npy(samples_path, &rows, &cols);
  // (n_samples, dim) rows are samples; the reference takes the smaller
  // extent as the dimension (validate_cli.cpp:96-99)
  const long long dim = std::min(rows, cols), n_total = std::max(rows, cols);
  std::vector<float> S;
  if (rows >= cols) {
    S.swap(raw);
  } else {
    S.resize(raw.size());
    for (long long dd = 0; dd < dim; ++dd)
      for (long long s = 0; s < n_total; ++s) S[s * dim + dd] = raw[dd * n_total + s];
  }
  const long long spc = n_total / n_chains;
  std::cerr << "  shape: (" << dim << ", " << n_total << ") = " << n_chains << " chains x " << spc << " samples" << std::endl;
  if (n_total % n_chains != 0)
    throw std::runtime_error("n_total (" + std::to_string(n_total) + ") not divisible by n_chains (" +
                             std::to_string(n_chains) + ")");
  int active = 0;
  for (long long dd = 0; dd < dim; ++dd) {
    double mean = 0, var = 0;
    for (long long s = 0; s < n_total; ++s) mean += S[s * dim + dd];
    mean /= n_total;
    for (long long s = 0; s < n_total; ++s) var += (S[s * dim + dd] - mean) * (S[s * dim + dd] - mean);
    if (var / n_total > 1e-20) ++active;
  }
  std::cerr << "  computing ESS..." << std::endl << "  computing split-R-hat..." << std::endl;
  std::vector<double> ess(static_cast<size_t>(dim) * n_chains), rh(static_cast<size_t>(dim));
  check(naja_validate(S.data(), n_total, static_cast<int>(dim), n_chains, 0, ess.data(), rh.data(), nullptr));
  std::vector<float> ess_dim(dim), rh_f(dim);
  for (long long dd = 0; dd < dim; ++dd) {
    double mn = 1e300;
    for (int k = 0; k < n_chains; ++k) mn = std::min(mn, ess[dd * n_chains + k]);
    ess_dim[dd] = static_cast<float>(mn);
    rh_f[dd] = static_cast<float>(rh[dd]);
  }
  const float ess_min = *std::min_element(ess_dim.begin(), ess_dim.end());
  const float ess_max = *std::max_element(ess_dim.begin(), ess_dim.end());
  const float ess_p10 = percentile(ess_dim, 0.10f), ess_med = percentile(ess_dim, 0.50f);
  const float rh_med = percentile(rh_f, 0.50f), rh_max = *std::max_element(rh_f.begin(), rh_f.end());
  int a11 = 0, a12 = 0;
  for (float r : rh_f) {
    a11 += r > 1.1f;
    a12 += r > 1.2f;
  }
  bool has_bounds = false;
  long long n_viol = 0, n_checked = 0;
  double worst = 0.0;
  if (!model_dir.empty()) {
    std::string md = model_dir;
    if (!md.empty() && md.back() == '/') md.pop_back();
    const auto slash = md.find_last_of('/');
    const std::string name = slash == std::string::npos ? md : md.substr(slash + 1);
    const std::string Tp = md + "/rounding/" + name + "_rounding_T.csv", sp = md + "/rounding/" + name + "_rounding_shift.csv";
    const std::string lp = md + "/gem/l_bounds.csv", up = md + "/gem/u_bounds.csv";
    if (path_exists(Tp) && path_exists(lp)) {
      std::cerr << "  checking bounds compliance..." << std::endl;
      const Csv T = load_csv(Tp), sh = load_csv(sp), l = load_csv(lp), u = load_csv(up);
      // samples in the reduced space are mapped with v = T y + shift; samples
      // written with --backmap are already in reaction space and checked as they are
      const bool reduced = T.cols == dim;
      if (!reduced && T.rows != dim)
        throw std::runtime_error("samples have " + std::to_string(dim) + " values, T is " + std::to_string(T.rows) +
                                 " x " + std::to_string(T.cols));
      // every max(1, n/1000)-th sample (src/validate/bounds_check.cpp:8-39)
      const long long step = std::max<long long>(1, n_total / 1000);
      // every (sample, reaction) pair counts once; violation = max(lb - v - eps, v - ub - eps) > 0
      for (long long s = 0; s < n_total; s += step) {
        for (int i = 0; i < T.rows; ++i) {
          double v;
          if (reduced) {
            v = sh.v[i];
            for (long long k = 0; k < dim; ++k) v += T.v[static_cast<size_t>(i) * T.cols + k] * S[s * dim + k];
          } else {
            v = S[s * dim + i];
          }
          ++n_checked;
          const double viol = std::max(l.v[i] - v - 1e-6, v - u.v[i] - 1e-6);
          if (viol > 0.0) {
            ++n_viol;
            worst = std::max(worst, viol);
          }
        }
      }
      has_bounds = true;
    }
  }
  std::string status = "OK";
  if (a12 > dim / 4) status = "FAIL";
  else if (a11 > dim / 4 || ess_min < 10) status = "WARN";
  std::cerr << "\n[" << status << "] ESS min=" << std::setprecision(0) << std::fixed << ess_min << " p10=" << ess_p10
            << " med=" << ess_med << "  R-hat med=" << std::setprecision(3) << rh_med << " max=" << rh_max
            << " >1.1=" << a11 << " >1.2=" << a12;
  if (has_bounds) std::cerr << "  bounds=" << n_viol << "/" << n_checked;
  std::cerr << std::endl;
  std::cout << "{\n  \"samples_file\": \"" << samples_path << "\",\n  \"shape\": [" << n_total << ", " << dim << "],\n"
            << "  \"n_chains\": " << n_chains << ",\n  \"n_samples_per_chain\": " << spc << ",\n"
            << "  \"active_dims\": " << active << ",\n  \"status\": \"" << status << "\",\n"
            << "  \"ess\": {\n    \"min\": " << std::setprecision(1) << std::fixed << ess_min << ",\n"
            << "    \"p10\": " << ess_p10 << ",\n    \"median\": " << ess_med << ",\n    \"max\": " << ess_max << "\n  },\n"
            << "  \"rhat\": {\n    \"median\": " << std::setprecision(4) << rh_med << ",\n    \"max\": " << rh_max << ",\n"
            << "    \"above_1_1\": " << a11 << ",\n    \"above_1_2\": " << a12 << "\n  }";
  if (has_bounds)
    std::cout << ",\n  \"bounds\": {\n    \"n_checked\": " << n_checked << ",\n    \"n_violations\": " << n_viol
              << ",\n    \"max_violation\": " << std::setprecision(6) << worst << "\n  }";
  std::cout << "\n}\n";
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  try {
    if (argc >= 3 && std::string(argv[1]) == "sample" && std::string(argv[2]) == "run")
      return cmd_sample_run(argc - 3, argv + 3);
    if (argc >= 3 && std::string(argv[1]) == "sample" && std::string(argv[2]) == "bulk")
      return cmd_sample_bulk(argc - 3, argv + 3);
    if (argc >= 3 && std::string(argv[1]) == "sample" && std::string(argv[2]) == "calibrate-rounding")
      return cmd_calibrate_rounding(argc - 3, argv + 3);
    if (argc >= 2 && std::string(argv[1]) == "validate") return cmd_validate(argc - 2, argv + 2);
    if (argc >= 2 && std::string(argv[1]) == "version") {
      std::cout << naja_version() << std::endl;
      return 0;
    }
    std::cerr << "usage:\n  naja sample run --model-dir <dir> --out-root <dir> --n-chains K --n-samples S [...]\n"
              << "  naja sample bulk --models-root <dir> --model-list <file> --out-root <dir> --name <run> --gpus <csv>\n"
              << "      --n-chains K --n-samples S [--skip-existing] [--resume-from <run_dir>] [...]\n"
              << "  naja sample calibrate-rounding --models-root <dir> --model-list <file> --out <csv> [...]\n"
              << "  naja validate --samples <file.npy> [--model-dir <dir>] [--n-chains 4]\n  naja version\n";
    return 2;
  } catch (const std::exception& e) {
    std::cerr << "error: " << e.what() << std::endl;
    return 1;
  }
}
