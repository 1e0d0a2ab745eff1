// owl_host.cpp -- the PRP / LL test drivers and savefiles above libowl.
//
// This is the host surface the reference keeps in C++ (Gpu::isPrimePRP and
// Gpu::isPrimeLL, src/Gpu.cpp:1400-1663; Saver, src/Saver.cpp; the Gerbicz
// state rebuild and check, src/Gpu.cpp:738-771), restated on the engine calls
// of owl.h. The loop logic follows the reference so that savefiles, residues
// and error handling behave the same; only the kernel plumbing is replaced --
// where the reference enqueued one squaring at a time with leadIn/leadOut
// flags, this loop hands whole stretches between its stop points to
// owl_square, which keeps the data in the FFT domain inside the stretch.
#include <algorithm>
#include <array>
#include <cinttypes>
#include <cmath>
#include <memory>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <stdexcept>
#include <string>
#include <system_error>
#include <vector>

#include "owl.h"
#include "owl_host.h"
#include "owl_sha3.hpp"

namespace fs = std::filesystem;

namespace owl_detail {
// owl_last_error() text for this thread (libowl's error channel)
void set_error_string(const std::string& msg);
}

namespace {

using Words = std::vector<uint32_t>;

struct HostError {
  int code;
  std::string msg;
};

[[noreturn]] void fail(int code, const std::string& msg) { throw HostError{code, msg}; }

void ck(int st) {
  if (st != OWL_OK) { fail(st, owl_last_error()); }
}

uint32_t n_words(uint32_t E) { return (E - 1) / 32 + 1; }
uint64_t res64_of(const Words& w) { return w.size() < 2 ? 0 : ((uint64_t)w[1] << 32) | w[0]; }

// ---- CRC-32 (IEEE, reflected polynomial 0xEDB88320) ----
struct CrcTable {
  uint32_t t[256];
  CrcTable() {
    for (uint32_t i = 0; i < 256; ++i) {
      uint32_t c = i;
      for (int k = 0; k < 8; ++k) { c = (c & 1) ? (0xEDB88320u ^ (c >> 1)) : (c >> 1); }
      t[i] = c;
    }
  }
};
uint32_t crc32(const void* data, size_t size) {
  static const CrcTable tab;
  uint32_t crc = ~0u;
  const unsigned char* p = static_cast<const unsigned char*>(data);
  for (size_t i = 0; i < size; ++i) { crc = tab.t[(crc ^ p[i]) & 0xff] ^ (crc >> 8); }
  return ~crc;
}
uint32_t crc32(const Words& w) { return crc32(w.data(), w.size() * sizeof(uint32_t)); }

// ---- savefiles (src/Saver.cpp) ----
// headers: "OWL PRP 13 N=1*2^E-1 k= block= res64= err= time=" (src/Saver.cpp:22) and
// "OWL LL 13 N=1*2^E-1 k= time=" (src/Saver.cpp:30); the older "OWL PRP 12" and "OWL LL 1"
// headers are read too. Body: u32 CRC32 of the words, then nWords(E) little-endian u32.
constexpr const char* kPrp13 = "OWL PRP 13 N=1*2^%u-1 k=%u block=%u res64=%016" SCNx64 " err=%u time=%lf\n";
constexpr const char* kPrp12 = "OWL PRP 12 %u %u %u %016" SCNx64 " %u %u\n";
constexpr const char* kLL13 = "OWL LL 13 N=1*2^%u-1 k=%u time=%lf\n";
constexpr const char* kLL1 = "OWL LL 1 E=%u k=%u CRC=%u\n";

struct PrpState {
  uint32_t E = 0, k = 0, blockSize = 0;
  uint64_t res64 = 0;
  Words check;
  uint32_t nErrors = 0;
  double elapsed = 0;
};

struct LLState {
  uint32_t E = 0, k = 0;
  Words data;
  double elapsed = 0;
};

std::string str9(uint32_t k) {
  char buf[32];
  std::snprintf(buf, sizeof(buf), "%09u", k);
  return buf;
}

struct FileCloser {
  FILE* f;
  ~FileCloser() {
    if (f) { std::fclose(f); }
  }
};

// writes to "<path>.new" and renames it over <path> (the reference's CycleFile)
void write_file(const fs::path& path, const std::string& header, const Words& w) {
  fs::path tmp = path;
  tmp += ".new";
  {
    FILE* f = std::fopen(tmp.string().c_str(), "wb");
    if (!f) { fail(OWL_ERR_ARG, "cannot write " + tmp.string()); }
    FileCloser fc{f};
    uint32_t crc = crc32(w);
    if (std::fwrite(header.data(), 1, header.size(), f) != header.size() || std::fwrite(&crc, 4, 1, f) != 1 ||
        std::fwrite(w.data(), 4, w.size(), f) != w.size()) {
      fail(OWL_ERR_ARG, "short write " + tmp.string());
    }
  }
  std::error_code ec;
  fs::rename(tmp, path, ec);
  if (ec) { fail(OWL_ERR_ARG, "rename " + tmp.string() + ": " + ec.message()); }
}

std::string read_line(FILE* f) {
  char buf[1024];
  buf[0] = 0;
  if (!std::fgets(buf, sizeof(buf), f)) { return ""; }
  return buf;
}

bool read_words(FILE* f, uint32_t n, uint32_t crc, Words& out) {
  out.assign(n, 0);
  if (std::fread(out.data(), 4, n, f) != n) { return false; }
  return crc32(out) == crc;
}

bool read_prp(const fs::path& path, uint32_t E, PrpState& st) {
  FILE* f = std::fopen(path.string().c_str(), "rb");
  if (!f) { return false; }
  FileCloser fc{f};
  std::string h = read_line(f);
  uint32_t e = 0, k = 0, b = 0, err = 0, crc = 0;
  uint64_t res = 0;
  double el = 0;
  if (std::sscanf(h.c_str(), kPrp13, &e, &k, &b, &res, &err, &el) == 6) {
    if (std::fread(&crc, 4, 1, f) != 1) { return false; }
  } else if (std::sscanf(h.c_str(), kPrp12, &e, &k, &b, &res, &err, &crc) == 6) {
    el = 0;
  } else {
    return false;
  }
  if (e != E) { return false; }
  st.E = e;
  st.k = k;
  st.blockSize = b;
  st.res64 = res;
  st.nErrors = err;
  st.elapsed = el;
  return read_words(f, n_words(E), crc, st.check);
}

bool read_ll(const fs::path& path, uint32_t E, LLState& st) {
  FILE* f = std::fopen(path.string().c_str(), "rb");
  if (!f) { return false; }
  FileCloser fc{f};
  std::string h = read_line(f);
  uint32_t e = 0, k = 0, crc = 0;
  double el = 0;
  if (std::sscanf(h.c_str(), kLL13, &e, &k, &el) == 3) {
    if (std::fread(&crc, 4, 1, f) != 1) { return false; }
  } else if (std::sscanf(h.c_str(), kLL1, &e, &k, &crc) == 3) {
    el = 0;
  } else {
    return false;
  }
  if (e != E) { return false; }
  st.E = e;
  st.k = k;
  st.elapsed = el;
  return read_words(f, n_words(E), crc, st.data);
}

std::string fmt(const char* f, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, f);
  std::vsnprintf(buf, sizeof(buf), f, ap);
  va_end(ap);
  return buf;
}

// A savefile directory: <dir>/<E>/ for PRP, <dir>/ll-<E>/ for LL (src/Saver.cpp:160-166).
class SaveDir {
 public:
  SaveDir(const char* root, uint32_t E, bool prp, uint32_t nKeep)
      : E_(E), prp_(prp), nKeep_(nKeep ? nKeep : 4), prefix_(std::to_string(E) + "-") {
    if (root) {
      base_ = fs::path(root) / (prp ? std::to_string(E) : "ll-" + std::to_string(E));
      fs::create_directories(base_);
    }
  }
  bool enabled() const { return !base_.empty(); }
  const char* kind() const { return prp_ ? "prp" : "ll"; }
  fs::path pathFor(uint32_t k) const { return base_ / (prefix_ + str9(k) + "." + kind()); }
  fs::path unverified() const { return base_ / (prefix_ + "unverified.prp"); }

  // the k's of the regular savefiles, ascending
  std::vector<uint32_t> list() const {
    std::vector<uint32_t> v;
    if (!enabled()) { return v; }
    for (const auto& ent : fs::directory_iterator(base_)) {
      if (!ent.is_regular_file()) { continue; }
      std::string name = ent.path().filename().string();
      std::string suffix = std::string(".") + kind();
      if (name.rfind(prefix_, 0) != 0 || name.size() <= prefix_.size() + suffix.size() ||
          name.compare(name.size() - suffix.size(), suffix.size(), suffix) != 0) {
        continue;
      }
      std::string id = name.substr(prefix_.size(), name.size() - prefix_.size() - suffix.size());
      if (id.empty() || id.find_first_not_of("0123456789") != std::string::npos) { continue; }
      v.push_back((uint32_t)std::stoul(id));
    }
    std::sort(v.begin(), v.end());
    return v;
  }

  fs::path mostRecent() const {
    std::error_code ec;
    if (prp_ && fs::is_regular_file(unverified(), ec)) { return unverified(); }
    auto v = list();
    return v.empty() ? fs::path() : pathFor(v.back());
  }

  void moveToTrash(const fs::path& p) const {
    std::error_code ec;
    fs::path bad = p;
    bad += ".bad";
    fs::rename(p, bad, ec);
  }

  void dropMostRecent() const {
    fs::path p = mostRecent();
    if (!p.empty()) { moveToTrash(p); }
  }

  // src/Saver.cpp:142-156 roundNumberScore and 245-272 trimFiles: drop the file whose removal
  // leaves the smallest gap, favouring round iteration counts
  static double roundScore(uint32_t x) {
    if (x == 0) { return 1; }
    double score = 0;
    while (x % 10 == 0) {
      x /= 10;
      ++score;
    }
    if (x % 5 == 0) { score += .7; }
    if (x % 2 == 0) { score += .3; }
    return score;
  }
  void trim() const {
    auto v = list();
    while (v.size() > nKeep_) {
      int best = -1;
      double bestSpan = 1e20;
      uint32_t prevK = 0;
      for (size_t i = 0; i + 1 < v.size(); ++i) {
        double bias = std::min(1.0, roundScore(v[i]) - 4);
        double span = (double)(v[i + 1] - prevK) * bias;
        prevK = v[i];
        if (span < bestSpan) {
          bestSpan = span;
          best = (int)i;
        }
      }
      std::error_code ec;
      fs::remove(pathFor(v[best]), ec);
      v.erase(v.begin() + best);
    }
  }

  void savePrp(const PrpState& s) const {
    write_file(pathFor(s.k), fmt(kPrp13, E_, s.k, s.blockSize, s.res64, s.nErrors, s.elapsed), s.check);
    trim();
    std::error_code ec;
    fs::remove(unverified(), ec);
  }
  void savePrpUnverified(const PrpState& s) const {
    write_file(unverified(), fmt(kPrp13, E_, s.k, s.blockSize, s.res64, s.nErrors, s.elapsed), s.check);
  }
  void saveLL(const LLState& s) const {
    write_file(pathFor(s.k), fmt(kLL13, E_, s.k, s.elapsed), s.data);
    trim();
  }

  // src/Saver.cpp:212-243: the most recent good file; a bad one is moved to *.bad and the next tried
  bool loadPrp(PrpState& s) const {
    for (int i = 0; i < 2 && enabled(); ++i) {
      fs::path p = mostRecent();
      if (p.empty()) { return false; }
      if (read_prp(p, E_, s)) { return true; }
      moveToTrash(p);
    }
    return false;
  }
  bool loadLL(LLState& s) const {
    for (int i = 0; i < 2 && enabled(); ++i) {
      fs::path p = mostRecent();
      if (p.empty()) { return false; }
      if (read_ll(p, E_, s)) { return true; }
      moveToTrash(p);
    }
    return false;
  }

 private:
  uint32_t E_;
  bool prp_;
  uint32_t nKeep_;
  std::string prefix_;
  fs::path base_;
};

// ---- the engine, as the reference's Gpu sees it ----
class HostGpu {
 public:
  HostGpu(int device, uint32_t E, uint32_t W, uint32_t H, int split = 0, uint32_t colVariant = 0) : E_(E) {
    ck(owl_plan_create(device, E, W, H, &plan_));
    if (split) { ck(owl_plan_set_split(plan_, split)); }
    if (colVariant) { ck(owl_plan_set_column_variant(plan_, colVariant)); }
    ck(owl_buf_alloc(plan_, &data));
    ck(owl_buf_alloc(plan_, &check));
    ck(owl_buf_alloc(plan_, &aux));
  }
  ~HostGpu() {
    if (plan_) { owl_plan_destroy(plan_); }
  }
  HostGpu(const HostGpu&) = delete;
  HostGpu& operator=(const HostGpu&) = delete;

  void writeIn(int32_t* b, const Words& w) { ck(owl_write_words(plan_, b, w.data())); }
  Words readOut(const int32_t* b) {
    Words w(n_words(E_));
    ck(owl_read_words(plan_, b, w.data()));
    return w;
  }
  void squareLoop(int32_t* out, const int32_t* in, uint32_t n, uint32_t flags = 0) {
    ck(owl_square(plan_, out, in, n, flags));
  }
  void modMul(int32_t* a, const int32_t* b, bool mul3 = false) { ck(owl_modmul(plan_, a, b, mul3 ? 1 : 0)); }
  bool isEqual(const int32_t* a, const int32_t* b) {
    int eq = 0;
    ck(owl_is_equal(plan_, a, b, &eq));
    return eq != 0;
  }
  uint64_t residue(const int32_t* b) {
    uint64_t r = 0;
    ck(owl_res64(plan_, b, &r));
    return r;
  }
  void copy(int32_t* dst, const int32_t* src) { ck(owl_buf_copy(plan_, dst, src)); }
  // per-squaring round-off maxima recorded since the last call (Gpu::readROE, src/Gpu.cpp:624-637)
  std::vector<float> readRoe() {
    std::vector<float> v(1u << 16);
    uint32_t n = 0;
    ck(owl_read_roe(plan_, v.data(), (uint32_t)v.size(), &n));
    v.resize(n);
    return v;
  }

  // src/Gpu.cpp:738-765: data = 3 * check^(2^B - 1), rebuilt from the saved check
  void writeState(const Words& checkWords, uint32_t B) {
    writeIn(check, checkWords);
    copy(data, check);
    copy(aux, check);
    uint32_t n = 1;
    for (; B % (2 * n) == 0; n *= 2) {
      squareLoop(data, data, n, OWL_SQ_NO_ROE);
      modMul(data, aux);
      copy(aux, data);
    }
    uint32_t blocks = B / n;
    if (blocks < 2) { fail(OWL_ERR_ARG, "block size must not be a power of two"); }
    for (uint32_t i = 0; i + 2 < blocks; ++i) {
      squareLoop(data, data, n, OWL_SQ_NO_ROE);
      modMul(data, aux);
    }
    squareLoop(data, data, n, OWL_SQ_NO_ROE);
    modMul(data, aux, true);
  }

  // src/Gpu.cpp:767-771
  bool doCheck(uint32_t B) {
    squareLoop(aux, check, B, OWL_SQ_MUL3 | OWL_SQ_NO_ROE);
    modMul(check, data);
    return isEqual(check, aux);
  }

  // reference Gpu::expMul(Buffer A, h, Buffer B): A := A^h * B
  void expMul(int32_t* a, uint64_t h, const int32_t* b) { ck(owl_exp_mul(plan_, a, h, b)); }
  // reference Gpu::expMul(Words A, h, Words B, doSquareB) (src/Gpu.cpp:839-847): A^h * (B or B^2)
  Words expMul(const Words& A, uint64_t h, const Words& B, bool doSquareB) {
    writeIn(check, B);
    if (doSquareB) { squareLoop(check, check, 1); }
    writeIn(data, A);
    expMul(data, h, check);
    return readOut(data);
  }
  // reference Gpu::expExp2 (src/Gpu.cpp:813-831): A^(2^n), in blocks of squarings
  Words expExp2(const Words& A, uint32_t n) {
    writeIn(data, A);
    for (uint32_t k = 0; k < n;) {
      const uint32_t its = std::min(1000u, n - k);
      squareLoop(data, data, its, OWL_SQ_NO_ROE);
      k += its;
    }
    return readOut(data);
  }
  int32_t* allocBuf() {
    int32_t* b = nullptr;
    ck(owl_buf_alloc(plan_, &b));
    return b;
  }
  void freeBuf(int32_t* b) { owl_buf_free(plan_, b); }

  void injectFault(int32_t* b) {
    uint32_t N = 0;
    ck(owl_plan_shape(plan_, &N, nullptr, nullptr));
    std::vector<int32_t> d(N);
    ck(owl_read_digits(plan_, b, d.data()));
    d[777 % N] ^= 1;
    ck(owl_write_digits(plan_, b, d.data()));
  }

  int32_t* data = nullptr;
  int32_t* check = nullptr;
  int32_t* aux = nullptr;

 private:
  uint32_t E_;
  owl_plan* plan_ = nullptr;
};

// ---- PRP proofs (src/Proof.cpp, src/Proof.h) ----
using Hash4 = std::array<uint64_t, 4>;

Words make_words(uint32_t E, uint32_t v) {
  Words w(n_words(E), 0);
  w[0] = v;
  return w;
}
// SHA3-256 of the first (E-1)/8+1 bytes of the words, optionally after a 32-byte prefix (src/Proof.cpp:22-28)
Hash4 hash_words(uint32_t E, const Words& w) {
  owl::Sha3_256 h;
  h.update(w.data(), (E - 1) / 8 + 1);
  return h.finish();
}
Hash4 hash_words(uint32_t E, const Hash4& prefix, const Words& w) {
  owl::Sha3_256 h;
  h.update(prefix.data(), sizeof(prefix));
  h.update(w.data(), (E - 1) / 8 + 1);
  return h.finish();
}

// "PRP PROOF\nVERSION=2\nHASHSIZE=64\nPOWER=%u\nNUMBER=M%u\n" + B + middles, (E-1)/8+1 bytes each
// (src/Proof.h:42-49, src/Proof.cpp:62-86)
constexpr const char* kProofHeader = "PRP PROOF\nVERSION=2\nHASHSIZE=64\nPOWER=%u\nNUMBER=M%u%c";

struct Proof {
  uint32_t E = 0;
  Words B;
  std::vector<Words> middles;

  void save(const fs::path& path) const {
    FILE* f = std::fopen(path.string().c_str(), "wb");
    if (!f) { fail(OWL_ERR_ARG, "cannot write " + path.string()); }
    FileCloser fc{f};
    std::fprintf(f, kProofHeader, (unsigned)middles.size(), E, '\n');
    const size_t nb = (E - 1) / 8 + 1;
    bool ok = std::fwrite(B.data(), 1, nb, f) == nb;
    for (const Words& w : middles) { ok = ok && std::fwrite(w.data(), 1, nb, f) == nb; }
    if (!ok) { fail(OWL_ERR_ARG, "short write " + path.string()); }
  }

  static Proof load(const fs::path& path) {
    FILE* f = std::fopen(path.string().c_str(), "rb");
    if (!f) { fail(OWL_ERR_READ, "cannot open " + path.string()); }
    FileCloser fc{f};
    unsigned power = 0, E = 0;
    char c = 0;
    if (std::fscanf(f, kProofHeader, &power, &E, &c) != 3 || c != '\n' || power == 0 || power > 12 || E < 32) {
      fail(OWL_ERR_READ, "invalid proof header");
    }
    const size_t nb = (E - 1) / 8 + 1;
    auto readWords = [&]() {
      Words w(n_words(E), 0);
      if (std::fread(w.data(), 1, nb, f) != nb) { fail(OWL_ERR_READ, "truncated proof"); }
      return w;
    };
    Proof p;
    p.E = E;
    p.B = readWords();
    for (unsigned i = 0; i < power; ++i) { p.middles.push_back(readWords()); }
    return p;
  }

  // src/Proof.cpp:88-128
  bool verify(HostGpu& gpu, const std::vector<uint64_t>& hashes, bool* isPrime) const {
    const uint32_t power = (uint32_t)middles.size();
    *isPrime = (B == make_words(E, 9));
    Words A = make_words(E, 3), Bw = B;
    Hash4 hash = hash_words(E, Bw);
    uint32_t span = E;
    for (uint32_t i = 0; i < power; ++i, span = (span + 1) / 2) {
      const Words& M = middles[i];
      hash = hash_words(E, hash, M);
      const uint64_t h = hash[0];
      if (hashes.size() > i && h != hashes[i]) { return false; }
      Bw = gpu.expMul(M, h, Bw, span % 2 != 0);
      A = gpu.expMul(A, h, M, false);
    }
    A = gpu.expExp2(A, span);
    return A == Bw;
  }
};

// The residues a power-p proof needs (src/Proof.cpp:132-185): every sum of a subset of the
// spans (E+1)/2, then halved (rounding up) p-1 times, with the empty sum replaced by E.
std::vector<uint32_t> proof_points(uint32_t E, uint32_t power) {
  std::vector<uint32_t> pts{0};
  for (uint32_t p = 0, span = (E + 1) / 2; p < power; ++p, span = (span + 1) / 2) {
    for (size_t i = 0, end = pts.size(); i < end; ++i) { pts.push_back(pts[i] + span); }
  }
  pts.front() = E;
  std::sort(pts.begin(), pts.end());
  return pts;
}

bool proof_in_points(uint32_t E, uint32_t power, uint32_t k) {  // src/Proof.cpp:187-200
  if (k == E) { return true; }
  uint32_t start = 0;
  for (uint32_t p = 0, span = (E + 1) / 2; p < power; ++p, span = (span + 1) / 2) {
    if (k > start + span) {
      start += span;
    } else if (k == start + span) {
      return true;
    }
  }
  return false;
}

class ProofSet {
 public:
  // residues live in <root>/<E>/proof/<k> (src/Proof.h:70), like the savefiles
  ProofSet(const fs::path& root, uint32_t E, uint32_t power) : E(E), power(power), dir_(root / std::to_string(E) / "proof") {
    if (power == 0 || power > 12) { fail(OWL_ERR_ARG, "invalid proof power"); }
    fs::create_directories(dir_);
    points_ = proof_points(E, power);
    points_.push_back(UINT32_MAX);  // guard
  }
  const uint32_t E, power;

  uint32_t next(uint32_t k) const { return *std::upper_bound(points_.begin(), points_.end(), k); }
  uint32_t point(size_t i) const { return points_[i]; }

  // file: u32 CRC32 of the words, then E/32+1 words (File::writeChecked, src/File.h:218-222)
  void save(uint32_t k, const Words& w) const {
    if (!k || k > E || !proof_in_points(E, power, k)) { fail(OWL_ERR_ARG, "not a proof point"); }
    const fs::path tmp = file(k).string() + ".tmp";
    {
      FILE* f = std::fopen(tmp.string().c_str(), "wb");
      if (!f) { fail(OWL_ERR_ARG, "cannot write " + tmp.string()); }
      FileCloser fc{f};
      const uint32_t crc = crc32(w);
      if (std::fwrite(&crc, 4, 1, f) != 1 || std::fwrite(w.data(), 4, w.size(), f) != w.size()) {
        fail(OWL_ERR_ARG, "short write " + tmp.string());
      }
    }
    fs::rename(tmp, file(k));
    if (load(k) != w) { fail(OWL_ERR_READ, "proof residue read-back differs"); }
  }
  Words load(uint32_t k) const {
    FILE* f = std::fopen(file(k).string().c_str(), "rb");
    if (!f) { fail(OWL_ERR_READ, "missing proof residue " + std::to_string(k)); }
    FileCloser fc{f};
    uint32_t crc = 0;
    Words w(E / 32 + 1);
    if (std::fread(&crc, 4, 1, f) != 1 || std::fread(w.data(), 4, w.size(), f) != w.size() || crc != crc32(w)) {
      fail(OWL_ERR_READ, "bad proof residue " + std::to_string(k));
    }
    return w;
  }
  bool fileExists(uint32_t k) const {
    std::error_code ec;
    return fs::file_size(file(k), ec) == (uintmax_t)(E / 32 + 2) * 4 && !ec;
  }
  // every residue up to limitK is present, the last one readable (src/Proof.cpp:217-240)
  bool isValidTo(uint32_t limitK) const {
    auto it = std::upper_bound(points_.begin(), points_.end(), limitK);
    if (it == points_.begin()) { return true; }
    --it;
    try {
      load(*it);
    } catch (const HostError&) {
      return false;
    }
    while (it != points_.begin()) {
      if (!fileExists(*--it)) { return false; }
    }
    return true;
  }
  // the largest power <= `power` whose residues up to k are all on disk (src/Proof.cpp:210-215)
  static uint32_t effectivePower(const fs::path& root, uint32_t E, uint32_t power, uint32_t k) {
    for (uint32_t p = power; p > 0; --p) {
      if (ProofSet(root, E, p).isValidTo(k)) { return p; }
    }
    return 0;
  }

  // src/Proof.cpp:256-297: middles M_p folded from the residues with the running hashes
  Proof computeProof(HostGpu& gpu, std::vector<uint64_t>& hashes) const {
    Proof pr;
    pr.E = E;
    pr.B = load(E);
    Hash4 hash = hash_words(E, pr.B);
    std::vector<int32_t*> bufs;
    for (uint32_t i = 0; i < power; ++i) { bufs.push_back(gpu.allocBuf()); }
    struct Free {
      HostGpu& g;
      std::vector<int32_t*>& b;
      ~Free() {
        for (int32_t* x : b) { g.freeBuf(x); }
      }
    } freeBufs{gpu, bufs};
    hashes.clear();
    for (uint32_t p = 0; p < power; ++p) {
      size_t it = 0;
      const uint32_t s = 1u << (power - p - 1);
      for (uint32_t i = 0; i < (1u << p); ++i) {
        gpu.writeIn(bufs[it++], load(points_[s * (i * 2 + 1) - 1]));
        for (uint32_t k = 0; i & (1u << k); ++k) {
          --it;
          gpu.expMul(bufs[it - 1], hashes[p - 1 - k], bufs[it]);
        }
      }
      if (it != 1) { fail(OWL_ERR_ARG, "proof fold"); }
      Words w = gpu.readOut(bufs[0]);
      pr.middles.push_back(w);
      hash = hash_words(E, hash, w);
      hashes.push_back(hash[0]);
    }
    return pr;
  }

 private:
  fs::path file(uint32_t k) const { return dir_ / std::to_string(k); }
  fs::path dir_;
  std::vector<uint32_t> points_;
};

// Gpu::saveProof (src/Gpu.cpp:1150-1166): generate into proof-tmp/, verify with the same hashes,
// then move to proof/<E>-<power>.proof
fs::path save_proof(HostGpu& gpu, const ProofSet& ps, const fs::path& root) {
  for (int retry = 0; retry < 2; ++retry) {
    std::vector<uint64_t> hashes;
    Proof pr = ps.computeProof(gpu, hashes);
    const std::string name = std::to_string(ps.E) + "-" + std::to_string(ps.power) + ".proof";
    fs::create_directories(root / "proof-tmp");
    fs::create_directories(root / "proof");
    const fs::path tmp = root / "proof-tmp" / name, out = root / "proof" / name;
    pr.save(tmp);
    bool isPrime = false;
    if (Proof::load(tmp).verify(gpu, hashes, &isPrime)) {
      fs::rename(tmp, out);
      return out;
    }
  }
  fail(OWL_ERR_READ, "bad proof generation");
}

uint32_t baseCheckStep(uint32_t B) {  // src/Gpu.cpp:347-356
  switch (B) {
    case 200: return 40000;
    case 400: return 160000;
    case 500: return 200000;
    case 1000: return 1000000;
    default: return B * 1000;
  }
}

bool equals9(const Words& w) {  // src/Gpu.cpp:1036-1040
  if (w.empty() || w[0] != 9) { return false; }
  for (size_t i = 1; i < w.size(); ++i) {
    if (w[i]) { return false; }
  }
  return true;
}

// src/Gpu.cpp:1120-1148: x / 3 mod 2^E - 1, twice
void div3(uint32_t E, Words& w) {
  uint32_t r = 0;
  for (uint32_t x : w) { r += x % 3; }
  r = (3 - r % 3) % 3;
  const int top = E % 32;
  {
    uint64_t x = ((uint64_t)r << top) + w.back();
    w.back() = (uint32_t)(x / 3);
    r = (uint32_t)(x % 3);
  }
  for (size_t i = w.size() - 1; i-- > 0;) {
    uint64_t x = ((uint64_t)r << 32) + w[i];
    w[i] = (uint32_t)(x / 3);
    r = (uint32_t)(x % 3);
  }
}

std::string hex64words(const Words& w) {
  std::string s;
  for (int i = 63; i >= 0; --i) {
    char b[16];
    std::snprintf(b, sizeof(b), "%08x", i < (int)w.size() ? w[i] : 0u);
    s += b;
  }
  return s;
}

// Round-off statistics of a sample of per-squaring maxima (src/Gpu.cpp:311-327 roeStat and the
// RoeInfo Gumbel fit of src/Gpu.h:62-81): beta = sd * sqrt(6) / pi, miu = mean - gamma * beta,
// Z(x) = (x - miu) / beta.
struct RoeInfo {
  uint32_t N = 0;
  double max = 0, mean = 0, sd = 0, beta = 0, miu = 0;
  explicit RoeInfo(const std::vector<float>& v) {
    double sum = 0, sum2 = 0;
    for (float f : v) {
      const double x = f;
      max = std::max(max, x);
      sum += x;
      sum2 += x * x;
    }
    N = (uint32_t)v.size();
    if (!N) { return; }
    sd = std::sqrt(std::max(0.0, N * sum2 - sum * sum)) / N;
    mean = sum / N;
    beta = sd * 0.779696801233676;       // sqrt(6) / pi
    miu = mean - beta * 0.577215664901533;  // Euler-Mascheroni
  }
  double z(double x = 0.5) const { return N && beta > 0 ? (x - miu) / beta : 0.0; }
};

// Which squarings feed the statistics: the reference measures the round-off on a few iterations
// only (wantROE, src/Gpu.cpp:1459-1464, 1026): 2,000 iterations once the first 30 of a run are
// past, then 400 after every log step; the other squarings run without the measurement.
struct RoeSampler {
  uint32_t skipTo = 0;
  uint32_t want = 0;
  std::vector<float> sample;
  double zSum = 0, zN = 0;
  void start(uint32_t startK) {
    skipTo = startK + 30;
    want = 2000;
  }
  // n squarings from iteration k with `flags`: the ones the sample wants measure their round-off,
  // the others run the kernels without the measurement (OWL_SQ_NO_ROE). With `whole`, a call the
  // sample reaches is measured whole (the PRP loop's calls are blocks of B squarings: this keeps the
  // number of distinct squaring graphs a plan caches small); its first squarings before skipTo are
  // left out of the sample.
  template <typename G> void square(G& gpu, int32_t* buf, uint32_t k, uint32_t n, uint32_t flags, bool whole = false) {
    if (whole) {
      if (want > 0 && k + n > skipTo) {
        gpu.readRoe();  // drops what other calls (the modMul) recorded
        gpu.squareLoop(buf, buf, n, flags);
        std::vector<float> v = gpu.readRoe();
        const size_t drop = k < skipTo ? std::min<size_t>(skipTo - k, v.size()) : 0;
        v.erase(v.begin(), v.begin() + drop);
        add(n, std::move(v));
      } else {
        gpu.squareLoop(buf, buf, n, flags | OWL_SQ_NO_ROE);
      }
      return;
    }
    const uint32_t skip = k < skipTo ? std::min(n, skipTo - k) : 0;
    const uint32_t take = std::min(n - skip, want);
    if (skip) { gpu.squareLoop(buf, buf, skip, flags | OWL_SQ_NO_ROE); }
    if (take) {
      gpu.readRoe();  // drops what other calls (the modMul) recorded
      gpu.squareLoop(buf, buf, take, flags);
      add(take, gpu.readRoe());
    }
    if (n - skip - take) { gpu.squareLoop(buf, buf, n - skip - take, flags | OWL_SQ_NO_ROE); }
  }
  void add(uint32_t iters, std::vector<float> v) {
    want = iters >= want ? 0 : want - iters;
    sample.insert(sample.end(), v.begin(), v.end());
  }
  // the statistics of the sample since the last log step; records them in the run result
  RoeInfo logStep(owl_run_result& res) {
    RoeInfo info(sample);
    sample.clear();
    want = 400;
    if (info.N) {
      res.roe_n += info.N;
      res.roe_max = std::max(res.roe_max, (float)info.max);
      res.roe_z = (float)info.z();
      zSum += info.z() * info.N;
      zN += info.N;
      res.roe_z_avg = (float)(zSum / zN);
    }
    return info;
  }
};

struct Log {
  const owl_run_opts& o;
  void checkpoint(uint32_t k, uint64_t res) {
    if (o.res_n && o.res_cap && o.res_k && o.res_res64 && *o.res_n < o.res_cap) {
      o.res_k[*o.res_n] = k;
      o.res_res64[*o.res_n] = res;
      ++*o.res_n;
    }
  }
  void line(const std::string& s) {
    if (o.verbose) { std::fprintf(stderr, "%s\n", s.c_str()); }
  }
};

uint32_t roundUp(uint32_t x, uint32_t m) { return ((x + m - 1) / m) * m; }

// Gpu::isPrimePRP (src/Gpu.cpp:1400-1584), with the proof residues and the proof at the end.
void prp(int device, uint32_t E, const owl_run_opts& o, owl_run_result& res) {
  const uint32_t B0 = o.block_size ? o.block_size : 1000;
  const uint32_t logStep = o.log_step ? o.log_step : 20000;
  if (B0 % 100 != 0 || 10000 % B0 != 0 || logStep % B0 != 0) { fail(OWL_ERR_ARG, "block size / log step"); }
  HostGpu gpu(device, E, o.W, o.H, o.split, o.column_variant);
  SaveDir saver(o.save_dir, E, true, o.n_savefiles);
  Log log{o};
  if (o.res_n) { *o.res_n = 0; }
  std::memset(&res, 0, sizeof(res));
  if (o.proof_power && !o.save_dir) { fail(OWL_ERR_ARG, "a proof needs save_dir"); }
  if (o.proof_power > 12) { fail(OWL_ERR_ARG, "invalid proof power"); }

  uint32_t nErrors = 0, nSeqErrors = 0;
  uint64_t lastFailedRes64 = 0;
  bool injected = false;
  for (int attempt = 0;; ++attempt) {  // the reference's "reload:" label
    PrpState st;
    bool fromFile = saver.loadPrp(st);
    if (!fromFile) {
      st = PrpState{E, 0, B0, 3, Words(n_words(E), 0), 0, 0};
      st.check[0] = 1;
    }
    nErrors = std::max(nErrors, st.nErrors);
    const uint32_t B = st.blockSize;
    gpu.writeState(st.check, B);
    uint64_t r0 = gpu.residue(gpu.data);
    if (r0 != st.res64) {
      log.line(fmt("EE %9u on-load: %016" PRIx64 " vs. %016" PRIx64, st.k, r0, st.res64));
      if (fromFile && st.k) {
        saver.dropMostRecent();
        continue;
      }
      fail(OWL_ERR_READ, "Error on load");
    }
    log.line(fmt("OK %9u on-load: blockSize %u, %016" PRIx64, st.k, B, r0));
    const uint32_t base = o.check_step ? o.check_step : baseCheckStep(B);
    const uint32_t checkStep = nErrors ? std::max(B, base / 2) : base;
    uint32_t k = st.k;
    const uint32_t startK = k, kEnd = E, kEndEnd = roundUp(kEnd, B);
    // proof residues (src/Gpu.cpp:1428-1431, 1450, 1486-1493)
    std::unique_ptr<ProofSet> proofSet;
    if (o.proof_power) {
      const uint32_t power = ProofSet::effectivePower(o.save_dir, E, o.proof_power, k);
      if (power != o.proof_power) { log.line(fmt("Proof using power %u (vs %u)", power, o.proof_power)); }
      if (power) { proofSet = std::make_unique<ProofSet>(o.save_dir, E, power); }
    }
    uint32_t persistK = proofSet ? proofSet->next(k) : UINT32_MAX;
    RoeSampler roe;
    roe.start(startK);
    bool skipNextCheckUpdate = false;
    bool reload = false;
    Words finalWords;
    while (true) {
      if (skipNextCheckUpdate) {
        skipNextCheckUpdate = false;
      } else if (k % B == 0) {
        gpu.modMul(gpu.check, gpu.data);
      }
      // squarings up to the next point where the loop looks at the data
      uint32_t next = roundUp(k + 1, B);
      if (k < kEnd && kEnd < next) { next = kEnd; }
      if (persistK > k && persistK < next) { next = persistK; }
      roe.square(gpu, gpu.data, k, next - k, 0, true);
      k = next;
      if (k == persistK) {
        proofSet->save(k, gpu.readOut(gpu.data));
        persistK = proofSet->next(k);
      }
      if (o.inject_fault_k && !injected && k >= o.inject_fault_k) {
        injected = true;
        gpu.injectFault(gpu.data);
        log.line(fmt("fault injected at %u", k));
      }
      if (k == kEnd) {
        finalWords = gpu.readOut(gpu.data);
        res.is_prime = equals9(finalWords);
        div3(E, finalWords);
        div3(E, finalWords);
        res.res64 = res64_of(finalWords);
        std::snprintf(res.res2048, sizeof(res.res2048), "%s", hex64words(finalWords).c_str());
        log.line(fmt("%s %8u / %u, %016" PRIx64, res.is_prime ? "PP" : "CC", kEnd, E, res.res64));
      }
      if (k % B != 0) { continue; }
      const bool doStop = o.stop_after && k - startK >= o.stop_after;
      const bool doCheck = doStop || (k % checkStep == 0) || (k >= kEndEnd) || (k - startK == 2 * B);
      const bool doLog = k % logStep == 0;
      if (!doCheck && !doLog) { continue; }
      const uint64_t r = gpu.residue(gpu.data);
      log.checkpoint(k, r);
      // src/Gpu.cpp:1011-1025 doBigLog: Z of the sampled round-off, and the danger warning
      const RoeInfo ri = roe.logStep(res);
      const std::string zs = ri.N ? fmt(" Z=%.0f (avg %.1f)", ri.z(), (double)res.roe_z_avg) : std::string();
      if (ri.N > 2 && ri.z() < 20) {
        ++res.n_danger_roe;
        log.line(fmt("Danger ROE! Z=%.1f is too small, increase precision or FFT size!", ri.z()));
      }
      Words rawCheck = gpu.readOut(gpu.check);
      if (!doCheck) {
        if (saver.enabled()) { saver.savePrpUnverified({E, k, B, r, rawCheck, nErrors, 0}); }
        log.line(fmt("   %9u %016" PRIx64 "%s", k, r, zs.c_str()));
        continue;
      }
      const bool ok = gpu.doCheck(B);
      if (ok) {
        nSeqErrors = 0;
        skipNextCheckUpdate = true;
        if (k < kEnd && saver.enabled()) { saver.savePrp({E, k, B, r, rawCheck, nErrors, 0}); }
        log.line(fmt("OK %9u %016" PRIx64 "%s", k, r, zs.c_str()));
        if (k >= kEndEnd) {
          if (proofSet) {
            const fs::path pf = save_proof(gpu, *proofSet, o.save_dir);
            res.proof_power = proofSet->power;
            std::snprintf(res.proof_file, sizeof(res.proof_file), "%s", pf.string().c_str());
            log.line("proof " + pf.string());
          }
          res.finished = 1;
          res.k = k;
          res.n_errors = nErrors;
          return;
        }
      } else {
        ++nErrors;
        log.line(fmt("EE %9u %016" PRIx64 "%s (check failed, %u errors)", k, r, zs.c_str(), nErrors));
        if (++nSeqErrors > 2) { fail(OWL_ERR_READ, "too many errors"); }
        if (r == lastFailedRes64) { fail(OWL_ERR_READ, "consistent error"); }
        lastFailedRes64 = r;
        if (!doStop) {
          reload = true;
          break;
        }
      }
      if (doStop) {
        res.finished = 0;
        res.k = k;
        res.n_errors = nErrors;
        return;
      }
    }
    if (!reload) { return; }
  }
}

// Gpu::isPrimeLL (src/Gpu.cpp:1586-1663)
void ll(int device, uint32_t E, const owl_run_opts& o, owl_run_result& res) {
  const uint32_t logStep = o.log_step ? o.log_step : 10000;
  HostGpu gpu(device, E, o.W, o.H, o.split, o.column_variant);
  SaveDir saver(o.save_dir, E, false, o.n_savefiles);
  Log log{o};
  if (o.res_n) { *o.res_n = 0; }
  std::memset(&res, 0, sizeof(res));
  for (int attempt = 0; attempt < 3; ++attempt) {
    LLState st;
    if (!saver.loadLL(st)) {
      st = LLState{E, 0, Words(n_words(E), 0), 0};
      st.data[0] = 4;
    }
    gpu.writeIn(gpu.data, st.data);
    if (gpu.residue(gpu.data) != res64_of(st.data)) { fail(OWL_ERR_READ, "Invalid savefile (res64)"); }
    uint32_t k = st.k;
    const uint32_t startK = k, kEnd = E - 2;
    bool reload = false;
    // round-off statistics per log step (the reference computes none in its LL loop, src/Gpu.cpp:1588;
    // the same sampling, Z and danger warning as the PRP loop's are used here)
    RoeSampler roe;
    roe.start(startK);
    while (true) {
      uint32_t next = roundUp(k + 1, logStep);
      if (next > kEnd) { next = kEnd; }
      if (o.stop_after && next - startK > o.stop_after) { next = std::max(k + 1, startK + o.stop_after); }
      roe.square(gpu, gpu.data, k, next - k, OWL_SQ_LL);
      k = next;
      const bool doStop = (k >= kEnd) || (o.stop_after && k - startK >= o.stop_after);
      Words w = gpu.readOut(gpu.data);
      bool allZero = true, allOnes = true;
      for (size_t i = 0; i < w.size(); ++i) {
        allZero &= (w[i] == 0);
        uint32_t full = (i + 1 == w.size() && E % 32) ? ((1u << (E % 32)) - 1) : 0xffffffffu;
        allOnes &= (w[i] == full);
      }
      const bool isZero = allZero || allOnes;
      uint64_t r = isZero ? 0 : res64_of(w);
      if (isZero && k < kEnd) {
        log.line(fmt("Error: early ZERO @ %u", k));
        reload = true;
        break;
      }
      if (!isZero && saver.enabled()) { saver.saveLL({E, k, w, 0}); }
      log.checkpoint(k, r);
      const RoeInfo ri = roe.logStep(res);
      if (ri.N > 2 && ri.z() < 20) {
        ++res.n_danger_roe;
        log.line(fmt("Danger ROE! Z=%.1f is too small, increase precision or FFT size!", ri.z()));
      }
      log.line(fmt("%9u %016" PRIx64 "%s", k, r,
                   ri.N ? fmt(" Z=%.0f (avg %.1f)", ri.z(), (double)res.roe_z_avg).c_str() : ""));
      if (k >= kEnd) {
        res.is_prime = isZero;
        res.res64 = r;
        res.finished = 1;
        res.k = k;
        return;
      }
      if (doStop) {
        res.finished = 0;
        res.k = k;
        res.res64 = r;
        return;
      }
    }
    if (!reload) { return; }
  }
  fail(OWL_ERR_READ, "repeated early zero");
}

template <typename F> int guarded(F&& f) {
  try {
    f();
    return OWL_OK;
  } catch (const HostError& e) {
    owl_detail::set_error_string(e.msg);
    return e.code;
  } catch (const std::exception& e) {
    owl_detail::set_error_string(e.what());
    return OWL_ERR_ARG;
  }
}

}  // namespace

extern "C" {

int owl_prp_run(int device, uint32_t E, const owl_run_opts* opts, owl_run_result* out) {
  return guarded([&] {
    if (!opts || !out) { fail(OWL_ERR_ARG, "null argument"); }
    prp(device, E, *opts, *out);
  });
}

int owl_ll_run(int device, uint32_t E, const owl_run_opts* opts, owl_run_result* out) {
  return guarded([&] {
    if (!opts || !out) { fail(OWL_ERR_ARG, "null argument"); }
    ll(device, E, *opts, *out);
  });
}

void owl_sha3_256(const void* data, size_t size, uint8_t out[32]) {
  owl::Sha3_256 h;
  h.update(data, size);
  owl::Sha3_256::digest_bytes(h.finish(), out);
}

int owl_proof_points(uint32_t E, uint32_t power, uint32_t* points, uint32_t cap, uint32_t* n) {
  return guarded([&] {
    if (power == 0 || power > 12 || E < 3 || !(E & 1)) { fail(OWL_ERR_ARG, "invalid exponent or proof power"); }
    const std::vector<uint32_t> pts = proof_points(E, power);
    if (n) { *n = (uint32_t)pts.size(); }
    for (uint32_t i = 0; points && i < cap && i < pts.size(); ++i) { points[i] = pts[i]; }
  });
}

int owl_proof_verify(int device, const char* proof_file, int* valid, int* is_prime) {
  return guarded([&] {
    if (!proof_file || !valid || !is_prime) { fail(OWL_ERR_ARG, "null argument"); }
    const Proof pr = Proof::load(proof_file);
    HostGpu gpu(device, pr.E, 0, 0);
    bool prime = false;
    *valid = pr.verify(gpu, {}, &prime) ? 1 : 0;
    *is_prime = prime ? 1 : 0;
  });
}

int owl_prp_save(const char* dir, uint32_t E, uint32_t k, uint32_t block, uint64_t res64, const uint32_t* check,
                 uint32_t nErrors, double elapsed) {
  return guarded([&] {
    if (!dir || !check) { fail(OWL_ERR_ARG, "null argument"); }
    SaveDir s(dir, E, true, 4);
    s.savePrp({E, k, block, res64, Words(check, check + n_words(E)), nErrors, elapsed});
  });
}

int owl_prp_load(const char* dir, uint32_t E, uint32_t* k, uint32_t* block, uint64_t* res64, uint32_t* check,
                 uint32_t* nErrors, double* elapsed) {
  return guarded([&] {
    if (!dir || !k || !block || !res64 || !check || !nErrors || !elapsed) { fail(OWL_ERR_ARG, "null argument"); }
    SaveDir s(dir, E, true, 4);
    PrpState st;
    if (!s.loadPrp(st)) { fail(OWL_ERR_READ, "no readable savefile"); }
    *k = st.k;
    *block = st.blockSize;
    *res64 = st.res64;
    std::memcpy(check, st.check.data(), st.check.size() * sizeof(uint32_t));
    *nErrors = st.nErrors;
    *elapsed = st.elapsed;
  });
}

int owl_ll_save(const char* dir, uint32_t E, uint32_t k, const uint32_t* data, double elapsed) {
  return guarded([&] {
    if (!dir || !data) { fail(OWL_ERR_ARG, "null argument"); }
    SaveDir s(dir, E, false, 4);
    s.saveLL({E, k, Words(data, data + n_words(E)), elapsed});
  });
}

int owl_ll_load(const char* dir, uint32_t E, uint32_t* k, uint32_t* data, double* elapsed) {
  return guarded([&] {
    if (!dir || !k || !data || !elapsed) { fail(OWL_ERR_ARG, "null argument"); }
    SaveDir s(dir, E, false, 4);
    LLState st;
    if (!s.loadLL(st)) { fail(OWL_ERR_READ, "no readable savefile"); }
    *k = st.k;
    std::memcpy(data, st.data.data(), st.data.size() * sizeof(uint32_t));
    *elapsed = st.elapsed;
  });
}

uint32_t owl_crc32(const void* data, size_t size) { return crc32(data, size); }

}  // extern "C"
