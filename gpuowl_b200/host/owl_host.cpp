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
#include <cinttypes>
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
  HostGpu(int device, uint32_t E, uint32_t W, uint32_t H, int split = 0) : E_(E) {
    ck(owl_plan_create(device, E, W, H, &plan_));
    if (split) { ck(owl_plan_set_split(plan_, 1)); }
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

  // src/Gpu.cpp:738-765: data = 3 * check^(2^B - 1), rebuilt from the saved check
  void writeState(const Words& checkWords, uint32_t B) {
    writeIn(check, checkWords);
    copy(data, check);
    copy(aux, check);
    uint32_t n = 1;
    for (; B % (2 * n) == 0; n *= 2) {
      squareLoop(data, data, n);
      modMul(data, aux);
      copy(aux, data);
    }
    uint32_t blocks = B / n;
    if (blocks < 2) { fail(OWL_ERR_ARG, "block size must not be a power of two"); }
    for (uint32_t i = 0; i + 2 < blocks; ++i) {
      squareLoop(data, data, n);
      modMul(data, aux);
    }
    squareLoop(data, data, n);
    modMul(data, aux, true);
  }

  // src/Gpu.cpp:767-771
  bool doCheck(uint32_t B) {
    squareLoop(aux, check, B, OWL_SQ_MUL3);
    modMul(check, data);
    return isEqual(check, aux);
  }

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

// Gpu::isPrimePRP (src/Gpu.cpp:1400-1584) without proof generation.
void prp(int device, uint32_t E, const owl_run_opts& o, owl_run_result& res) {
  const uint32_t B0 = o.block_size ? o.block_size : 1000;
  const uint32_t logStep = o.log_step ? o.log_step : 20000;
  if (B0 % 100 != 0 || 10000 % B0 != 0 || logStep % B0 != 0) { fail(OWL_ERR_ARG, "block size / log step"); }
  HostGpu gpu(device, E, o.W, o.H, o.split);
  SaveDir saver(o.save_dir, E, true, o.n_savefiles);
  Log log{o};
  if (o.res_n) { *o.res_n = 0; }
  std::memset(&res, 0, sizeof(res));

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
      gpu.squareLoop(gpu.data, gpu.data, next - k);
      k = next;
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
      Words rawCheck = gpu.readOut(gpu.check);
      if (!doCheck) {
        if (saver.enabled()) { saver.savePrpUnverified({E, k, B, r, rawCheck, nErrors, 0}); }
        log.line(fmt("   %9u %016" PRIx64, k, r));
        continue;
      }
      const bool ok = gpu.doCheck(B);
      if (ok) {
        nSeqErrors = 0;
        skipNextCheckUpdate = true;
        if (k < kEnd && saver.enabled()) { saver.savePrp({E, k, B, r, rawCheck, nErrors, 0}); }
        log.line(fmt("OK %9u %016" PRIx64, k, r));
        if (k >= kEndEnd) {
          res.finished = 1;
          res.k = k;
          res.n_errors = nErrors;
          return;
        }
      } else {
        ++nErrors;
        log.line(fmt("EE %9u %016" PRIx64 " (check failed, %u errors)", k, r, nErrors));
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
  HostGpu gpu(device, E, o.W, o.H, o.split);
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
    while (true) {
      uint32_t next = roundUp(k + 1, logStep);
      if (next > kEnd) { next = kEnd; }
      if (o.stop_after && next - startK > o.stop_after) { next = std::max(k + 1, startK + o.stop_after); }
      gpu.squareLoop(gpu.data, gpu.data, next - k, OWL_SQ_LL);
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
      log.line(fmt("%9u %016" PRIx64, k, r));
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
