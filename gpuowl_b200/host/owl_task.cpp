// owl_task.cpp -- the reference's work layer above the engine: worktodo parsing
// and the pooled work queue (src/Worktodo.cpp), task execution with its result
// lines (src/Task.cpp), the CERT squaring task (Gpu::isCERT, src/Gpu.cpp:1665-
// 1725) and the MD5 of proof files that the PRP result reports
// (proof::fileHash, src/Proof.cpp:30-37). Files live in a work directory:
// worktodo-<n>.txt, results-<n>.txt, M<E>.cert, and the savefile / proof tree
// of the PRP and LL drivers.
#include <algorithm>
#include <array>
#include <cctype>
#include <cinttypes>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <filesystem>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include <sys/utsname.h>

#include "owl.h"
#include "owl_host.h"
#include "owl_sha3.hpp"

namespace fs = std::filesystem;

namespace owl_detail {
void set_error_string(const std::string& msg);
}

namespace {

struct TaskError {
  int code;
  std::string msg;
};
[[noreturn]] void fail(int code, const std::string& msg) { throw TaskError{code, msg}; }
void ck(int st) {
  if (st != OWL_OK) { fail(st, owl_last_error()); }
}
template <typename F> int guarded(F&& f) {
  try {
    f();
    return OWL_OK;
  } catch (const TaskError& e) {
    owl_detail::set_error_string(e.msg);
    return e.code;
  } catch (const std::exception& e) {
    owl_detail::set_error_string(e.what());
    return OWL_ERR_ARG;
  }
}

// ---- MD5 (RFC 1321): T[i] = floor(2^32 |sin(i + 1)|), the four rounds' shift schedules ----
class Md5 {
 public:
  Md5() {
    static const Consts k;
    K_ = &k;
  }
  void update(const void* data, size_t n) {
    const uint8_t* p = static_cast<const uint8_t*>(data);
    total_ += n;
    while (n) {
      const size_t take = std::min(n, (size_t)64 - fill_);
      std::memcpy(buf_ + fill_, p, take);
      fill_ += take;
      p += take;
      n -= take;
      if (fill_ == 64) {
        block(buf_);
        fill_ = 0;
      }
    }
  }
  std::string hex() {
    const uint64_t bits = total_ * 8;
    const uint8_t one = 0x80, zero = 0;
    update(&one, 1);
    while (fill_ != 56) { update(&zero, 1); }
    uint8_t len[8];
    for (int i = 0; i < 8; ++i) { len[i] = (uint8_t)(bits >> (8 * i)); }
    update(len, 8);
    char out[33];
    for (int i = 0; i < 16; ++i) { std::snprintf(out + 2 * i, 3, "%02x", (unsigned)((h_[i / 4] >> (8 * (i % 4))) & 0xff)); }
    return out;
  }

 private:
  struct Consts {
    uint32_t T[64];
    Consts() {
      for (int i = 0; i < 64; ++i) { T[i] = (uint32_t)std::floor(std::fabs(std::sin((double)(i + 1))) * 4294967296.0); }
    }
  };
  static uint32_t rotl(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }
  void block(const uint8_t* b) {
    static const int S[4][4] = {{7, 12, 17, 22}, {5, 9, 14, 20}, {4, 11, 16, 23}, {6, 10, 15, 21}};
    uint32_t X[16];
    for (int i = 0; i < 16; ++i) {
      X[i] = (uint32_t)b[4 * i] | ((uint32_t)b[4 * i + 1] << 8) | ((uint32_t)b[4 * i + 2] << 16) |
             ((uint32_t)b[4 * i + 3] << 24);
    }
    uint32_t a = h_[0], bb = h_[1], c = h_[2], d = h_[3];
    for (int i = 0; i < 64; ++i) {
      const int round = i / 16;
      uint32_t f;
      int g;
      if (round == 0) {
        f = (bb & c) | (~bb & d);
        g = i;
      } else if (round == 1) {
        f = (d & bb) | (~d & c);
        g = (5 * i + 1) % 16;
      } else if (round == 2) {
        f = bb ^ c ^ d;
        g = (3 * i + 5) % 16;
      } else {
        f = c ^ (bb | ~d);
        g = (7 * i) % 16;
      }
      const uint32_t tmp = d;
      d = c;
      c = bb;
      bb = bb + rotl(a + f + K_->T[i] + X[g], S[round][i % 4]);
      a = tmp;
    }
    h_[0] += a;
    h_[1] += bb;
    h_[2] += c;
    h_[3] += d;
  }
  const Consts* K_ = nullptr;
  uint32_t h_[4] = {0x67452301u, 0xefcdab89u, 0x98badcfeu, 0x10325476u};
  uint8_t buf_[64];
  size_t fill_ = 0;
  uint64_t total_ = 0;
};

std::string file_md5(const fs::path& p) {
  std::ifstream f(p, std::ios::binary);
  if (!f) { fail(OWL_ERR_READ, "cannot open " + p.string()); }
  Md5 h;
  char buf[65536];
  while (f) {
    f.read(buf, sizeof(buf));
    if (f.gcount() > 0) { h.update(buf, (size_t)f.gcount()); }
  }
  return h.hex();
}

// ---- worktodo lines (src/Worktodo.cpp:26-87) ----
std::vector<std::string> split(const std::string& s, char d) {
  std::vector<std::string> out;
  std::string cur;
  for (char c : s) {
    if (c == d) {
      out.push_back(cur);
      cur.clear();
    } else {
      cur += c;
    }
  }
  out.push_back(cur);
  return out;
}
std::string rstrip(std::string s) {
  while (!s.empty() && (s.back() == '\n' || s.back() == '\r')) { s.pop_back(); }
  return s;
}
bool is_hex32(const std::string& s) {
  return s.size() == 32 && std::all_of(s.begin(), s.end(), [](char c) { return std::isxdigit((unsigned char)c); });
}
bool to_u64(const std::string& s, uint64_t* v) {
  if (s.empty()) { return false; }
  uint64_t x = 0;
  for (char c : s) {
    if (c < '0' || c > '9') { return false; }
    x = x * 10 + (uint64_t)(c - '0');
    if (x > (1ull << 40)) { return false; }
  }
  *v = x;
  return true;
}

// Examples: PRP=<AID>,1,2,124647911,-1,77,0   DoubleCheck=<AID>,70198703,75,1   Cert=<AID>,1,2,82997591,-1,162105
bool parse_line(const std::string& raw, owl_task* t) {
  const std::string line = rstrip(raw);
  if (line.empty() || line[0] == '#') { return false; }
  std::memset(t, 0, sizeof(*t));
  std::snprintf(t->line, sizeof(t->line), "%s", line.c_str());
  const std::vector<std::string> top = split(line, '=');
  if (top.size() != 2) { return false; }
  const std::string& kind = top[0];
  std::vector<std::string> parts = split(top[1], ',');
  if (kind == "PRP" || kind == "PRPDC" || kind == "Test" || kind == "DoubleCheck") {
    if (!parts.empty() && (parts.front() == "N/A" || parts.front().empty())) { parts.erase(parts.begin()); }
    if (!parts.empty() && is_hex32(parts.front())) {
      std::snprintf(t->aid, sizeof(t->aid), "%s", parts.front().c_str());
      parts.erase(parts.begin());
    }
    const std::string s = (parts.size() >= 4 && parts[0] == "1" && parts[1] == "2" && parts[3] == "-1")
                              ? parts[2]
                              : (!parts.empty() ? parts[0] : "");
    uint64_t e = 0;
    if (!to_u64(s, &e) || e <= 1000 || e > 0xffffffffull) { return false; }
    t->kind = (kind == "PRP" || kind == "PRPDC") ? OWL_TASK_PRP : OWL_TASK_LL;
    t->exponent = (uint32_t)e;
    return true;
  }
  if (kind == "Cert") {
    if (parts.empty() || !is_hex32(parts.front())) { return false; }
    std::snprintf(t->aid, sizeof(t->aid), "%s", parts.front().c_str());
    parts.erase(parts.begin());
    if (parts.size() == 5 && parts[0] == "1" && parts[1] == "2" && parts[3] == "-1") {
      uint64_t e = 0, sq = 0;
      if (to_u64(parts[2], &e) && to_u64(parts[4], &sq) && e > 1000 && sq > 100 && e <= 0xffffffffull &&
          sq <= 0xffffffffull) {
        t->kind = OWL_TASK_CERT;
        t->exponent = (uint32_t)e;
        t->squarings = (uint32_t)sq;
        return true;
      }
    }
  }
  return false;
}

std::vector<std::string> read_lines(const fs::path& p) {
  std::vector<std::string> out;
  std::ifstream f(p);
  std::string s;
  while (std::getline(f, s)) { out.push_back(s); }
  return out;
}

// the smallest CERT, else the smallest exponent (src/Worktodo.cpp:90-102)
bool best_task(const fs::path& file, owl_task* best) {
  bool found = false;
  for (const std::string& l : read_lines(file)) {
    owl_task t;
    if (!parse_line(l, &t)) { continue; }
    if (!found || (best->kind != OWL_TASK_CERT && t.kind == OWL_TASK_CERT) ||
        ((best->kind != OWL_TASK_CERT || t.kind == OWL_TASK_CERT) && t.exponent < best->exponent)) {
      *best = t;
      found = true;
    }
  }
  return found;
}

uint64_t bytes_of(const fs::path& p) {
  std::error_code ec;
  const auto s = fs::file_size(p, ec);
  return ec ? 0 : (uint64_t)s;
}

void append_line(const fs::path& p, const std::string& line) {
  std::ofstream f(p, std::ios::app);
  f << rstrip(line) << '\n';
  if (!f) { fail(OWL_ERR_ARG, "cannot append to " + p.string()); }
}

// rewrite `p` without the first line equal to `target`, unless its size moved away from initialSize
// (src/fs.cpp:60-69)
bool delete_line(const fs::path& p, const std::string& target, uint64_t initialSize = 0) {
  if (!initialSize) { initialSize = bytes_of(p); }
  const std::vector<std::string> lines = read_lines(p);
  const fs::path tmp = p.string() + "-tmp";
  bool removed = false;
  {
    std::ofstream f(tmp);
    for (const std::string& l : lines) {
      if (!removed && rstrip(l) == rstrip(target)) {
        removed = true;
        continue;
      }
      f << l << '\n';
    }
  }
  if (!removed || bytes_of(p) != initialSize) {
    std::error_code ec;
    fs::remove(tmp, ec);
    return false;
  }
  fs::rename(tmp, p);
  return true;
}

fs::path work_name(const fs::path& dir, int instance) { return dir / ("worktodo-" + std::to_string(instance) + ".txt"); }

// ---- result lines (src/Task.cpp:98-190) ----
std::string jq(const std::string& s) { return "\"" + s + "\""; }
std::string jkv(const std::string& k, const std::string& rawValue) { return jq(k) + ":" + rawValue; }
std::string jobj(const std::vector<std::string>& fields) {
  std::string s;
  for (const std::string& f : fields) {
    if (f.empty()) { continue; }
    s += (s.empty() ? "{" : ", ") + f;
  }
  return s.empty() ? "" : s + "}";
}
std::string hex16(uint64_t x) {
  char b[17];
  std::snprintf(b, sizeof(b), "%016" PRIx64, x);
  return b;
}
std::string utc_now() {
  const std::time_t t = std::time(nullptr);
  char b[64];
  std::strftime(b, sizeof(b), "%Y-%m-%d %H:%M:%S", std::gmtime(&t));
  return b;
}
std::vector<std::string> tail_fields(const owl_task& t) {
  utsname u{};
  uname(&u);
  return {jkv("program", jobj({jkv("name", jq("gpuowl-b200")), jkv("version", jq("1.0")), jkv("port", "8"),
                               jkv("os", jobj({jkv("os", jq(u.sysname)), jkv("version", jq(u.release)),
                                               jkv("architecture", jq(u.machine))}))})),
          t.aid[0] ? jkv("aid", jq(t.aid)) : "", jkv("timestamp", jq(utc_now()))};
}
std::string result_line(const owl_task& t, const char* worktype, const char* status, std::vector<std::string> extras) {
  std::vector<std::string> f{jkv("status", jq(status)), jkv("exponent", std::to_string(t.exponent)),
                             jkv("worktype", jq(worktype))};
  f.insert(f.end(), extras.begin(), extras.end());
  for (auto& x : tail_fields(t)) { f.push_back(x); }
  return jobj(f);
}

uint32_t fft_length(uint32_t E, const owl_run_opts& o) {
  if (o.W && o.H) { return 2 * o.W * o.H; }
  uint32_t N = 0, W = 0, H = 0;
  ck(owl_fft_choose(E, 0, &N, &W, &H));
  return N;
}

// Gpu::isCERT: squarings of the start value in M<E>.cert, then SHA3-256 of the result's bytes
void cert(int device, uint32_t E, uint32_t squarings, const fs::path& certFile, std::array<uint64_t, 4>& hash,
          uint64_t* res64, uint32_t* fftN) {
  const uint32_t nw = (E - 1) / 32 + 1, nb = (E - 1) / 8 + 1;
  std::vector<uint32_t> w(nw, 0);
  {
    std::ifstream f(certFile, std::ios::binary);
    if (!f || !f.read(reinterpret_cast<char*>(w.data()), nb)) { fail(OWL_ERR_READ, "cannot read " + certFile.string()); }
  }
  owl_plan* plan = nullptr;
  ck(owl_plan_create(device, E, 0, 0, &plan));
  struct Destroy {
    owl_plan* p;
    ~Destroy() { owl_plan_destroy(p); }
  } destroy{plan};
  ck(owl_plan_shape(plan, fftN, nullptr, nullptr));
  int32_t* data = nullptr;
  ck(owl_buf_alloc(plan, &data));
  ck(owl_write_words(plan, data, w.data()));
  for (uint32_t k = 0; k < squarings;) {
    const uint32_t its = std::min(1000u, squarings - k);
    ck(owl_square(plan, data, data, its, 0));
    k += its;
  }
  ck(owl_read_words(plan, data, w.data()));
  owl::Sha3_256 h;
  h.update(w.data(), nb);
  hash = h.finish();
  *res64 = ((uint64_t)w[1] << 32) | w[0];
}

}  // namespace

extern "C" {

int owl_worktodo_parse(const char* line, owl_task* task) {
  return guarded([&] {
    if (!line || !task) { fail(OWL_ERR_ARG, "null argument"); }
    if (!parse_line(line, task)) { fail(OWL_ERR_ARG, "worktodo line ignored"); }
  });
}

int owl_worktodo_get(const char* dir, int instance, const char* master_dir, owl_task* task, int* found) {
  return guarded([&] {
    if (!dir || !task || !found) { fail(OWL_ERR_ARG, "null argument"); }
    *found = 0;
    const fs::path local = work_name(dir, instance);
    if (best_task(local, task)) {
      *found = 1;
      return;
    }
    if (!master_dir || !*master_dir) { return; }
    // move one task from the shared worktodo.txt to the local file (src/Worktodo.cpp:111-163)
    const fs::path global = fs::path(master_dir) / "worktodo.txt";
    for (int retry = 0; retry < 2; ++retry) {
      const uint64_t size0 = bytes_of(global);
      if (!size0) { return; }
      owl_task t;
      if (!best_task(global, &t)) { return; }
      append_line(local, t.line);
      if (delete_line(global, t.line, size0)) {
        *task = t;
        *found = 1;
        return;
      }
      if (!delete_line(local, t.line)) { delete_line(local, t.line); }
    }
  });
}

int owl_cert_run(int device, uint32_t E, uint32_t squarings, const char* cert_file, uint8_t sha3[32],
                 uint64_t* res64) {
  return guarded([&] {
    if (!cert_file || !sha3) { fail(OWL_ERR_ARG, "null argument"); }
    std::array<uint64_t, 4> h{};
    uint64_t r = 0;
    uint32_t N = 0;
    cert(device, E, squarings, cert_file, h, &r, &N);
    owl::Sha3_256::digest_bytes(h, sha3);
    if (res64) { *res64 = r; }
  });
}

int owl_file_md5(const char* path, char out[33]) {
  return guarded([&] {
    if (!path || !out) { fail(OWL_ERR_ARG, "null argument"); }
    std::snprintf(out, 33, "%s", file_md5(path).c_str());
  });
}

int owl_task_run(int device, const char* dir, int instance, const owl_task* task, const owl_run_opts* opts,
                 char* result, size_t result_len) {
  return guarded([&] {
    if (!dir || !task) { fail(OWL_ERR_ARG, "null argument"); }
    owl_run_opts o{};
    if (opts) { o = *opts; }
    const std::string root = dir;
    o.save_dir = root.c_str();
    std::string line;
    if (task->kind == OWL_TASK_PRP) {
      owl_run_result r{};
      ck(owl_prp_run(device, task->exponent, &o, &r));
      if (!r.finished) { fail(OWL_ERR_ARG, "PRP stopped before the end"); }
      const uint32_t N = fft_length(task->exponent, o);
      std::vector<std::string> ex{jkv("res64", jq(hex16(r.res64))), jkv("res2048", jq(r.res2048)),
                                  jkv("residue-type", "1"),
                                  jkv("errors", jobj({jkv("gerbicz", std::to_string(r.n_errors))})),
                                  jkv("fft-length", std::to_string(N))};
      if (r.proof_file[0] && r.proof_power) {
        ex.push_back(jkv("proof", jobj({jkv("version", "1"), jkv("power", std::to_string(r.proof_power)),
                                        jkv("hashsize", "64"), jkv("md5", jq(file_md5(r.proof_file)))})));
      }
      line = result_line(*task, "PRP-3", r.is_prime ? "P" : "C", ex);
    } else if (task->kind == OWL_TASK_LL) {
      owl_run_result r{};
      ck(owl_ll_run(device, task->exponent, &o, &r));
      if (!r.finished) { fail(OWL_ERR_ARG, "LL stopped before the end"); }
      const uint32_t N = fft_length(task->exponent, o);
      line = result_line(*task, "LL", r.is_prime ? "P" : "C",
                         {jkv("res64", jq(hex16(r.res64))), jkv("fft-length", std::to_string(N)),
                          jkv("shift-count", "0"), jkv("error-code", jq("00000000"))});
    } else if (task->kind == OWL_TASK_CERT) {
      const fs::path certFile = fs::path(root) / ("M" + std::to_string(task->exponent) + ".cert");
      std::array<uint64_t, 4> h{};
      uint64_t r = 0;
      uint32_t N = 0;
      cert(device, task->exponent, task->squarings, certFile, h, &r, &N);
      std::error_code ec;
      fs::remove(certFile, ec);
      // the digest as one little-endian 256-bit number, printed most significant first (src/Task.cpp:172-174)
      const std::string hexhash = hex16(h[3]) + hex16(h[2]) + hex16(h[1]) + hex16(h[0]);
      std::vector<std::string> f{jkv("worktype", jq("Cert")), jkv("exponent", std::to_string(task->exponent)),
                                 jkv("sha3-hash", jq(hexhash)), jkv("squarings", std::to_string(task->squarings)),
                                 jkv("fft-length", std::to_string(N)), jkv("shift-count", "0"),
                                 jkv("error-code", jq("00000000"))};
      for (auto& x : tail_fields(*task)) { f.push_back(x); }
      line = jobj(f);
    } else {
      fail(OWL_ERR_ARG, "unknown task kind");
    }
    append_line(fs::path(root) / ("results-" + std::to_string(instance) + ".txt"), line);
    if (task->line[0]) { delete_line(work_name(root, instance), task->line); }
    if (result && result_len) { std::snprintf(result, result_len, "%s", line.c_str()); }
  });
}

}  // extern "C"
