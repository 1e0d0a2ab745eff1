// emu_main.cpp -- runs libowl's kernels on the CPU (owl_emu_rt.hpp) with the
// same launch sequence as owl_square / owl_modmul, and prints the result as
// compact words so that tests/test_emulator.py can compare it with GMP.
//
// TEST INFRASTRUCTURE ONLY. Usage:
//   owl_emu square E W H n flags seed   (seed 0: start from 3, or 4 with LL)
//   owl_emu modmul E W H mul3 seedA seedB
//   owl_emu pack E N pattern            (device expand / compact vs owl_words.hpp; prints "pack ok")
//   owl_emu chain nblocks seed          (the block-carry chain vs its serial definition; "chain ok")
// With OWL_EMU_SPLIT=<flags> in the environment the column pass (flag 1, H = 2048 or 2560) and the
// line pass (flag 2, W = 2048) run their split-precision kernels (k_pass2_tc, k_pass1<..., SPLIT>) on the emulated
// tensor cores. With OWL_EMU_NO_ROE=1 the fused line passes run the build without the round-off
// measurement. OWL_EMU_COL=<v> runs the
// column pass's variant v (owl::COL_V16 / COL_V8 / COL_V16_OCC2) with its stage tables. With
// OWL_EMU_GROUP=1 the line passes run the grouped kernel of a batch (one plan as the group).
// Output: one line "roe <max>" then one line of nWords hex u32 (little-endian order).
#define OWL_EMU 1
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "owl_kernels.cuh"
#include "owl_pass2_tc.cuh"
#include "owl_pack.cuh"
#include "owl_tables.hpp"
#include "owl_words.hpp"

using namespace owl;

namespace {

constexpr int kR = 2;

struct EmuPlan {
  Tables t;
  Args a{};
  std::vector<C> twW, twH, rootH, twLo, twHi, F1, F2;
  std::vector<long long> shuttle, pending;
  std::vector<uint32_t> flags;
  Ctl ctl{};
  std::vector<float> roe;
  int roePos = 0;
  bool split = false;
  bool splitLine = false;
  std::vector<uint8_t> tc1B;
  int colVariant = COL_V16;
  std::vector<C> twHtc;
  std::vector<uint8_t> tcB;
};

std::vector<C> toC(const std::vector<HostC>& v) {
  std::vector<C> r(v.size());
  for (size_t i = 0; i < v.size(); ++i) { r[i] = make_double2(v[i].x, v[i].y); }
  return r;
}

void init(EmuPlan& p, uint32_t E, uint32_t W, uint32_t H) {
  p.t = make_tables(E, W, H);
  p.twW = toC(p.t.twW);
  p.twH = toC(p.t.twH);
  p.rootH = toC(p.t.rootH);
  p.twLo = toC(p.t.twLo);
  p.twHi = toC(p.t.twHi);
  p.F1.assign(p.t.hN, make_double2(0, 0));
  p.F2.assign(p.t.hN, make_double2(0, 0));
  p.shuttle.assign((size_t)(H / kR) * W, 0);
  p.pending.assign(2 * kPendingCap, 0);
  p.flags.assign(H / kR, 0);
  p.roe.assign(4096, 0.0f);
  Args& a = p.a;
  a.twW = p.twW.data();
  a.twH = p.twH.data();
  a.rootH = p.rootH.data();
  a.twLo = p.twLo.data();
  a.twHi = p.twHi.data();
  a.wt1 = p.t.wt1.data();
  a.iwt1 = p.t.iwt1.data();
  a.x1 = p.t.x1.data();
  a.wt2 = p.t.wt2.data();
  a.iwt2 = p.t.iwt2.data();
  a.x2 = p.t.x2.data();
  a.p1masks = reinterpret_cast<const uint2*>(p.t.p1masks.data());
  a.shuttle = p.shuttle.data();
  a.pending = p.pending.data();
  a.flags = p.flags.data();
  a.ctl = &p.ctl;
  a.roe = p.roe.data();
  a.E = E;
  a.N = p.t.N;
  a.W = W;
  a.H = H;
  a.hN = p.t.hN;
  a.bitsLo = E / p.t.N;
  a.eModN = E % p.t.N;
  a.scaleLo = std::ldexp(1.0, (int)(E / p.t.N));
  a.iscaleLo = std::ldexp(1.0, -(int)(E / p.t.N));
  a.loShift = p.t.loShift;
  a.timeoutNs = 60ull * 1000000000ull;
  if (const char* cv = std::getenv("OWL_EMU_COL")) {
    p.colVariant = std::atoi(cv);
    if (!col_variant_ok((int)H, p.colVariant)) { throw std::runtime_error("column variant not built for H"); }
    p.twH = toC(col_stage_tables(H, p.colVariant));
    a.twH = p.twH.data();
  }
  const char* sp = std::getenv("OWL_EMU_SPLIT");
  const int spf = sp ? std::atoi(sp) : 0;  // split flags: 1 columns, 2 lines
  if ((spf & 1) && tc_height((int)H)) {
    p.split = true;
    p.twHtc = toC(stage_tables(H, 8, H == 2048 ? TcCfg<2048>::R1 : TcCfg<2560>::R1));
    p.tcB = H == 2048 ? tc_dft_digits<2048>() : tc_dft_digits<2560>();
  }
  if ((spf & 2) && W == (uint32_t)kLtcW) {
    p.splitLine = true;
    p.tc1B = line_tc_dft_digits();
    a.tc1B = p.tc1B.data();
  }
}

template <int W, int M> void p1m(EmuPlan& p, C* F, int32_t* words, int slot, int flags) {
  constexpr int T = kR * W / 16;
  size_t sm = (size_t)kR * p1_line_stride<W, kR>() * sizeof(C);
  Args a = p.a;
  if constexpr (W == kLtcW) {
    if (p.splitLine) {
      const size_t smx = sm + ltc_extra_smem();
      if (M == P1_FUSED && std::getenv("OWL_EMU_NO_ROE")) {
        emu_launch(p.t.H / kR, T, smx, [=] { k_pass1<W, kR, M, false, true>(a, F, words, -1, flags, -1); });
      } else {
        emu_launch(p.t.H / kR, T, smx, [=] { k_pass1<W, kR, M, true, true>(a, F, words, slot, flags, -1); });
      }
      return;
    }
  }
  if (std::getenv("OWL_EMU_GROUP")) {
    // the grouped kernel of a batch, as a group of this one plan
    GroupArgs ga{};
    ga.a[0] = a;
    ga.F[0] = F;
    ga.words[0] = words;
    if (M == P1_FUSED && std::getenv("OWL_EMU_NO_ROE")) {
      emu_launch(p.t.H / kR, T, sm, [=] { k_pass1_group<W, kR, M, false>(ga, -1, flags); });
    } else {
      emu_launch(p.t.H / kR, T, sm, [=] { k_pass1_group<W, kR, M>(ga, slot, flags); });
    }
    return;
  }
  if (M == P1_FUSED && std::getenv("OWL_EMU_NO_ROE")) {
    // the build without the round-off measurement (OWL_SQ_NO_ROE)
    emu_launch(p.t.H / kR, T, sm, [=] { k_pass1<W, kR, M, false>(a, F, words, -1, flags, -1); });
    return;
  }
  emu_launch(p.t.H / kR, T, sm, [=] { k_pass1<W, kR, M>(a, F, words, slot, flags, -1); });
}
template <int H, int M, int CV> void p2mv(EmuPlan& p, C* F, const C* Fb, C* Fq) {
  constexpr int V = col_vpt(CV), MB = col_minb(CV);
  constexpr int T = 2 * H / V;
  size_t sm = 2 * (size_t)p2_col_stride<H, V>() * sizeof(C);
  Args a = p.a;
  emu_launch(p.t.W / 2, T, sm, [=] { k_pass2<H, kR, M, V, MB>(a, F, Fb, Fq, -1); });
}
template <int H, int M> void p2m(EmuPlan& p, C* F, const C* Fb, C* Fq) {
  if constexpr (col_variant_ok(H, COL_V8)) {
    if (p.colVariant == COL_V8) { return p2mv<H, M, COL_V8>(p, F, Fb, Fq); }
  }
  if constexpr (col_variant_ok(H, COL_V16_OCC2)) {
    if (p.colVariant == COL_V16_OCC2) { return p2mv<H, M, COL_V16_OCC2>(p, F, Fb, Fq); }
  }
  p2mv<H, M, COL_V16>(p, F, Fb, Fq);
}

template <int H, int M> void p2m_tch(EmuPlan& p, C* F, const C* Fb, C* Fq) {
  Args a = p.a;
  const unsigned char* tcB = p.tcB.data();
  const C* twT = p.twHtc.data();
  emu_launch(p.t.W / 2, H / 8, TcCfg<H>::SMEM, [=] { k_pass2_tc<H, kR, M>(a, tcB, twT, F, Fb, Fq, -1); });
}
template <int M> void p2m_tc(EmuPlan& p, C* F, const C* Fb, C* Fq) {
  if (p.t.H == 2560) {
    p2m_tch<2560, M>(p, F, Fb, Fq);
  } else {
    p2m_tch<2048, M>(p, F, Fb, Fq);
  }
}

template <int W> void p1w(EmuPlan& p, int mode, C* F, int32_t* words, int flags) {
  int slot = -1;
  if (mode != P1_IN) { slot = p.roePos++; }
  if (mode == P1_FUSED) p1m<W, P1_FUSED>(p, F, words, slot, flags);
  else if (mode == P1_IN) p1m<W, P1_IN>(p, F, words, slot, flags);
  else p1m<W, P1_OUT>(p, F, words, slot, flags);
}
template <int H> void p2h(EmuPlan& p, int mode, C* F, const C* Fb, C* Fq) {
  if (mode == P2_SQUARE) p2m<H, P2_SQUARE>(p, F, Fb, Fq);
  else if (mode == P2_FWD) p2m<H, P2_FWD>(p, F, Fb, Fq);
  else p2m<H, P2_MUL>(p, F, Fb, Fq);
}

void pass1(EmuPlan& p, int mode, C* F, int32_t* words, int flags) {
  switch (p.t.W) {
    case 64: p1w<64>(p, mode, F, words, flags); break;
    case 128: p1w<128>(p, mode, F, words, flags); break;
    case 256: p1w<256>(p, mode, F, words, flags); break;
    case 512: p1w<512>(p, mode, F, words, flags); break;
    case 1024: p1w<1024>(p, mode, F, words, flags); break;
    case 2048: p1w<2048>(p, mode, F, words, flags); break;
    default: throw std::runtime_error("emu W");
  }
  if (mode == P1_OUT) {
    Args a = p.a;
    emu_launch(1, 32, 0, [=] { k_carry_fixup(a, words); });
  }
  if (p.ctl.error) { throw std::runtime_error("device wait timeout in emulation"); }
}
void pass2(EmuPlan& p, int mode, C* F, const C* Fb, C* Fq) {
  if (p.split) {
    if (mode == P2_SQUARE) p2m_tc<P2_SQUARE>(p, F, Fb, Fq);
    else if (mode == P2_FWD) p2m_tc<P2_FWD>(p, F, Fb, Fq);
    else p2m_tc<P2_MUL>(p, F, Fb, Fq);
    if (p.ctl.error) { throw std::runtime_error("tensor-core wait timeout in emulation"); }
    return;
  }
  switch (p.t.H) {
    case 64: p2h<64>(p, mode, F, Fb, Fq); break;
    case 128: p2h<128>(p, mode, F, Fb, Fq); break;
    case 256: p2h<256>(p, mode, F, Fb, Fq); break;
    case 512: p2h<512>(p, mode, F, Fb, Fq); break;
    case 640: p2h<640>(p, mode, F, Fb, Fq); break;
    case 1280: p2h<1280>(p, mode, F, Fb, Fq); break;
    case 2560: p2h<2560>(p, mode, F, Fb, Fq); break;
    case 2048: p2h<2048>(p, mode, F, Fb, Fq); break;
    default: throw std::runtime_error("emu H");
  }
}

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9e3779b97f4a7c15ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

std::vector<uint32_t> start_words(uint32_t E, uint64_t seed, uint32_t small) {
  std::vector<uint32_t> w(n_words(E), 0);
  if (seed == 0) {
    w[0] = small;
    return w;
  }
  uint64_t s = seed;
  for (auto& x : w) { x = (uint32_t)splitmix(s); }
  uint32_t top = E % 32;
  if (top) { w.back() &= (1u << top) - 1; }
  return w;
}

void print_words(const std::vector<int32_t>& d, uint32_t N, uint32_t E, float roe) {
  // every digit of a block-exit buffer must be balanced: -2^(b-1) <= d < 2^(b-1)
  for (uint32_t k = 0; k < N; ++k) {
    int32_t half = 1 << (word_bits(N, E, k) - 1);
    if (d[k] < -half || d[k] >= half) {
      std::printf("error unbalanced digit %u\n", k);
      std::exit(5);
    }
  }
  std::vector<uint32_t> out(n_words(E));
  if (!compact_bits(d.data(), N, E, out.data())) {
    std::printf("error compact\n");
    std::exit(3);
  }
  std::printf("roe %.6f\n", roe);
  for (size_t i = 0; i < out.size(); ++i) { std::printf("%08x%c", out[i], i + 1 == out.size() ? '\n' : ' '); }
}

float max_roe(const EmuPlan& p) {
  float m = 0;
  for (int i = 0; i < p.roePos; ++i) { m = std::max(m, p.roe[i]); }
  return m;
}

}  // namespace

// pattern 0: 3, 1: 2^E - 1, 2: every raw digit 2^(len-1) - 1 (a carry that propagates through all
// digits), 3: zero, 4: 2^E - 2, other: random words from that seed
std::vector<uint32_t> pack_words(uint32_t E, uint32_t N, uint64_t pattern) {
  const uint32_t nw = n_words(E);
  std::vector<uint32_t> w(nw, 0);
  auto mask_top = [&] {
    if (E % 32) { w.back() &= (1u << (E % 32)) - 1; }
  };
  if (pattern == 0) {
    w[0] = 3;
  } else if (pattern == 1 || pattern == 4) {
    for (auto& x : w) { x = 0xffffffffu; }
    mask_top();
    if (pattern == 4) { w[0] -= 1; }
  } else if (pattern == 2) {
    uint64_t bit = 0;
    for (uint32_t k = 0; k < N; ++k) {
      const uint32_t len = word_bits(N, E, k);
      const uint64_t v = (1ull << (len - 1)) - 1;
      for (uint32_t b = 0; b < len; ++b, ++bit) {
        if ((v >> b) & 1) { w[bit / 32] |= 1u << (bit % 32); }
      }
    }
  } else if (pattern != 3) {
    w = start_words(E, pattern, 3);
  }
  return w;
}

int pack_test(uint32_t E, uint32_t N, uint64_t pattern) {
  const uint32_t nw = n_words(E), nb = (N + kPackDigits - 1) / kPackDigits;
  std::vector<uint32_t> words = pack_words(E, N, pattern), blk(nb), dwords(nw + 2, 0), want(nw);
  std::vector<int32_t> host(N), dev(N);
  PackCtl ctl{};
  if (!expand_bits(words.data(), N, E, host.data())) { return 3; }
  const uint32_t* pw = words.data();
  uint32_t* pb = blk.data();
  int32_t* pd = dev.data();
  PackCtl* pc = &ctl;
  emu_launch(nb, kPackThreads, 0, [=] { k_pack_summary<true>(pw, nullptr, nw, E, N, pb); });
  emu_launch(1, kPackThreads, 0, [=] { k_pack_chain(pb, nb, pc); });
  emu_launch(nb, kPackThreads, 0, [=] { k_expand_digits(pw, nw, E, N, pb, pc, pd); });
  if (dev != host) {
    std::printf("error expand differs\n");
    return 5;
  }
  // compact the digits back and compare with the host compact
  if (!compact_bits(host.data(), N, E, want.data())) { return 3; }
  const int32_t* ph = host.data();
  uint32_t* po = dwords.data();
  emu_launch(nb, kPackThreads, 0, [=] { k_pack_summary<false>(nullptr, ph, nw, E, N, pb); });
  emu_launch(1, kPackThreads, 0, [=] { k_pack_chain(pb, nb, pc); });
  emu_launch(nb, kPackThreads, 0, [=] { k_compact_words(ph, nw, E, N, pb, pc, po); });
  emu_launch(1, 32, 0, [=] { k_compact_finish(pc, nw, po); });
  if (ctl.error || !std::equal(want.begin(), want.end(), dwords.begin())) {
    std::printf("error compact differs\n");
    return 6;
  }
  std::printf("pack ok\n");
  return 0;
}

// the block-carry chain alone on nb random statuses (runs of propagating blocks included), against
// the serial definition: carry into block b = the last non-propagating status below b, else 0
int chain_test(uint32_t nb, uint64_t seed) {
  std::vector<uint32_t> st(nb), blk(nb), want(nb);
  uint64_t sd = seed;
  for (uint32_t b = 0; b < nb; ++b) {
    const uint64_t r = splitmix(sd) % 8;
    st[b] = r < 5 ? (uint32_t)ST_PROP : (r < 7 ? (uint32_t)ST_KILL : (uint32_t)ST_GEN);
  }
  uint32_t c = 0;
  for (uint32_t b = 0; b < nb; ++b) {
    want[b] = c;
    c = (st[b] == ST_PROP) ? c : st[b];
  }
  blk = st;
  PackCtl ctl{};
  ctl.carryOut = 7;
  uint32_t* pb = blk.data();
  PackCtl* pc = &ctl;
  emu_launch(1, kPackThreads, 0, [=] { k_pack_chain(pb, nb, pc); });
  if (blk != want || ctl.carryOut != c) {
    std::printf("error chain differs\n");
    return 7;
  }
  std::printf("chain ok\n");
  return 0;
}

int main(int argc, char** argv) {
  if (argc < 2) { return 2; }
  std::string mode = argv[1];
  try {
    if (mode == "chain" && argc == 4) {
      return chain_test(std::strtoul(argv[2], nullptr, 10), std::strtoull(argv[3], nullptr, 10));
    }
    if (mode == "pack" && argc == 5) {
      return pack_test(std::strtoul(argv[2], nullptr, 10), std::strtoul(argv[3], nullptr, 10),
                       std::strtoull(argv[4], nullptr, 10));
    }
    if (mode == "square" && argc == 8) {
      uint32_t E = std::strtoul(argv[2], nullptr, 10), W = std::strtoul(argv[3], nullptr, 10),
               H = std::strtoul(argv[4], nullptr, 10), n = std::strtoul(argv[5], nullptr, 10),
               flags = std::strtoul(argv[6], nullptr, 10);
      uint64_t seed = std::strtoull(argv[7], nullptr, 10);
      EmuPlan p;
      init(p, E, W, H);
      const uint32_t N = p.t.N;
      auto w = start_words(E, seed, (flags & FL_LL) ? 4 : 3);
      std::vector<int32_t> in(N), out(N);
      if (!expand_bits(w.data(), N, E, in.data())) { return 3; }
      pass1(p, P1_IN, p.F1.data(), in.data(), 0);
      for (uint32_t k = 0; k < n; ++k) {
        pass2(p, P2_SQUARE, p.F1.data(), nullptr, nullptr);
        if (k + 1 < n) pass1(p, P1_FUSED, p.F1.data(), nullptr, flags & FL_LL);
        else pass1(p, P1_OUT, p.F1.data(), out.data(), flags);
      }
      print_words(out, N, E, max_roe(p));
      return 0;
    }
    if (mode == "modmul" && argc == 8) {
      uint32_t E = std::strtoul(argv[2], nullptr, 10), W = std::strtoul(argv[3], nullptr, 10),
               H = std::strtoul(argv[4], nullptr, 10), mul3 = std::strtoul(argv[5], nullptr, 10);
      uint64_t sa = std::strtoull(argv[6], nullptr, 10), sb = std::strtoull(argv[7], nullptr, 10);
      EmuPlan p;
      init(p, E, W, H);
      const uint32_t N = p.t.N;
      auto wa = start_words(E, sa, 3), wb = start_words(E, sb, 3);
      std::vector<int32_t> a(N), b(N);
      if (!expand_bits(wa.data(), N, E, a.data()) || !expand_bits(wb.data(), N, E, b.data())) { return 3; }
      pass1(p, P1_IN, p.F2.data(), b.data(), 0);
      pass2(p, P2_FWD, p.F2.data(), nullptr, p.F2.data());
      pass1(p, P1_IN, p.F1.data(), a.data(), 0);
      pass2(p, P2_MUL, p.F1.data(), p.F2.data(), nullptr);
      pass1(p, P1_OUT, p.F1.data(), a.data(), mul3 ? FL_MUL3 : 0);
      print_words(a, N, E, max_roe(p));
      return 0;
    }
  } catch (const std::exception& e) {
    std::printf("error %s\n", e.what());
    return 4;
  }
  return 2;
}
