// Test infrastructure: runs the packed 16-bit filter core (storm_b200/csrc/filter_core.cuh),
// compiled for the host, against the oracle's filter on random cases.  Prints the number of
// cases checked and exits non-zero on the first mismatch.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

#include "../storm_b200/csrc/filter_core.cuh"

extern "C" int or_sw_filter(int W, int L, uint32_t match, uint32_t mismatch, uint32_t gapopen,
                            uint32_t gapext, uint32_t threshold, const uint8_t* genome, int64_t pos,
                            const uint8_t* read);

static void pack(const std::vector<int>& c, uint8_t* out) {
  for (size_t i = 0; i < c.size(); ++i) out[i >> 2] |= (uint8_t)(c[i] << ((i & 3) * 2));
}

template <int W>
static int filter_ws(const uint8_t* gexp, int64_t pos, const uint8_t* rexp, int L, int fm, int fx, int fo, int fe) {
  uint32_t TLO, THI, NFE, CFO;
  sg::filter_split_consts(fm, fx, fo, fe, TLO, THI, NFE, CFO);
  return sg::filter_split<W>(gexp, pos, rexp, L, TLO, THI, NFE, CFO);
}

template <int W>
static int filter_w(const uint8_t* g, int64_t pos, const uint8_t* r, int64_t rstride, int L, int fm, int fx,
                    int fo, int fe) {
  const uint32_t T = (uint32_t)(fm & 0xff) | ((uint32_t)((256 - fx) & 0xff) << 8) |
                     ((uint32_t)((256 - fx) & 0xff) << 16) | ((uint32_t)((256 - fx) & 0xff) << 24);
  const uint32_t NFE = (uint32_t)(uint16_t)(-fe) * 0x10001u, NFO = (uint32_t)(uint16_t)(-fo) * 0x10001u;
  return sg::filter_dpx<W>(g, pos, r, rstride, L, T, NFE, NFO);
}

int main(int argc, char** argv) {
  const int cases = argc > 1 ? atoi(argv[1]) : 20000;
  std::mt19937_64 rng(12345);
  const int G = 6000, PAD = 4096;
  std::vector<uint8_t> gbuf(PAD + G / 4 + PAD + 64, 0);
  uint8_t* gen = gbuf.data() + PAD;
  std::vector<int> g(G);
  for (int i = 0; i < G; ++i) g[i] = rng() & 3;
  pack(g, gen);
  std::vector<uint8_t> gxbuf(PAD * 4 + G + PAD * 4, 0);
  uint8_t* gexp = gxbuf.data() + PAD * 4;
  for (int i = 0; i < G; ++i) gexp[i] = (uint8_t)(g[i] * 0x11);
  int checked3 = 0;
  int checked = 0;
  for (int t = 0; t < cases; ++t) {
    const int Ws[4] = {2, 4, 8, 16};
    const int W = Ws[rng() % 4];
    const int Ls[18] = {1, 2, 3, 4, 7, 8, 12, 15, 16, 17, 23, 24, 35, 49, 50, 100, 150, 1000};
    const int L = Ls[rng() % 18];
    const int fm = (int)(rng() % 2 ? 5 : 1 + rng() % 20), fx = 1 + (int)(rng() % 8);
    const int fo = (int)(rng() % 12), fe = (int)(rng() % 6);
    const int thr = (int)(rng() % 260);
    const int src = (int)(rng() % (G - L - 40));
    std::vector<int> read(L);
    const double rate = (rng() % 4) * 0.1;
    for (int i = 0; i < L; ++i) read[i] = (rng() % 1000 < rate * 1000) ? (int)(rng() & 3) : g[src + i];
    const int64_t stride = ((L + 3) / 4 + 7 + 8) & ~7;
    std::vector<uint8_t> rb(stride + 16, 0);
    pack(read, rb.data());
    int64_t pos = (rng() % 3 == 0) ? (int64_t)(rng() % (G + 2 * L)) - L : src - (int64_t)(rng() % (2 * W));
    int got;
    switch (W) {
    case 2: got = filter_w<2>(gen, pos, rb.data(), stride, L, fm, fx, fo, fe); break;
    case 4: got = filter_w<4>(gen, pos, rb.data(), stride, L, fm, fx, fo, fe); break;
    case 8: got = filter_w<8>(gen, pos, rb.data(), stride, L, fm, fx, fo, fe); break;
    default: got = filter_w<16>(gen, pos, rb.data(), stride, L, fm, fx, fo, fe); break;
    }
    const int pass = got > (thr >= 255 ? 254 : thr);
    if (L >= W) {
      std::vector<uint8_t> rexp(((L + W + 8 + 3) & ~3) + 16, 0xC4);
      for (int i = 0; i < L; ++i) rexp[i] = (uint8_t)(0xC4 + read[i] * 0x11);
      int got4;
      switch (W) {
      case 2: got4 = filter_ws<2>(gexp, pos, rexp.data(), L, fm, fx, fo, fe); break;
      case 4: got4 = filter_ws<4>(gexp, pos, rexp.data(), L, fm, fx, fo, fe); break;
      case 8: got4 = filter_ws<8>(gexp, pos, rexp.data(), L, fm, fx, fo, fe); break;
      default: got4 = filter_ws<16>(gexp, pos, rexp.data(), L, fm, fx, fo, fe); break;
      }
      if (got4 != got) {
        printf("MISMATCH split case %d: W=%d L=%d fm=%d fx=%d fo=%d fe=%d pos=%lld max=%d stream-max=%d\n", t, W, L,
               fm, fx, fo, fe, (long long)pos, got4, got);
        return 1;
      }
      const int pass3 = got4 > (thr >= 255 ? 254 : thr);
      const int exp3 = or_sw_filter(W, L, fm, fx, fo, fe, thr, gen, pos, rb.data());
      if (pass3 != exp3) {
        printf("MISMATCH split case %d: W=%d L=%d fm=%d fx=%d fo=%d fe=%d thr=%d pos=%lld max=%d exp=%d\n", t, W, L,
               fm, fx, fo, fe, thr, (long long)pos, got4, exp3);
        return 1;
      }
      checked3++;
    }
    const int exp = or_sw_filter(W, L, fm, fx, fo, fe, thr, gen, pos, rb.data());
    if (pass != exp) {
      printf("MISMATCH case %d: W=%d L=%d fm=%d fx=%d fo=%d fe=%d thr=%d pos=%lld max=%d exp=%d\n", t, W, L, fm,
             fx, fo, fe, thr, (long long)pos, got, exp);
      return 1;
    }
    checked++;
  }
  printf("checked %d (split layout %d)\n", checked, checked3);
  return 0;
}
