// Host check of the MILU sweeps' bulk copies (sweep_lane, kernels.h): for
// every tile, mode, step and copy of a set of grids and tile shapes, the
// source run lies inside its array, source, destination and size are
// multiples of 16 bytes, copies of one step do not overlap in the ring
// slot, and every ring entry that a column of k_sweep reads at a step was
// copied for that step (the reads of sweep_body's prepare, all cells taken
// as computed).  Prints the number of failures; exit status 1 if any.
#include "kernels.h"
#include <algorithm>
#include <cstdio>
#include <vector>
using namespace cadmas;

static long long fails = 0, checks = 0;
#define CHECK(c, ...)                                      \
  do {                                                     \
    ++checks;                                              \
    if (!(c)) {                                            \
      if (fails++ < 10) { printf(__VA_ARGS__); printf("\n"); } \
    }                                                      \
  } while (0)

static void run(int NI, int NJ, int NK, int TI, int TJ, int es, int mode) {
  SkewGeo q{};
  q.TI = TI; q.TJ = TJ; q.TIp = (TI + 3) & ~3; q.T = q.TIp * TJ; q.W = (NK - 2) + (TI - 1) + (TJ - 1);
  q.ntx = (NI - 2 + TI - 1) / TI;
  const int nty = (NJ - 2 + TJ - 1) / TJ;
  q.nb = q.ntx * nty; q.split = 1;
  const int T = q.T, TIp = q.TIp, SS = sweep_slot(q, mode, es);
  const long long nsys = (long long)q.nb * q.W * SYS_N * T, nvec = (long long)q.nb * q.W * T;
  const bool BWD = mode >= SWEEP_BWD;
  const int SF = sweep_sys_first(mode) - sweep_sys_dst(mode);
  auto o = [&](int a) { return (a - SF) * T; };
  for (int b = 0; b < q.nb; ++b) {
    const int bx = b % q.ntx, by = b / q.ntx;
    const int wi = std::min(TI, NI - (2 + bx * TI)), wj = std::min(TJ, NJ - (2 + by * TJ));
    const int nsteps = (NK - 2) + (wi - 1) + (wj - 1);
    std::vector<std::vector<char>> cp(nsteps, std::vector<char>(SS, 0));
    for (int u = 0; u < nsteps; ++u) {
      const int w = BWD ? nsteps - 1 - u : u;
      for (int c = 0; c < 32; ++c) {
        SweepLane l;
        if (c >= sweep_ncopy(q, mode) || !sweep_lane(q, mode, b, c, l, es)) continue;
        if (w < l.dlo || w > l.dhi) continue;
        const long long src = l.base + (long long)w * l.wstride, n = l.arr == 0 ? nsys : nvec;
        const int ne = l.bytes / es;
        CHECK(src >= 0 && src + ne <= n, "source outside its array: mode %d tile %d step %d copy %d", mode, b, u, c);
        CHECK(src * es % 16 == 0 && l.bytes % 16 == 0 && l.bytes > 0, "unaligned source: mode %d copy %d", mode, c);
        CHECK(l.dst * es % 16 == 0 && l.dst >= 0 && l.dst + ne <= SS, "destination: mode %d copy %d", mode, c);
        for (int e = std::max(l.dst, 0); e < std::min(l.dst + ne, SS); ++e) {
          CHECK(!cp[u][e], "copies overlap: mode %d step %d copy %d entry %d", mode, u, c, e);
          cp[u][e] = 1;
        }
      }
    }
    auto rd = [&](int s, int e, const char *what, int ti, int tj) {
      CHECK(s >= 0 && s < nsteps && e >= 0 && e < SS && cp[s][e],
            "%s not copied: grid %dx%dx%d tile %dx%d es %d mode %d tile %d step %d column (%d,%d)", what, NI, NJ,
            NK, TI, TJ, es, mode, b, s, ti, tj);
    };
    const int hl0 = halo_left(q, es) + halo_lofs(q, es), hr0 = halo_right(q, es), hd0 = halo_down(q, es),
              hu0 = halo_up(q, es);
    for (int tj = 0; tj < wj; ++tj)
      for (int ti = 0; ti < wi; ++ti) {
        const int tid = ti + TIp * tj, ri = wi - 1 - ti, rj = wj - 1 - tj;
        const int slo = BWD ? ri + rj : ti + tj, shi = slo + NK - 3;
        const bool ex0 = ti == 0, ex1 = ti == wi - 1, ey0 = tj == 0, ey1 = tj == wj - 1;
        for (int s = slo; s <= shi; ++s) {
          if (mode == SWEEP_FWD_AX) {
            const int k = 2 + s - ti - tj;
            rd(s, o(SYS_DD) + tid, "DD", ti, tj);
            rd(s, 8 * T + tid, "P", ti, tj);
            if (ex0) { if (bx > 0) rd(s, hl0 + TIp * tj, "left halo", ti, tj); }
            else rd(s - 1, 8 * T + tid - 1, "P(i-1)", ti, tj);
            if (ey0) { if (by > 0) rd(s, hd0 + ti, "lower halo", ti, tj); }
            else rd(s - 1, 8 * T + tid - TIp, "P(j-1)", ti, tj);
            if (ex1) { if (bx < q.ntx - 1) rd(s, hr0 + TIp * tj, "right halo", ti, tj); }
            else rd(s + 1, 8 * T + tid + 1, "P(i+1)", ti, tj);
            if (ey1) { if (by < nty - 1) rd(s, hu0 + ti, "upper halo", ti, tj); }
            else rd(s + 1, 8 * T + tid + TIp, "P(j+1)", ti, tj);
            if (k < NK - 1) rd(s + 1, 8 * T + tid, "P(k+1)", ti, tj);
            for (int a : {SYS_AD, SYS_ALI, SYS_ALJ, SYS_ALK, SYS_AUI, SYS_AUJ, SYS_AUK}) rd(s, o(a) + tid, "A", ti, tj);
            if (ti > 0) rd(s - 1, o(SYS_DD) + tid - 1, "DD(i-1)", ti, tj);
            if (tj > 0) rd(s - 1, o(SYS_DD) + tid - TIp, "DD(j-1)", ti, tj);
          } else if (mode == SWEEP_FWD) {
            rd(s, o(SYS_DD) + tid, "DD", ti, tj);
            rd(s, tid, "Y", ti, tj);
            for (int a : {SYS_ALI, SYS_ALJ, SYS_ALK}) rd(s, o(a) + tid, "A", ti, tj);
            if (ti > 0) rd(s - 1, o(SYS_DD) + tid - 1, "DD(i-1)", ti, tj);
            if (tj > 0) rd(s - 1, o(SYS_DD) + tid - TIp, "DD(j-1)", ti, tj);
          } else {
            rd(s, o(SYS_DD) + tid, "DD", ti, tj);
            rd(s, tid, "T", ti, tj);
            for (int a : {SYS_AUI, SYS_AUJ, SYS_AUK}) rd(s, o(a) + tid, "U", ti, tj);
            if (sweep_ndot(mode) > 0) rd(s, 5 * T + tid, "R0", ti, tj);
            if (sweep_ndot(mode) == 5) rd(s, 6 * T + tid, "RR", ti, tj);
          }
        }
      }
  }
}

int main() {
  // NI, NJ, NK (with the ghost layers), TI, TJ: full and ragged tiles, the
  // bench's 16x16 and 8x16 shapes, thin and odd shapes, few layers
  const int geos[][5] = {{12, 10, 8, 4, 4},   {36, 20, 12, 16, 16}, {40, 37, 9, 16, 8},  {19, 23, 30, 7, 5},
                         {70, 34, 20, 16, 16}, {50, 40, 5, 8, 16},   {34, 34, 130, 16, 16}, {10, 10, 4, 13, 3},
                         {27, 9, 6, 32, 4},    {66, 66, 7, 8, 8},    {5, 5, 5, 1, 1},      {22, 40, 11, 3, 19}};
  int cases = 0;
  for (const auto &g : geos)
    for (int es : {4, 8})
      for (int m = SWEEP_FWD; m <= SWEEP_BWD5; ++m) {
        run(g[0], g[1], g[2], g[3], g[4], es, m);
        ++cases;
      }
  printf("%d cases, %lld checks, %lld failures\n", cases, checks, fails);
  return fails != 0;
}
