// k_drop.cu -- the TimerDoor droplet model VF_FDROPF (vf_fdropf.f:63-671).
//
//   k_drop_start     vf_fdropf.f:69-290, one thread per cell: new droplet
//                    cells get their velocity, old ones resting on an
//                    obstacle slide, other cells lose their droplet values
//   k_drop_line<AX>  vf_fdropf.f:292-610 for one axis and direction: one
//                    line of cells along the axis per thread (y, z) or per
//                    warp with the line's F and NF staged in shared memory
//                    (x, whose lines are contiguous in memory)
//
// A droplet cell is a gas cell (NF = 8) holding water (F > FLOWER).  In a
// directional pass the reference clears seven weighted-sum arrays, sweeps
// every line against the direction of motion (a droplet moves its water
// one cell on, adding water-weighted droplet values to the receiving
// cell), then replaces the droplet values of every droplet cell by the
// weighted means.  A cell's sums receive their last term one step after
// the cell itself is swept (from the cell swept next, which moves water
// into it), so the line walk below keeps the sums of the previous cell in
// registers and finishes that cell -- its F and its means -- right after
// the next step: the same terms added in the same order as the
// reference's arrays, with no scratch arrays.
#include <mutex>
#include "cadmas_dev.cuh"
#include "kernels.h"

namespace cadmas {

#define XX_(m, i) gx(g, m, i)
#define YY_(m, j) gy(g, m, j)
#define ZZ_(m, k) gz(g, m, k)

__device__ __forceinline__ void drop_clear(const DropArrays &d, long long c) {
  d.tx[c] = -1.0e10; d.ty[c] = 0.0; d.tz[c] = 0.0; d.uu[c] = 0.0; d.vv[c] = 0.0; d.ww[c] = 0.0;
}

// ------------------------------------------------------ vf_fdropf.f:69-290
__global__ void k_drop_start(Geo g, Fld f, Prm p, DropArrays d) {
  const int ni = g.NI - 2, nj = g.NJ - 2, nk = g.NK - 2;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)ni * nj * nk) return;
  const int I = 2 + (int)(t % ni), J = 2 + (int)((t / ni) % nj), K = 2 + (int)(t / ((long long)ni * nj));
  const long long c = cid(g, I, J, K);
  if (!(f.ff[c] > p.flower && f.nf[c] == 8)) {
    drop_clear(d, c);
    return;
  }
  const int *NF = f.nf;
  if (d.tx[c] < 0.0) {  // a new droplet
    d.tx[c] = p.tnow; d.ty[c] = p.tnow; d.tz[c] = p.tnow;
    int IP = 0;
    double UP = 0.0, VP = 0.0, WP = 0.0;
    auto take = [&](int i, int j, int k) {
      IP = IP + 1;
      UP = UP + 0.5 * (f.uu[cid(g, i + 1, j, k)] + f.uu[cid(g, i, j, k)]);
      VP = VP + 0.5 * (f.vv[cid(g, i, j + 1, k)] + f.vv[cid(g, i, j, k)]);
      WP = WP + 0.5 * (f.ww[cid(g, i, j, k + 1)] + f.ww[cid(g, i, j, k)]);
    };
    // fluid neighbour across an edge, reached past an open face cell a or b
    auto edge = [&](int i1, int j1, int k1, long long a, long long b) {
      if (NF[cid(g, i1, j1, k1)] == 0 && (NF[a] != -1 || NF[b] != -1)) take(i1, j1, k1);
    };
    for (int dk = -1; dk <= 1; dk += 2)  // x-z plane (:79-114)
      for (int di = -1; di <= 1; di += 2) edge(I + di, J, K + dk, cid(g, I + di, J, K), cid(g, I, J, K + dk));
    for (int dj = -1; dj <= 1; dj += 2)  // x-y plane (:115-150)
      for (int di = -1; di <= 1; di += 2) edge(I + di, J + dj, K, cid(g, I + di, J, K), cid(g, I, J + dj, K));
    for (int dk = -1; dk <= 1; dk += 2)  // y-z plane (:151-186)
      for (int dj = -1; dj <= 1; dj += 2) edge(I, J + dj, K + dk, cid(g, I, J + dj, K), cid(g, I, J, K + dk));
    if (IP == 0) {  // face neighbours that are fluid or surface, x, z, y (:188-231)
      const int nb[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, 0, -1}, {0, 0, 1}, {0, -1, 0}, {0, 1, 0}};
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        const int N1 = NF[cid(g, I + nb[q][0], J + nb[q][1], K + nb[q][2])];
        if (N1 != -1 && N1 != 8) take(I + nb[q][0], J + nb[q][1], K + nb[q][2]);
      }
    }
    double du, dv, dw;
    if (IP >= 1) {
      const double CP = 1.0 / (double)IP;
      du = UP * CP; dv = VP * CP; dw = WP * CP;
    } else {  // its own cell-centre velocity
      du = 0.5 * (f.uu[c] + f.uu[cid(g, I + 1, J, K)]);
      dv = 0.5 * (f.vv[c] + f.vv[cid(g, I, J + 1, K)]);
      dw = 0.5 * (f.ww[c] + f.ww[cid(g, I, J, K + 1)]);
    }
    if (NF[cid(g, I, J, K - 1)] == -1) { du = 0.0; dv = 0.0; dw = 0.0; }  // resting on an obstacle
    d.uu[c] = du; d.vv[c] = dv; d.ww[c] = dw;
  } else if (NF[cid(g, I, J, K - 1)] == -1) {  // an old droplet on an obstacle slides (:253-280)
    auto h = [&](long long n) { return NF[n] == -1 ? 1.0 : 1.0 - f.ggv[n]; };
    double HX = 0.5 * (h(cid(g, I + 1, J, K)) - h(cid(g, I - 1, J, K))) * ZZ_(2, K);
    double HY = 0.5 * (h(cid(g, I, J + 1, K)) - h(cid(g, I, J - 1, K))) * ZZ_(2, K);
    HX = HX / XX_(2, I);
    HY = HY / YY_(2, J);
    const double DN = 1.0 / (HX * HX + HY * HY + 1.0);
    HX = -(p.grz0 * HX * DN);
    HY = -(p.grz0 * HY * DN);
    d.uu[c] = d.uu[c] + p.dtnow * HX;
    d.vv[c] = d.vv[c] + p.dtnow * HY;
  }
}

// ---------------------------------------------------- vf_fdropf.f:292-610
// Weighted sums of one cell (WKTX..WKFF of the reference).
struct DropSums {
  double tx, ty, tz, uu, vv, ww, ff;
};

// Walk one line along axis AX (0 x, 1 y, 2 z) for direction L (1: +, 2: -).
// (I,J,K) give the line (the AX component is ignored); F(s)/setF/NF(s)
// read and write the line's F and NF at position s of the axis.  Writes
// that would store the value already there are left out: F is written only
// where water moved, and the reference's clearing of every cell that holds
// no droplet water is done only for cells that lost it in this pass -- the
// others hold the cleared values already (k_drop_start cleared every
// non-droplet cell, and a droplet cell that runs dry is cleared in the
// step that empties it).  Returns whether any F changed.
// next(s) gives the first position at or after s in walk order (s itself
// when stepping through every cell) that may hold a droplet, or DROP_END:
// the walk visits only those.  Skipping a stretch of cells that hold no
// droplet changes nothing: such a cell only finishes its predecessor and
// becomes the next cell's predecessor with no sums and unchanged F, which
// the walk sets up again at the next droplet (F of a cell is changed only
// by the walk's visits to it and to the cell after it, so a cell not yet
// visited still holds its starting value).
constexpr int DROP_END = -(1 << 30);
template <int AX, class FGet, class FSet, class NGet, class Next>
__device__ __forceinline__ bool drop_walk(const Geo &g, const Fld &f, const Prm &p, const DropArrays &d, int L, int I,
                                          int J, int K, FGet F, FSet setF, NGet NFat, Next next) {
  const int NA = AX == 0 ? g.NI : (AX == 1 ? g.NJ : g.NK);
  const int lo = 2, hi = NA - 1, dl = (L == 1) ? -1 : 1;
  const int s0 = (L == 1) ? hi : lo, s1 = (L == 1) ? lo : hi;
  const double FL = p.flower, G = p.grz0, SG = (L == 1) ? 1.0 : -1.0;
  auto at = [&](int s) -> long long {
    return AX == 0 ? cid(g, s, J, K) : (AX == 1 ? cid(g, I, s, K) : cid(g, I, J, s));
  };
  auto vol = [&](int s) -> double {  // XX(2,I)*YY(2,J)*ZZ(2,K) of the cell at s
    const int i = AX == 0 ? s : I, j = AX == 1 ? s : J, k = AX == 2 ? s : K;
    return XX_(2, i) * YY_(2, j) * ZZ_(2, k);
  };
  auto fvol = [&](double Fv, int s) -> double {  // FF*XX(2,I)*YY(2,J)*ZZ(2,K), left to right
    const int i = AX == 0 ? s : I, j = AX == 1 ? s : J, k = AX == 2 ? s : K;
    return Fv * XX_(2, i) * YY_(2, j) * ZZ_(2, k);
  };
  // the cell swept before (position q): its F, NF and sums
  int q = s0 - dl;
  double Fq = F(q);
  int Nq = NFat(q);
  bool dq = false;  // F of cell q changed
  bool any = false;
  DropSums Wq = {0, 0, 0, 0, 0, 0, 0};
  auto finish = [&](int s, double Fs, int Ns, bool dirty, const DropSums &W) {
    if (dirty) { setF(s, Fs); any = true; }
    if (s < lo || s > hi || !(Fs > FL && Ns == 8)) return;
    const long long c = at(s);
    const double w = 1.0 / W.ff;
    d.tx[c] = W.tx * w; d.ty[c] = W.ty * w; d.tz[c] = W.tz * w;
    double du = W.uu * w, dv = W.vv * w, dw = W.ww * w;
    if (AX == 2 && L == 1) {  // stopped under a ceiling (:590-597)
      const double X = sqrt(2.0 * G * ZZ_(2, s));
      const int Nu = NFat(s + 1);
      if (Nu == -1 && dw > X) { du = 0.0; dv = 0.0; dw = 0.0; }
    }
    d.uu[c] = du; d.vv[c] = dv; d.ww[c] = dw;
  };
  for (int s = next(s0); s != DROP_END; s = (s == s1) ? DROP_END : next(s + dl)) {
    if (s - dl != q) {  // cells skipped since q: q is complete, s-dl is s's predecessor
      finish(q, Fq, Nq, dq, Wq);
      q = s - dl; Fq = F(q); Nq = NFat(q); dq = false; Wq = DropSums{0, 0, 0, 0, 0, 0, 0};
    }
    const long long c = at(s);
    double Fs = F(s);
    const int Ns = NFat(s);
    DropSums W = {0, 0, 0, 0, 0, 0, 0};
    bool ds = false;
    if (Fs > FL && Ns == 8) {
      const double tx = d.tx[c], ty = d.ty[c], tz = d.tz[c], du = d.uu[c], dv = d.vv[c], dw = d.ww[c];
      double DT = 0.0;
      bool go = false;
      if (Nq != -1) {
        if (AX < 2) {
          const double D = AX == 0 ? du : dv;
          if (SG * D > 0.0) {
            DT = (AX == 0 ? XX_(2, s) : YY_(2, s)) / fabs(D);
            go = (p.tnow - (AX == 0 ? tx : ty)) > DT;
            if (!go) DT = 0.0;
          }
        } else {
          const double X = sqrt(2.0 * G * ZZ_(2, s));
          if (L == 1) {
            if (dw > X) DT = (dw - sqrt(dw * dw - X * X)) / G;
          } else if (dw <= X) {
            if (dw <= 0.0) DT = (dw + sqrt(dw * dw + X * X)) / G;
            else DT = 2.0 * dw / G;
          }
          go = DT > 0.0 && (p.tnow - tz) > DT;
          if (!go) DT = 0.0;
        }
      }
      // droplet values carried by this cell's water in this pass
      const double vx = AX == 0 ? tx + DT : tx, vy = AX == 1 ? ty + DT : ty, vz = AX == 2 ? tz + DT : tz,
                   vw = AX == 2 ? dw - DT * G : dw;
      if (go) {
        const long long cq = at(q);
        const double V0 = vol(s) * f.ggv[c], V1 = vol(q) * f.ggv[cq];
        const double FMOVE = dmin((1.0 - Fq) * V1, Fs * V0);
        Fs = Fs - FMOVE / V0;
        Fq = Fq + FMOVE / V1;
        ds = true; dq = true;
        if (Nq == 8) {
          Wq.tx = Wq.tx + FMOVE * vx; Wq.ty = Wq.ty + FMOVE * vy; Wq.tz = Wq.tz + FMOVE * vz;
          Wq.uu = Wq.uu + FMOVE * du; Wq.vv = Wq.vv + FMOVE * dv; Wq.ww = Wq.ww + FMOVE * vw;
          Wq.ff = Wq.ff + FMOVE;
        }
      }
      if (Fs > FL) {  // the water that stays
        const double FOLD = fvol(Fs, s) * f.ggv[c];
        W.tx = 0.0 + FOLD * vx; W.ty = 0.0 + FOLD * vy; W.tz = 0.0 + FOLD * vz;
        W.uu = 0.0 + FOLD * du; W.vv = 0.0 + FOLD * dv; W.ww = 0.0 + FOLD * vw;
        W.ff = 0.0 + FOLD;
      } else {
        drop_clear(d, c);  // its water moved on
      }
    }
    // the cell before is complete now
    finish(q, Fq, Nq, dq, Wq);
    q = s; Fq = Fs; Nq = Ns; dq = ds; Wq = W;
  }
  finish(q, Fq, Nq, dq, Wq);
  return any;
}

// y and z lines: one thread per line; consecutive threads take consecutive I.
// The thread finds the droplet cells of its line 32 walk positions at a
// time (the loads of a group issued together, its droplet mask kept) and
// walks from droplet to droplet.
template <int AX>
__global__ void k_drop_line(Geo g, Fld f, Prm p, DropArrays d, int L) {
  const int ni = g.NI - 2, nb = AX == 1 ? g.NK - 2 : g.NJ - 2;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)ni * nb) return;
  const int I = 2 + (int)(t % ni), o = 2 + (int)(t / ni);
  const int J = AX == 1 ? 0 : o, K = AX == 1 ? o : 0;
  double *FF = f.ff;
  const int *NF = f.nf;
  auto at = [&](int s) -> long long { return AX == 1 ? cid(g, I, s, K) : cid(g, I, J, s); };
  const int NA = AX == 1 ? g.NJ : g.NK, dl = (L == 1) ? -1 : 1, s0 = (L == 1) ? NA - 1 : 2, n = NA - 2;
  const double FL = p.flower;
  int cc = -1;      // group of walk positions whose mask is held
  unsigned cm = 0;  // its droplet cells (bit j: walk position 32*cc + j)
  auto next = [&](int s) -> int {
    int u = (s - s0) * dl;
    while (u < n) {
      const int cu = u >> 5;
      if (cu != cc) {
        unsigned m = 0;
#pragma unroll 8
        for (int j = 0; j < 32; ++j) {
          const int uu = (cu << 5) + j;
          if (uu < n) {
            const long long a = at(s0 + uu * dl);
            const double fv = FF[a];
            const int nv = NF[a];
            if (fv > FL && nv == 8) m |= 1u << j;
          }
        }
        cc = cu;
        cm = m;
      }
      const unsigned bits = cm & (0xffffffffu << (u & 31));
      if (bits) return s0 + ((cu << 5) + __ffs(bits) - 1) * dl;
      u = (cu + 1) << 5;
    }
    return DROP_END;
  };
  drop_walk<AX>(g, f, p, d, L, I, J, K, [&](int s) { return FF[at(s)]; },
                [&](int s, double v) { FF[at(s)] = v; }, [&](int s) { return NF[at(s)]; }, next);
}

// x lines: one warp per line (J,K); the warp stages the line's F and NF
// (I = 1..NI) in shared memory with a mask of its droplet cells (bit I-1),
// and leaves the line at once when it holds none.  Lane 0 walks from
// droplet to droplet; the warp writes F back if it changed.
__global__ void k_drop_line_x(Geo g, Fld f, Prm p, DropArrays d, int L) {
  extern __shared__ __align__(16) double dsm[];
  const int NI = g.NI, lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int nw = (NI + 31) >> 5;
  const long long line = (long long)blockIdx.x * wpb + wib;
  const int nj = g.NJ - 2;
  if (line >= (long long)nj * (g.NK - 2)) return;
  const int J = 2 + (int)(line % nj), K = 2 + (int)(line / nj);
  double *Fs = dsm + (size_t)wib * NI;  // F(1..NI) at Fs[0..NI-1]
  int *Ns = reinterpret_cast<int *>(dsm + (size_t)wpb * NI) + (size_t)wib * NI;
  unsigned *Ds = reinterpret_cast<unsigned *>(reinterpret_cast<int *>(dsm + (size_t)wpb * NI) + (size_t)wpb * NI) +
                 (size_t)wib * nw;
  const long long row = cid(g, 1, J, K);
  const double FL = p.flower;
  unsigned anyd = 0;
  for (int base = 0; base < NI; base += 32) {
    const int i = base + lane;
    bool dr = false;
    if (i < NI) {
      const double fv = f.ff[row + i];
      const int nv = f.nf[row + i];
      Fs[i] = fv; Ns[i] = nv;
      dr = i >= 1 && i <= NI - 2 && fv > FL && nv == 8;  // interior I = 2..NI-1
    }
    const unsigned m = __ballot_sync(0xffffffffu, dr);
    if (lane == 0) Ds[base >> 5] = m;
    anyd |= m;
  }
  if (anyd == 0) return;  // the same for every lane of the warp
  __syncwarp();
  bool any = false;
  if (lane == 0) {
    // first droplet at or after position s in walk order (s = I)
    auto next_up = [&](int s) -> int {  // L = 2: increasing I
      if (s > NI - 1) return DROP_END;
      int x = s - 1, w = x >> 5;
      unsigned bits = Ds[w] & (0xffffffffu << (x & 31));
      while (bits == 0) {
        if (++w >= nw) return DROP_END;
        bits = Ds[w];
      }
      return (w << 5) + __ffs(bits);  // (w*32 + bit) + 1
    };
    auto next_down = [&](int s) -> int {  // L = 1: decreasing I
      if (s < 2) return DROP_END;
      int x = s - 1, w = x >> 5;
      unsigned bits = Ds[w] & (0xffffffffu >> (31 - (x & 31)));
      while (bits == 0) {
        if (--w < 0) return DROP_END;
        bits = Ds[w];
      }
      return (w << 5) + (31 - __clz(bits)) + 1;
    };
    auto F = [&](int s) { return Fs[s - 1]; };
    auto setF = [&](int s, double v) { Fs[s - 1] = v; };
    auto NFat = [&](int s) { return Ns[s - 1]; };
    any = (L == 1) ? drop_walk<0>(g, f, p, d, L, 0, J, K, F, setF, NFat, next_down)
                   : drop_walk<0>(g, f, p, d, L, 0, J, K, F, setF, NFat, next_up);
  }
  any = __shfl_sync(0xffffffffu, any, 0);
  __syncwarp();
  if (any)
    for (int i = lane; i < NI; i += 32) f.ff[row + i] = Fs[i];
}

// Shared memory of one warp of k_drop_line_x: F and NF of a whole x line
// and its droplet mask.
static size_t drop_x_bytes(const Geo &g) { return (size_t)g.NI * 12 + (size_t)((g.NI + 31) / 32) * 4; }
// Warps per block of k_drop_line_x.
static int drop_x_warps(const Geo &g) {
  const size_t per = drop_x_bytes(g);
  for (int w : {4, 2, 1})
    if (per * w <= 96 * 1024) return w;
  return 0;
}
bool drop_supported(const Geo &g) { return drop_x_bytes(g) <= 200 * 1024; }

void launch_fdropf(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, const DropArrays &d) {
  const long long ncell = (long long)(g.NI - 2) * (g.NJ - 2) * (g.NK - 2);
  k_drop_start<<<(unsigned)((ncell + 255) / 256), 256, 0, s>>>(g, f, p, d);
  count_launch();
  int wpb = drop_x_warps(g);
  if (wpb == 0) wpb = 1;
  const size_t xsm = drop_x_bytes(g) * wpb;
  // the limit only rises (handles of other grids may be stepped from other
  // host threads at the same time)
  raise_dynamic_smem((const void *)k_drop_line_x, xsm);
  const long long nx = (long long)(g.NJ - 2) * (g.NK - 2);
  const long long ny = (long long)(g.NI - 2) * (g.NK - 2), nz = (long long)(g.NI - 2) * (g.NJ - 2);
  for (int L = 1; L <= 2; ++L) {
    k_drop_line_x<<<(unsigned)((nx + wpb - 1) / wpb), 32 * wpb, xsm, s>>>(g, f, p, d, L);
    count_launch();
  }
  for (int L = 1; L <= 2; ++L) {
    k_drop_line<1><<<(unsigned)((ny + 127) / 128), 128, 0, s>>>(g, f, p, d, L);
    count_launch();
  }
  for (int L = 1; L <= 2; ++L) {
    k_drop_line<2><<<(unsigned)((nz + 127) / 128), 128, 0, s>>>(g, f, p, d, L);
    count_launch();
  }
}

// DROPTX..DROPWW at their start values (vf_cinit.f:412-427).
__global__ void k_drop_reset(long long n, DropArrays d) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
    drop_clear(d, c);
}
void launch_drop_reset(cudaStream_t s, long long n, const DropArrays &d) {
  k_drop_reset<<<(unsigned)std::min<long long>((n + 255) / 256, 148LL * 16), 256, 0, s>>>(n, d);
  count_launch();
}

}  // namespace cadmas
