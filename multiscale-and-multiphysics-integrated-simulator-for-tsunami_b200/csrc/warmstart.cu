// warmstart.cu -- the learned initial guess of the pressure solve
// (warm_start = 2): the hook that replaces PT = 0 of VF_VPSOL
// (vf_vpsol.f:52-58).
//
//   k_ws_rows      row partials of BB^2 and of the count of computed cells
//   k_ws_scale     s = sqrt(mean BB^2) over INDC != -1 (1 if none)
//   k_ws_features  the network's input per voxel (x,y,z) = cell (x+1,y+1,z+1):
//                  BB/s, F, GGV, INDC != -1; zeros outside the grid
//   k_ws_output    PT = s c y on interior INDC != -1 cells, else 0 (c the
//                  network's output scale)
//   k_ws_resid     row partials of |BB - A PT|^2 and |BB|^2 (A as VF_MZAX
//                  applies it, vf_mzax.f:42-56) over interior INDC != -1
//   k_ws_decide    keep the guess only if |BB - A PT| < |BB| (a NaN or a
//                  network timeout drops it too) and count the outcome
//   k_ws_clear     PT = 0 when dropped
// Sums use the fixed row tree (row_store, block_final), so the guess and
// the decision are the same from run to run.
#include "cadmas_dev.cuh"
#include "kernels.h"

namespace cadmas {

#define A(a, i, j, k) a[cid(g, i, j, k)]

__device__ __forceinline__ bool ws_inner(const Geo &g, int I, int J, int K) {
  return I >= 2 && I <= g.NI - 1 && J >= 2 && J <= g.NJ - 1 && K >= 2 && K <= g.NK - 1;
}

__global__ void k_ws_rows(Geo g, const int *INDC, const double *BB, double *r0, double *r1) {
  const long long nrows = (long long)g.NJ * g.NK;
  double s = 0.0, n = 0.0;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  if (ws_inner(g, I, J, K) && INDC[c] != -1) { s = s + BB[c] * BB[c]; n = n + 1.0; }
  ROW_LOOP_END
  row_store(s, r0, row_, nrows);
  row_store(n, r1, row_, nrows);
}

__global__ void k_ws_scale(const double *r0, const double *r1, long long nrows, double *scal) {
  const double s = block_final(r0, nrows);
  const double n = block_final(r1, nrows);
  if (threadIdx.x == 0) scal[0] = (n > 0.0 && s > 0.0) ? sqrt(s / n) : 1.0;
}

__global__ void k_ws_features(Geo g, Fld f, const double *BB, const double *scal, float *x4, int X, int Y, int Z) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)X * Y * Z) return;
  const int x = (int)(i % X), y = (int)((i / X) % Y), z = (int)(i / ((long long)X * Y));
  const int I = x + 1, J = y + 1, K = z + 1;
  float v0 = 0.0f, v1 = 0.0f, v2 = 0.0f, v3 = 0.0f;
  if (I <= g.NI && J <= g.NJ && K <= g.NK) {
    const long long c = cid(g, I, J, K);
    const bool live = f.indc[c] != -1;
    v0 = live ? (float)(BB[c] / scal[0]) : 0.0f;
    v1 = (float)f.ff[c];
    v2 = (float)f.ggv[c];
    v3 = live ? 1.0f : 0.0f;
  }
  x4[4 * i + 0] = v0; x4[4 * i + 1] = v1; x4[4 * i + 2] = v2; x4[4 * i + 3] = v3;
}

__global__ void k_ws_output(Geo g, const int *INDC, const float *y, const double *scal, double *PT, int X, int Y) {
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  double v = 0.0;
  if (ws_inner(g, I, J, K) && INDC[c] != -1)
    v = scal[0] * scal[3] * (double)y[(long long)(I - 1) + (long long)X * ((long long)(J - 1) + (long long)Y * (K - 1))];
  PT[c] = v;
  ROW_LOOP_END
}

__global__ void k_ws_resid(Geo g, SysPtr a, const int *INDC, const double *PT, double *r0, double *r1) {
  const long long nrows = (long long)g.NJ * g.NK;
  double sr = 0.0, sb = 0.0;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  if (ws_inner(g, I, J, K) && INDC[c] != -1) {
    const double ax = a.ad[c] * PT[c] + a.ali[c] * A(PT, I - 1, J, K) + a.alj[c] * A(PT, I, J - 1, K) +
                      a.alk[c] * A(PT, I, J, K - 1) + a.aui[c] * A(PT, I + 1, J, K) + a.auj[c] * A(PT, I, J + 1, K) +
                      a.auk[c] * A(PT, I, J, K + 1);
    const double r = a.bb[c] - ax;
    sr = sr + r * r;
    sb = sb + a.bb[c] * a.bb[c];
  }
  ROW_LOOP_END
  row_store(sr, r0, row_, nrows);
  row_store(sb, r1, row_, nrows);
}

__global__ void k_ws_decide(const double *r0, const double *r1, long long nrows, const int *net_err, double *scal,
                            int *cnt) {
  const double r2 = block_final(r0, nrows);
  const double b2 = block_final(r1, nrows);
  if (threadIdx.x == 0) {
    const bool keep = (r2 < b2) && *net_err == 0;
    scal[1] = r2;
    scal[2] = b2;
    cnt[2] = keep ? 0 : 1;
    cnt[keep ? 0 : 1] += 1;
  }
}

__global__ void k_ws_clear(long long n, const int *cnt, double *PT) {
  if (cnt[2] == 0) return;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    PT[i] = 0.0;
}

#undef A

void launch_warm_guess(cudaStream_t s, const Geo &g, const Fld &f, const SysPtr &a, cadmas_unet *net, double *rows0,
                       double *rows1, double *scal, int *cnt, double *PT) {
  const long long nrows = (long long)g.NJ * g.NK;
  int X, Y, Z;
  unet_dims(net, X, Y, Z);
  k_ws_rows<<<row_blocks(g), ROW_THREADS, 0, s>>>(g, f.indc, a.bb, rows0, rows1);
  k_ws_scale<<<1, 1024, 0, s>>>(rows0, rows1, nrows, scal);
  const long long V = (long long)X * Y * Z;
  k_ws_features<<<(unsigned)((V + 255) / 256), 256, 0, s>>>(g, f, a.bb, scal, unet_input(net), X, Y, Z);
  count_launch(3);
  unet_run_forward(net);
  k_ws_output<<<row_blocks(g), ROW_THREADS, 0, s>>>(g, f.indc, unet_output(net), scal, PT, X, Y);
  k_ws_resid<<<row_blocks(g), ROW_THREADS, 0, s>>>(g, a, f.indc, PT, rows0, rows1);
  k_ws_decide<<<1, 1024, 0, s>>>(rows0, rows1, nrows, unet_error(net), scal, cnt);
  k_ws_clear<<<296, 256, 0, s>>>(g.N, cnt, PT);
  count_launch(4);
}

}  // namespace cadmas
