// k_unet.cu -- kernels of the learned warm start: a 3-level 3-D U-Net
// (BF16 weights and activations, FP32 accumulation) that maps (right-hand
// side, F, porosity, computed-cell mask) to an initial pressure correction.
//
// The 3x3x3 convolutions are implicit GEMMs on the tcgen05 tensor cores:
//   k_conv   D[voxel, cout] = sum over 27 taps and cin of X[voxel+tap, cin]
//            * W[cout, tap, cin].  A CTA of 128 threads owns 128 voxels
//            (M = 128) and all Cout (N); per tap every thread gathers its
//            voxel's neighbour row (Cin BF16 values, zero outside the
//            volume) into a shared-memory stage while the MMAs of the
//            previous tap run; one thread issues Cin/16 MMAs (K = 16) per
//            tap into a TMEM accumulator and commits them to the stage's
//            mbarrier.  The epilogue reads TMEM (tcgen05.ld), adds the
//            bias, applies ReLU or a ReLU-backward mask and stores BF16 or
//            FP32.  The input-gradient of a convolution is the same kernel
//            with the weights flipped and transposed.
//   k_wgrad  dW[(tap,cin), cout] = sum over voxels of X[voxel+tap, cin] *
//            dY[voxel, cout]: M = 27*Cin rows in tiles of 128, N = Cout,
//            K = a slice of voxels in chunks of 64; each CTA writes its
//            slice's partial sums, which k_wgrad_reduce adds in slice order.
// The rest are elementwise or gather kernels on CUDA cores.
//
// Layouts: activations channels-last, voxel v = x + X*(y + Y*(z + Z*b)),
// value [v*C + c]; weights [cout][tap][cin] with tap = (dz+1)*9 + (dy+1)*3
// + (dx+1).  Every wait on an mbarrier is bounded: on a timeout the CTA
// records an error, waits once more for its MMAs, frees its TMEM and ends.
#include <cuda_bf16.h>
#include "cadmas_dev.cuh"
#include "kernels.h"
#include "umma.cuh"

namespace cadmas {

using bf16 = __nv_bfloat16;

struct Vol {
  int X, Y, Z, B;
  __host__ __device__ __forceinline__ long long n() const { return (long long)X * Y * Z * B; }
};

// neighbour voxel of v at (dx,dy,dz), or -1 outside the volume
__device__ __forceinline__ long long nbr(const Vol &g, int x, int y, int z, int b, int dx, int dy, int dz) {
  const int xx = x + dx, yy = y + dy, zz = z + dz;
  if (xx < 0 || xx >= g.X || yy < 0 || yy >= g.Y || zz < 0 || zz >= g.Z) return -1;
  return (long long)xx + (long long)g.X * ((long long)yy + (long long)g.Y * ((long long)zz + (long long)g.Z * b));
}

__device__ __forceinline__ void decomp(const Vol &g, long long v, int &x, int &y, int &z, int &b) {
  x = (int)(v % g.X);
  long long r = v / g.X;
  y = (int)(r % g.Y);
  r /= g.Y;
  z = (int)(r % g.Z);
  b = (int)(r / g.Z);
}

// Every thread waits (bounded) for the phase of the given parity; the CTA
// goes on only if all of them saw it, so that no thread is left at a later
// barrier.
__device__ __forceinline__ bool cta_wait(uint64_t *bar, uint32_t parity) {
  const bool w = umma::mbar_wait(bar, parity);
  return __syncthreads_and(w) != 0;
}

// ------------------------------------------------------------- k_conv
// dynamic shared memory: A stages 2 x 128*KC, B stages 2 x N*KC (BF16),
// then 2 mbarriers and the TMEM address.
constexpr int CONV_M = 128;

__global__ void __launch_bounds__(128) k_conv(Vol g, const bf16 *__restrict__ X, int Cin,
                                              const bf16 *__restrict__ W, const float *__restrict__ bias,
                                              int Cout, int mode, const bf16 *__restrict__ mask, void *Y,
                                              int *err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const int KC = Cin, N = Cout;
  const uint32_t a_bytes = CONV_M * KC * 2, b_bytes = N * KC * 2;
  unsigned char *As[2] = {smem, smem + a_bytes};
  unsigned char *Bs[2] = {smem + 2 * a_bytes, smem + 2 * a_bytes + b_bytes};
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + 2 * a_bytes + 2 * b_bytes);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 2);
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t ncols = umma::tmem_cols(N);
  if (warp == 0) umma::tmem_alloc(tslot, ncols);
  if (tid == 0) {
    umma::mbar_init(&bar[0], 1);
    umma::mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *tslot;
  const uint32_t idesc = umma::idesc_bf16_f32(CONV_M, N);

  const long long V = g.n();
  const long long v = (long long)blockIdx.x * CONV_M + tid;
  int x = 0, y = 0, z = 0, b = 0;
  const bool live = v < V;
  if (live) decomp(g, v, x, y, z, b);
  bool ok = true;
  int committed = 0;  // commits issued
  for (int t = 0; t < 27 && ok; ++t) {
    const int s = t & 1;
    if (t >= 2) {
      // the MMAs of tap t-2 have read stage s
      if (!cta_wait(&bar[s], ((t - 2) >> 1) & 1)) { ok = false; break; }
    }
    // A: this thread's row
    const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
    const long long nv = live ? nbr(g, x, y, z, b, dx, dy, dz) : -1;
    const uint4 zero = make_uint4(0, 0, 0, 0);
    for (int c8 = 0; c8 < KC / 8; ++c8) {
      uint4 q = zero;
      if (nv >= 0) q = *reinterpret_cast<const uint4 *>(X + nv * Cin + c8 * 8);
      *reinterpret_cast<uint4 *>(As[s] + umma::kmajor_offset(CONV_M, tid, c8 * 8)) = q;
    }
    // B: the tap's N x KC weights; consecutive threads take consecutive
    // rows n, whose 16-byte chunks are adjacent in the core matrices
    const int nq = N * (KC / 8);
    for (int q = tid; q < nq; q += 128) {
      const int n = q % N, c8 = q / N;
      const uint4 w = *reinterpret_cast<const uint4 *>(W + ((long long)n * 27 + t) * Cin + c8 * 8);
      *reinterpret_cast<uint4 *>(Bs[s] + umma::kmajor_offset(N, n, c8 * 8)) = w;
    }
    umma::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      umma::fence_after_sync();
      const uint32_t a0 = umma::smem_u32(As[s]), b0 = umma::smem_u32(Bs[s]);
      for (int kk = 0; kk < KC / 16; ++kk) {
        const uint64_t ad = umma::smem_desc(a0 + kk * 2 * CONV_M * 16, CONV_M * 16, 128);
        const uint64_t bd = umma::smem_desc(b0 + kk * 2 * N * 16, N * 16, 128);
        umma::mma_bf16(tmem, ad, bd, idesc, (t | kk) != 0);
      }
      umma::mma_commit(&bar[s]);
    }
    ++committed;
  }
  // the last commit covers every MMA issued before it
  if (committed > 0) {
    // on an earlier timeout this is the one more bounded wait for the MMAs
    // in flight before the TMEM is freed
    const int tl = committed - 1;
    if (!cta_wait(&bar[tl & 1], (tl >> 1) & 1)) ok = false;
  }
  if (!ok) {
    if (tid == 0) atomicOr(err, 1);
  } else {
    umma::fence_after_sync();
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
    for (int c0 = 0; c0 < N; c0 += 8) {
      float a[8];
      umma::tmem_ld8(lane_base + c0, a);
      if (!live) continue;
      if (bias)
#pragma unroll
        for (int i = 0; i < 8; ++i) a[i] += bias[c0 + i];
      if (mode == CONV_RELU_BF16) {
#pragma unroll
        for (int i = 0; i < 8; ++i) a[i] = fmaxf(a[i], 0.0f);
      } else if (mode == CONV_MASK_BF16) {
        // input gradient times the ReLU derivative of the layer below
        const uint4 mq = *reinterpret_cast<const uint4 *>(mask + v * Cout + c0);
        const bf16 *m = reinterpret_cast<const bf16 *>(&mq);
#pragma unroll
        for (int i = 0; i < 8; ++i) a[i] = (__bfloat162float(m[i]) > 0.0f) ? a[i] : 0.0f;
      }
      if (mode == CONV_F32) {
        float *o = reinterpret_cast<float *>(Y) + v * Cout + c0;
#pragma unroll
        for (int i = 0; i < 8; ++i) o[i] = a[i];
      } else {
        __align__(16) bf16 o[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) o[i] = __float2bfloat16(a[i]);
        *reinterpret_cast<uint4 *>(reinterpret_cast<bf16 *>(Y) + v * Cout + c0) = *reinterpret_cast<uint4 *>(o);
      }
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_free(tmem, ncols);
}

// ------------------------------------------------------------ k_wgrad
// rows m = tap*Cin + cin (27*Cin of them, tiles of 128), N = Cout, K = the
// voxels of this CTA's slice in chunks of 64.
constexpr int WG_K = 64;

__global__ void __launch_bounds__(128) k_wgrad(Vol g, const bf16 *__restrict__ X, int Cin,
                                               const bf16 *__restrict__ DY, int Cout, long long slice,
                                               float *__restrict__ part, int *err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const int N = Cout;
  const uint32_t a_bytes = 128 * WG_K * 2, b_bytes = N * WG_K * 2;
  unsigned char *As[2] = {smem, smem + a_bytes};
  unsigned char *Bs[2] = {smem + 2 * a_bytes, smem + 2 * a_bytes + b_bytes};
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + 2 * a_bytes + 2 * b_bytes);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 2);
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t ncols = umma::tmem_cols(N);
  if (warp == 0) umma::tmem_alloc(tslot, ncols);
  if (tid == 0) {
    umma::mbar_init(&bar[0], 1);
    umma::mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *tslot;
  const uint32_t idesc = umma::idesc_bf16_f32(128, N);
  const int M = 27 * Cin;
  const int m0 = blockIdx.x * 128;
  const long long V = g.n();
  const long long v0 = (long long)blockIdx.y * slice;
  const long long v1 = min(V, v0 + slice);
  const int nchunk = (int)((v1 - v0 + WG_K - 1) / WG_K);
  // thread: voxel k = tid % 64 of each chunk, row half h = tid / 64
  const int kq = tid & (WG_K - 1), h = tid >> 6;
  bool ok = true;
  int committed = 0;
  for (int ch = 0; ch < nchunk && ok; ++ch) {
    const int s = ch & 1;
    if (ch >= 2 && !cta_wait(&bar[s], ((ch - 2) >> 1) & 1)) { ok = false; break; }
    const long long v = v0 + (long long)ch * WG_K + kq;
    const bool live = v < v1;
    int x = 0, y = 0, z = 0, b = 0;
    if (live) decomp(g, v, x, y, z, b);
    // A: rows m0 + 64h .. m0 + 64h + 63 of column kq
    for (int r = 64 * h; r < 64 * h + 64; ++r) {
      const int m = m0 + r;
      bf16 val = __float2bfloat16(0.0f);
      if (live && m < M) {
        const int t = m / Cin, ci = m % Cin;
        const long long nv = nbr(g, x, y, z, b, t % 3 - 1, (t / 3) % 3 - 1, t / 9 - 1);
        if (nv >= 0) val = X[nv * Cin + ci];
      }
      *reinterpret_cast<bf16 *>(As[s] + umma::kmajor_offset(128, r, kq)) = val;
    }
    // B: rows n of column kq (half the threads)
    if (h == 0) {
      for (int n = 0; n < N; ++n) {
        const bf16 val = live ? DY[v * Cout + n] : __float2bfloat16(0.0f);
        *reinterpret_cast<bf16 *>(Bs[s] + umma::kmajor_offset(N, n, kq)) = val;
      }
    }
    umma::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      umma::fence_after_sync();
      const uint32_t a0 = umma::smem_u32(As[s]), b0 = umma::smem_u32(Bs[s]);
      for (int kk = 0; kk < WG_K / 16; ++kk) {
        const uint64_t ad = umma::smem_desc(a0 + kk * 2 * 128 * 16, 128 * 16, 128);
        const uint64_t bd = umma::smem_desc(b0 + kk * 2 * N * 16, N * 16, 128);
        umma::mma_bf16(tmem, ad, bd, idesc, (ch | kk) != 0);
      }
      umma::mma_commit(&bar[s]);
    }
    ++committed;
  }
  if (committed > 0) {
    // on an earlier timeout this is the one more bounded wait for the MMAs
    // in flight before the TMEM is freed
    const int tl = committed - 1;
    if (!cta_wait(&bar[tl & 1], (tl >> 1) & 1)) ok = false;
  }
  if (!ok) {
    if (tid == 0) atomicOr(err, 1);
  } else {
    umma::fence_after_sync();
    const int m = m0 + warp * 32 + (tid & 31);
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
    float *o = part + ((long long)blockIdx.y * M + m) * N;
    for (int c0 = 0; c0 < N; c0 += 8) {
      float a[8];
      umma::tmem_ld8(lane_base + c0, a);
      if (m < M && committed > 0)
#pragma unroll
        for (int i = 0; i < 8; ++i) o[c0 + i] = a[i];
      else if (m < M)
#pragma unroll
        for (int i = 0; i < 8; ++i) o[c0 + i] = 0.0f;
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_free(tmem, ncols);
}

// dW[cout][tap][cin] = sum over slices (in order) of part[s][tap*Cin+cin][cout]
__global__ void k_wgrad_reduce(const float *part, int nslices, int Cin, int Cout, float *dW) {
  const int M = 27 * Cin;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M * Cout) return;
  const int m = i / Cout, n = i % Cout;
  float s = 0.0f;
  for (int q = 0; q < nslices; ++q) s += part[((long long)q * M + m) * Cout + n];
  const int t = m / Cin, ci = m % Cin;
  dW[((long long)n * 27 + t) * Cin + ci] = s;
}

// bias gradient: db[c] = sum over voxels of dY[v][c] (FP32 partials per block
// of 1024 voxels, then the same in order)
__global__ void k_bias_part(const bf16 *DY, long long V, int C, float *part) {
  const int c = threadIdx.x;
  if (c >= C) return;
  const long long v0 = (long long)blockIdx.x * 1024, v1 = min(V, v0 + 1024);
  float s = 0.0f;
  for (long long v = v0; v < v1; ++v) s += __bfloat162float(DY[v * C + c]);
  part[(long long)blockIdx.x * C + c] = s;
}
__global__ void k_bias_reduce(const float *part, int nb, int C, float *db) {
  const int c = threadIdx.x;
  if (c >= C) return;
  float s = 0.0f;
  for (int q = 0; q < nb; ++q) s += part[(long long)q * C + c];
  db[c] = s;
}

// ------------------------------------------------ pooling and upsampling
// 2x2x2 average: coarse (X/2, Y/2, Z/2) from fine
__global__ void k_pool(Vol gc, const bf16 *F, int C, bf16 *Cc) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= gc.n() * C) return;
  const long long vc = i / C;
  const int c = (int)(i % C);
  int x, y, z, b;
  decomp(gc, vc, x, y, z, b);
  const Vol gf{2 * gc.X, 2 * gc.Y, 2 * gc.Z, gc.B};
  float s = 0.0f;
  for (int q = 0; q < 8; ++q) {
    const long long vf = nbr(gf, 2 * x, 2 * y, 2 * z, b, q & 1, (q >> 1) & 1, q >> 2);
    s += __bfloat162float(F[vf * C + c]);
  }
  Cc[i] = __float2bfloat16(0.125f * s);
}
// its backward, added to dF (fine) where acc != 0, else stored
__global__ void k_pool_bwd(Vol gc, const bf16 *dC, int C, bf16 *dF, int acc) {
  const Vol gf{2 * gc.X, 2 * gc.Y, 2 * gc.Z, gc.B};
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= gf.n() * C) return;
  const long long vf = i / C;
  const int c = (int)(i % C);
  int x, y, z, b;
  decomp(gf, vf, x, y, z, b);
  const long long vc = (long long)(x >> 1) + (long long)gc.X * ((long long)(y >> 1) + (long long)gc.Y *
                                                                 ((long long)(z >> 1) + (long long)gc.Z * b));
  float d = 0.125f * __bfloat162float(dC[vc * C + c]);
  if (acc) d += __bfloat162float(dF[i]);
  dF[i] = __float2bfloat16(d);
}
// out[vf] = (coarse[vf/2] (C1 channels), skip[vf] (C2 channels))
__global__ void k_upcat(Vol gf, const bf16 *Cc, int C1, const bf16 *S, int C2, bf16 *O) {
  const int C = C1 + C2;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= gf.n() * C) return;
  const long long vf = i / C;
  const int c = (int)(i % C);
  if (c >= C1) { O[i] = S[vf * C2 + (c - C1)]; return; }
  int x, y, z, b;
  decomp(gf, vf, x, y, z, b);
  const Vol gc{gf.X / 2, gf.Y / 2, gf.Z / 2, gf.B};
  const long long vc = (long long)(x >> 1) + (long long)gc.X * ((long long)(y >> 1) + (long long)gc.Y *
                                                                 ((long long)(z >> 1) + (long long)gc.Z * b));
  O[i] = Cc[vc * C1 + c];
}
// backward: dCoarse = sum of the 8 children's first C1 channels; dSkip
// (+)= the last C2 channels
__global__ void k_upcat_bwd_coarse(Vol gc, const bf16 *dO, int C1, int C2, bf16 *dC) {
  const int C = C1 + C2;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= gc.n() * C1) return;
  const long long vc = i / C1;
  const int c = (int)(i % C1);
  int x, y, z, b;
  decomp(gc, vc, x, y, z, b);
  const Vol gf{2 * gc.X, 2 * gc.Y, 2 * gc.Z, gc.B};
  float s = 0.0f;
  for (int q = 0; q < 8; ++q) {
    const long long vf = nbr(gf, 2 * x, 2 * y, 2 * z, b, q & 1, (q >> 1) & 1, q >> 2);
    s += __bfloat162float(dO[vf * C + c]);
  }
  dC[i] = __float2bfloat16(s);
}
__global__ void k_upcat_bwd_skip(long long Vf, const bf16 *dO, int C1, int C2, bf16 *dS, int acc) {
  const int C = C1 + C2;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= Vf * C2) return;
  const long long vf = i / C2;
  const int c = (int)(i % C2);
  float d = __bfloat162float(dO[vf * C + C1 + c]);
  if (acc) d += __bfloat162float(dS[i]);
  dS[i] = __float2bfloat16(d);
}
// dX *= (act > 0) (ReLU backward in place)
__global__ void k_relu_mask(long long n, const bf16 *act, bf16 *d) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (!(__bfloat162float(act[i]) > 0.0f)) d[i] = __float2bfloat16(0.0f);
}

// ------------------------------------------------------------- head
// y[v] = sum_c wh[c] a[v][c] + bh (FP32)
__global__ void k_head(long long V, const bf16 *A, int C, const float *wh, const float *bh, float *Yo) {
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= V) return;
  float s = bh[0];
  for (int c = 0; c < C; ++c) s += wh[c] * __bfloat162float(A[v * C + c]);
  Yo[v] = s;
}
// masked MSE: dy = 2 (y - t) m / sum(m); per-block partial loss sums
__global__ void k_mse(long long V, const float *Yo, const float *T, const float *Mk, float inv_n, float *dy,
                      float *lpart) {
  __shared__ float red[256];
  const long long v = (long long)blockIdx.x * 256 + threadIdx.x;
  float l = 0.0f;
  if (v < V) {
    const float e = (Yo[v] - T[v]) * Mk[v];
    dy[v] = 2.0f * e * inv_n;
    l = e * e;
  }
  red[threadIdx.x] = l;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) lpart[blockIdx.x] = red[0];
}
// head backward: dA[v][c] = dy[v] wh[c] (BF16), masked by the ReLU of A
__global__ void k_head_bwd_act(long long V, const float *dy, const bf16 *A, int C, const float *wh, bf16 *dA) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V * C) return;
  const long long v = i / C;
  const int c = (int)(i % C);
  const float d = (__bfloat162float(A[i]) > 0.0f) ? dy[v] * wh[c] : 0.0f;
  dA[i] = __float2bfloat16(d);
}
// head parameter gradients: partials over blocks of 1024 voxels of
// (dy a[c], dy) in FP32
__global__ void k_head_bwd_par(long long V, const float *dy, const bf16 *A, int C, float *part) {
  const int c = threadIdx.x;
  if (c > C) return;
  const long long v0 = (long long)blockIdx.x * 1024, v1 = min(V, v0 + 1024);
  float s = 0.0f;
  for (long long v = v0; v < v1; ++v) s += dy[v] * (c < C ? __bfloat162float(A[v * C + c]) : 1.0f);
  part[(long long)blockIdx.x * (C + 1) + c] = s;
}

// ---------------------------------------------------- residual loss
// The pressure system of each sample in the network's volume: per voxel
// the 7 coefficients (AD, ALI, ALJ, ALK, AUI, AUJ, AUK, FP32) of VF_MZAX's
// row (vf_mzax.f:42-56), b = the input's channel 0 (BB/s).  With the output
// y, taken as 0 off the counted cells as the solver's guess is, and the
// fixed scale c: r = m (b - c A (m y)); loss |r|^2 / sum(m).
__device__ __forceinline__ float vget(const Vol &g, const float *a, const float *Mk, int x, int y, int z, int b,
                                      int dx, int dy, int dz) {
  const long long v = nbr(g, x, y, z, b, dx, dy, dz);
  return v >= 0 ? a[v] * Mk[v] : 0.0f;
}
__global__ void k_res_fwd(Vol g, const float *Yo, const float *A7, const float *X4, const float *Mk, float c,
                          float *R, float *lpart) {
  __shared__ float red[256];
  const long long v = (long long)blockIdx.x * 256 + threadIdx.x;
  float l = 0.0f;
  if (v < g.n()) {
    int x, y, z, b;
    decomp(g, v, x, y, z, b);
    const float *a = A7 + 7 * v;
    const float ay = a[0] * Yo[v] * Mk[v] + a[1] * vget(g, Yo, Mk, x, y, z, b, -1, 0, 0) +
                     a[2] * vget(g, Yo, Mk, x, y, z, b, 0, -1, 0) + a[3] * vget(g, Yo, Mk, x, y, z, b, 0, 0, -1) +
                     a[4] * vget(g, Yo, Mk, x, y, z, b, 1, 0, 0) + a[5] * vget(g, Yo, Mk, x, y, z, b, 0, 1, 0) +
                     a[6] * vget(g, Yo, Mk, x, y, z, b, 0, 0, 1);
    const float r = Mk[v] * (X4[4 * v] - c * ay);
    R[v] = r;
    l = r * r;
  }
  red[threadIdx.x] = l;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) lpart[blockIdx.x] = red[0];
}
// dy += w * d(|r|^2 / n)/dy = -2 w c / n * m[v] (A^T r)[v]; (A^T r)[v] =
// AD[v] r[v] + the coefficients of the neighbours' rows that point at v
__global__ void k_res_bwd(Vol g, const float *A7, const float *R, const float *Mk, float scale, float *dy) {
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= g.n()) return;
  int x, y, z, b;
  decomp(g, v, x, y, z, b);
  auto term = [&](int dx, int dyy, int dz, int k) {
    const long long u = nbr(g, x, y, z, b, dx, dyy, dz);
    return u >= 0 ? A7[7 * u + k] * R[u] : 0.0f;
  };
  // row u = v+1 holds ALI (index 1) toward v, row v-1 holds AUI (4) ...
  const float atr = A7[7 * v] * R[v] + term(1, 0, 0, 1) + term(0, 1, 0, 2) + term(0, 0, 1, 3) + term(-1, 0, 0, 4) +
                    term(0, -1, 0, 5) + term(0, 0, -1, 6);
  dy[v] += scale * Mk[v] * atr;
}

// -------------------------------------------------------- Adam, casts
// FP32 master p, moments m, v; step t (1-based); then the BF16 copy
__global__ void k_adam(long long n, float *p, const float *g, float *m, float *v, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}
// weights [cout][27][cin] FP32 -> BF16 forward copy and the input-gradient
// copy Wt[cin][26 - tap][cout]
__global__ void k_wcast(const float *w, int Cin, int Cout, bf16 *wf, bf16 *wt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= Cout * 27 * Cin) return;
  const int ci = i % Cin, t = (i / Cin) % 27, co = i / (27 * Cin);
  const bf16 q = __float2bfloat16(w[i]);
  wf[i] = q;
  if (wt) wt[((long long)ci * 27 + (26 - t)) * Cout + co] = q;
}
// network input: 4 FP32 channels per voxel -> 16 BF16 channels (12 zero)
__global__ void k_pack_in(long long V, const float *x4, bf16 *x16) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V * 16) return;
  const long long v = i >> 4;
  const int c = (int)(i & 15);
  x16[i] = __float2bfloat16(c < 4 ? x4[v * 4 + c] : 0.0f);
}
__global__ void k_f32_to_bf16(long long n, const float *a, bf16 *b) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = __float2bfloat16(a[i]);
}
__global__ void k_fill_bf16(long long n, bf16 *a) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = __float2bfloat16(0.0f);
}

// ------------------------------------------------------------ launchers
static inline unsigned nb(long long n, int t) { return (unsigned)((n + t - 1) / t); }

// At least 56 KB of dynamic shared memory per CTA, so that at most four
// CTAs share an SM and their TMEM (at most 128 columns each) fits in the
// SM's 512 columns without an allocation having to wait.
static size_t smem_floor(size_t b) { return b < 56 * 1024 ? 56 * 1024 : b; }
size_t conv_smem_bytes(int Cin, int Cout) {
  return smem_floor((size_t)2 * CONV_M * Cin * 2 + (size_t)2 * Cout * Cin * 2 + 32);
}
size_t wgrad_smem_bytes(int Cout) { return smem_floor((size_t)2 * 128 * WG_K * 2 + (size_t)2 * Cout * WG_K * 2 + 32); }

bool unet_kernels_configure() {
  static int done = 0;
  if (done) return done > 0;
  const int mx = 200 * 1024;
  bool ok = cudaFuncSetAttribute(k_conv, cudaFuncAttributeMaxDynamicSharedMemorySize, mx) == cudaSuccess &&
            cudaFuncSetAttribute(k_wgrad, cudaFuncAttributeMaxDynamicSharedMemorySize, mx) == cudaSuccess;
  done = ok ? 1 : -1;
  return ok;
}

void launch_conv(cudaStream_t s, int X, int Y, int Z, int B, const void *x, int Cin, const void *w, const float *bias,
                 int Cout, int mode, const void *mask, void *y, int *err) {
  const Vol g{X, Y, Z, B};
  k_conv<<<nb(g.n(), CONV_M), 128, conv_smem_bytes(Cin, Cout), s>>>(
      g, (const bf16 *)x, Cin, (const bf16 *)w, bias, Cout, mode, (const bf16 *)mask, y, err);
  count_launch();
}
void launch_wgrad(cudaStream_t s, int X, int Y, int Z, int B, const void *x, int Cin, const void *dy, int Cout,
                  long long slice, float *part, float *dw, int *err) {
  const Vol g{X, Y, Z, B};
  const int ns = (int)((g.n() + slice - 1) / slice);
  dim3 grid((27 * Cin + 127) / 128, ns);
  k_wgrad<<<grid, 128, wgrad_smem_bytes(Cout), s>>>(g, (const bf16 *)x, Cin, (const bf16 *)dy, Cout, slice, part,
                                                      err);
  k_wgrad_reduce<<<nb(27LL * Cin * Cout, 256), 256, 0, s>>>(part, ns, Cin, Cout, dw);
  count_launch(2);
}
void launch_bias_grad(cudaStream_t s, long long V, const void *dy, int C, float *part, float *db) {
  const int n = (int)nb(V, 1024);
  k_bias_part<<<n, 128, 0, s>>>((const bf16 *)dy, V, C, part);
  k_bias_reduce<<<1, 128, 0, s>>>(part, n, C, db);
  count_launch(2);
}
void launch_pool(cudaStream_t s, int Xc, int Yc, int Zc, int B, const void *f, int C, void *c) {
  const Vol gc{Xc, Yc, Zc, B};
  k_pool<<<nb(gc.n() * C, 256), 256, 0, s>>>(gc, (const bf16 *)f, C, (bf16 *)c);
  count_launch();
}
void launch_pool_bwd(cudaStream_t s, int Xc, int Yc, int Zc, int B, const void *dc, int C, void *df, int acc) {
  const Vol gc{Xc, Yc, Zc, B};
  k_pool_bwd<<<nb(gc.n() * 8 * C, 256), 256, 0, s>>>(gc, (const bf16 *)dc, C, (bf16 *)df, acc);
  count_launch();
}
void launch_upcat(cudaStream_t s, int X, int Y, int Z, int B, const void *c, int C1, const void *sk, int C2, void *o) {
  const Vol gf{X, Y, Z, B};
  k_upcat<<<nb(gf.n() * (C1 + C2), 256), 256, 0, s>>>(gf, (const bf16 *)c, C1, (const bf16 *)sk, C2, (bf16 *)o);
  count_launch();
}
void launch_upcat_bwd(cudaStream_t s, int X, int Y, int Z, int B, const void *d, int C1, int C2, void *dc, void *dsk,
                      int acc) {
  const Vol gf{X, Y, Z, B};
  const Vol gc{X / 2, Y / 2, Z / 2, B};
  k_upcat_bwd_coarse<<<nb(gc.n() * C1, 256), 256, 0, s>>>(gc, (const bf16 *)d, C1, C2, (bf16 *)dc);
  k_upcat_bwd_skip<<<nb(gf.n() * C2, 256), 256, 0, s>>>(gf.n(), (const bf16 *)d, C1, C2, (bf16 *)dsk, acc);
  count_launch(2);
}
void launch_relu_mask(cudaStream_t s, long long n, const void *act, void *d) {
  k_relu_mask<<<nb(n, 256), 256, 0, s>>>(n, (const bf16 *)act, (bf16 *)d);
  count_launch();
}
void launch_head(cudaStream_t s, long long V, const void *a, int C, const float *wh, const float *bh, float *y) {
  k_head<<<nb(V, 256), 256, 0, s>>>(V, (const bf16 *)a, C, wh, bh, y);
  count_launch();
}
void launch_mse(cudaStream_t s, long long V, const float *y, const float *t, const float *m, float inv_n, float *dy,
                float *lpart) {
  k_mse<<<nb(V, 256), 256, 0, s>>>(V, y, t, m, inv_n, dy, lpart);
  count_launch();
}
void launch_head_bwd(cudaStream_t s, long long V, const float *dy, const void *a, int C, const float *wh, void *da,
                     float *part) {
  k_head_bwd_act<<<nb(V * C, 256), 256, 0, s>>>(V, dy, (const bf16 *)a, C, wh, (bf16 *)da);
  k_head_bwd_par<<<nb(V, 1024), 32, 0, s>>>(V, dy, (const bf16 *)a, C, part);
  count_launch(2);
}
void launch_res_fwd(cudaStream_t s, int X, int Y, int Z, int B, const float *y, const float *a7, const float *x4,
                    const float *m, float c, float *r, float *lpart) {
  const Vol g{X, Y, Z, B};
  k_res_fwd<<<nb(g.n(), 256), 256, 0, s>>>(g, y, a7, x4, m, c, r, lpart);
  count_launch();
}
void launch_res_bwd(cudaStream_t s, int X, int Y, int Z, int B, const float *a7, const float *r, const float *m,
                    float scale, float *dy) {
  const Vol g{X, Y, Z, B};
  k_res_bwd<<<nb(g.n(), 256), 256, 0, s>>>(g, a7, r, m, scale, dy);
  count_launch();
}
void launch_adam(cudaStream_t s, long long n, float *p, const float *g, float *m, float *v, float lr, float b1,
                 float b2, float eps, float c1, float c2) {
  k_adam<<<nb(n, 256), 256, 0, s>>>(n, p, g, m, v, lr, b1, b2, eps, c1, c2);
  count_launch();
}
void launch_wcast(cudaStream_t s, const float *w, int Cin, int Cout, void *wf, void *wt) {
  k_wcast<<<nb(27LL * Cin * Cout, 256), 256, 0, s>>>(w, Cin, Cout, (bf16 *)wf, (bf16 *)wt);
  count_launch();
}
void launch_pack_in(cudaStream_t s, long long V, const float *x4, void *x16) {
  k_pack_in<<<nb(V * 16, 256), 256, 0, s>>>(V, x4, (bf16 *)x16);
  count_launch();
}
void launch_bias_reduce(cudaStream_t s, const float *part, int n, int C, float *out) {
  k_bias_reduce<<<1, 128, 0, s>>>(part, n, C, out);
  count_launch();
}
void launch_f32_to_bf16(cudaStream_t s, long long n, const float *a, void *b) {
  k_f32_to_bf16<<<nb(n, 256), 256, 0, s>>>(n, a, (bf16 *)b);
  count_launch();
}
void launch_fill_bf16(cudaStream_t s, long long n, void *a) {
  k_fill_bf16<<<nb(n, 256), 256, 0, s>>>(n, (bf16 *)a);
  count_launch();
}

}  // namespace cadmas
