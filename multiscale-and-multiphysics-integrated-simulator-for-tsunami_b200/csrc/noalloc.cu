// noalloc.cu -- the allocation-free divergence norm (cadmas_divnorm_noalloc).
//
// cadmas_divnorm computes |VD| of VF_CDIV00 (vf_cdiv00.f:38-56) on the
// state of a handle, keeping its row partials in memory the handle
// allocated.  This entry point runs the same two kernels (row partials of
// VD^2, then the 1024-thread tree over the rows) on arrays the caller
// already holds on the device, without a handle and without allocating:
// its scratch is the file-scope device array below.
//
// Who needs it: callers that cannot allocate device memory at the moment
// they want the norm.  A run that has committed the whole device to its
// own arrays (large grids, many flumes) would fail a handle's roughly 60
// arrays or even one temporary buffer with cudaErrorMemoryAllocation.  A
// host time loop that checks the divergence between its own launches
// cannot afford the cudaMalloc/cudaFree pair either: cudaFree waits for
// the whole device, stalling the work it has queued on other streams.
// And a coupling layer that only holds raw device pointers has no handle
// to borrow scratch from.
//
// Contract:
//   - at most CADMAS_NOALLOC_MAX_ROWS rows (NUMJ*NUMK); larger grids get
//     CADMAS_ESCRATCH and nothing runs;
//   - nothing in the scratch has to start at zero: every row partial is
//     written before the final kernel reads it, and the result slot is
//     written before it is copied out;
//   - calls that overlap in time on one device race on the scratch (one
//     array per device, shared by all streams and threads): issue them
//     one after another;
//   - the first call on a device looks up the scratch's device address
//     (cudaGetSymbolAddress, which may load the module); make that first
//     call before anything that must not see such set-up work, e.g.
//     before stream capture begins;
//   - `stream` must belong to the current device (the scratch address is
//     the current device's); a stream of another device gets
//     CADMAS_EINVAL and nothing runs;
//   - a CUDA failure returns CADMAS_ECUDA with the failing call and its
//     message in cadmas_strerror; an error that earlier work left pending
//     is not blamed on this call: it is reported before any launch.
#include <cuda_runtime.h>
#include <atomic>
#include <cmath>
#include <mutex>

#include "cadmas_dev.cuh"
#include "kernels.h"
#include "../../include/cadmas_gpu.h"

using namespace cadmas;

namespace {
// Row partials [0, rows) followed by the two result slots of k_fin.
constexpr long long kScratchDoubles = CADMAS_NOALLOC_MAX_ROWS + 32;
__device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::atomic<double *> g_scratch_ptr[kMaxDevices];
std::mutex g_setup_mutex;

// Device address of the scratch on the current device (looked up once).
int scratch_for(int dev, double **out) {
  if (dev < 0 || dev >= kMaxDevices) return CADMAS_EINVAL;
  double *p = g_scratch_ptr[dev].load(std::memory_order_acquire);
  if (!p) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    p = g_scratch_ptr[dev].load(std::memory_order_acquire);
    if (!p) {
      void *addr = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
      if (e != cudaSuccess || !addr) {
        set_cuda_error("cudaGetSymbolAddress(g_noalloc_scratch)", e != cudaSuccess ? e : cudaErrorInvalidSymbol);
        return CADMAS_ECUDA;
      }
      p = static_cast<double *>(addr);
      g_scratch_ptr[dev].store(p, std::memory_order_release);
    }
  }
  *out = p;
  return CADMAS_OK;
}
}  // namespace

extern "C" int cadmas_divnorm_noalloc(const cadmas_dims *d, const double *xx, const double *yy,
                                      const double *zz, const double *ggx, const double *ggy,
                                      const double *ggz, const double *uu, const double *vv,
                                      const double *ww, const int *indc, void *stream, double *val) {
  if (!d || !xx || !yy || !zz || !ggx || !ggy || !ggz || !uu || !vv || !ww || !indc || !val)
    return CADMAS_EINVAL;
  if (d->numi < 3 || d->numj < 3 || d->numk < 3) return CADMAS_EINVAL;
  const long long rows = (long long)d->numj * d->numk;
  if (rows > CADMAS_NOALLOC_MAX_ROWS) return CADMAS_ESCRATCH;
#define NA_CK(call)                        \
  do {                                     \
    const cudaError_t e_ = (call);         \
    if (e_ != cudaSuccess) {               \
      set_cuda_error(#call, e_);           \
      return CADMAS_ECUDA;                 \
    }                                      \
  } while (0)
  // an error left pending by the caller's earlier work is theirs: report
  // it as such before this call launches anything
  {
    const cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess) {
      set_cuda_error("error pending before cadmas_divnorm_noalloc", pending);
      return CADMAS_ECUDA;
    }
  }
  int dev = -1;
  NA_CK(cudaGetDevice(&dev));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (s != nullptr) {  // the legacy/default stream follows the current device
    int sdev = -1;
    NA_CK(cudaStreamGetDevice(s, &sdev));
    if (sdev != dev) return CADMAS_EINVAL;
  }
  double *scratch = nullptr;
  int rc = scratch_for(dev, &scratch);
  if (rc) return rc;

  Geo g{};
  g.NI = d->numi; g.NJ = d->numj; g.NK = d->numk; g.NB = 0;
  g.N = (long long)d->numi * d->numj * d->numk;
  g.XX = xx; g.YY = yy; g.ZZ = zz;
  Fld f{};
  f.ggx = ggx; f.ggy = ggy; f.ggz = ggz;
  f.uu = const_cast<double *>(uu); f.vv = const_cast<double *>(vv); f.ww = const_cast<double *>(ww);
  f.indc = const_cast<int *>(indc);

  double *res = scratch + CADMAS_NOALLOC_MAX_ROWS;  // k_fin writes res[0], res[1]
  launch_cdiv(s, g, f, scratch);
  launch_fin(s, FIN_STORE, scratch, scratch, rows, nullptr, res, 0, 0, 0, 0);
  NA_CK(cudaGetLastError());
  double h = 0.0;
  NA_CK(cudaMemcpyAsync(&h, res, sizeof(double), cudaMemcpyDeviceToHost, s));
  NA_CK(cudaStreamSynchronize(s));
  *val = std::sqrt(h);
  return CADMAS_OK;
#undef NA_CK
}
