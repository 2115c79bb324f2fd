// unet.cu -- the learned warm start's network on the host side: the layer
// table of the 3-level 3-D U-Net, its buffers, forward, backward (input and
// weight gradients of every layer), the masked MSE loss and Adam, behind the
// cadmas_unet_* entry points.
//
// Architecture (channels-last BF16 activations, FP32 master weights):
//   in 4 (+12 zero) -> c11 16 -> c12 16 (skip1) -> pool -> c21 32 ->
//   c22 32 (skip2) -> pool -> c31 64 -> c32 64 -> up + skip2 (96) ->
//   c41 32 -> c42 32 -> up + skip1 (48) -> c51 16 -> c52 16 -> head 1
// every cNN a 3x3x3 convolution with bias and ReLU, pooling 2x2x2 average,
// upsampling nearest, the head a 1x1x1 convolution with bias (FP32 out).
// Parameters (FP32, in this order): per convolution W[cout][27][cin] then
// b[cout]; then the head's 16 weights and its bias.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#include "../../include/cadmas_gpu.h"
#include "kernels.h"

using namespace cadmas;

namespace {

struct Layer {
  int cin, cout, res;
  size_t w, b;  // offsets of W and b in the parameter vector
};

constexpr int NL = 10;
const int LCH[NL][3] = {{16, 16, 0}, {16, 16, 0}, {16, 32, 1}, {32, 32, 1}, {32, 64, 2},
                        {64, 64, 2}, {96, 32, 1}, {32, 32, 1}, {48, 16, 0}, {16, 16, 0}};

struct Table {
  Layer L[NL];
  size_t head_w, head_b, n;
  Table() {
    size_t o = 0;
    for (int l = 0; l < NL; ++l) {
      L[l] = Layer{LCH[l][0], LCH[l][1], LCH[l][2], o, o + (size_t)27 * LCH[l][0] * LCH[l][1]};
      o = L[l].b + LCH[l][1];
    }
    head_w = o;
    head_b = o + 16;
    n = o + 17;
  }
};
const Table TAB;

template <class T>
int dmalloc(T **p, size_t n) {
  return cudaMalloc((void **)p, (n ? n : 1) * sizeof(T)) == cudaSuccess ? CADMAS_OK : CADMAS_ENOMEM;
}

}  // namespace

struct cadmas_unet {
  cudaStream_t s = nullptr;
  bool own_stream = true;
  int X = 0, Y = 0, Z = 0, B = 0;
  long long V[3] = {0, 0, 0};
  float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
  long long step = 0;
  void *wf[NL] = {}, *wt[NL] = {};
  // activations (BF16) and their gradients
  void *xin = nullptr, *a[NL] = {}, *p1 = nullptr, *p2 = nullptr, *u2 = nullptr, *u1 = nullptr;
  void *d[NL] = {}, *du2 = nullptr, *du1 = nullptr, *dp1 = nullptr, *dp2 = nullptr;
  float *x4 = nullptr, *y = nullptr, *t = nullptr, *mk = nullptr, *dy = nullptr;
  float *part = nullptr, *bpart = nullptr, *lpart = nullptr;
  float *a7 = nullptr, *r = nullptr;  // pressure systems and residual (residual loss)
  size_t part_n = 0;
  long long slice = 8192;
  int *err = nullptr;
  std::vector<float> hl;
};

namespace {

void dims(const cadmas_unet *n, int res, int &X, int &Y, int &Z) {
  X = n->X >> res;
  Y = n->Y >> res;
  Z = n->Z >> res;
}

void conv(cadmas_unet *n, int res, const void *x, int cin, const void *w, const float *b, int cout, int mode,
          const void *mask, void *y) {
  int X, Y, Z;
  dims(n, res, X, Y, Z);
  launch_conv(n->s, X, Y, Z, n->B, x, cin, w, b, cout, mode, mask, y, n->err);
}

void cast_weights(cadmas_unet *n) {
  for (int l = 0; l < NL; ++l)
    launch_wcast(n->s, n->p + TAB.L[l].w, TAB.L[l].cin, TAB.L[l].cout, n->wf[l], l > 0 ? n->wt[l] : nullptr);
}

int check(cadmas_unet *n) {
  int e = 0;
  if (cudaMemcpyAsync(&e, n->err, sizeof(int), cudaMemcpyDeviceToHost, n->s) != cudaSuccess) return CADMAS_ECUDA;
  if (cudaStreamSynchronize(n->s) != cudaSuccess) return CADMAS_ECUDA;
  if (cudaGetLastError() != cudaSuccess) return CADMAS_ECUDA;
  return e ? CADMAS_ETIMEOUT : CADMAS_OK;
}

// forward of the batch in n->x4 (FP32, 4 channels) to n->y
void forward(cadmas_unet *n) {
  const auto &L = TAB.L;
  launch_pack_in(n->s, n->V[0], n->x4, n->xin);
  conv(n, 0, n->xin, 16, n->wf[0], n->p + L[0].b, 16, CONV_RELU_BF16, nullptr, n->a[0]);
  conv(n, 0, n->a[0], 16, n->wf[1], n->p + L[1].b, 16, CONV_RELU_BF16, nullptr, n->a[1]);
  launch_pool(n->s, n->X / 2, n->Y / 2, n->Z / 2, n->B, n->a[1], 16, n->p1);
  conv(n, 1, n->p1, 16, n->wf[2], n->p + L[2].b, 32, CONV_RELU_BF16, nullptr, n->a[2]);
  conv(n, 1, n->a[2], 32, n->wf[3], n->p + L[3].b, 32, CONV_RELU_BF16, nullptr, n->a[3]);
  launch_pool(n->s, n->X / 4, n->Y / 4, n->Z / 4, n->B, n->a[3], 32, n->p2);
  conv(n, 2, n->p2, 32, n->wf[4], n->p + L[4].b, 64, CONV_RELU_BF16, nullptr, n->a[4]);
  conv(n, 2, n->a[4], 64, n->wf[5], n->p + L[5].b, 64, CONV_RELU_BF16, nullptr, n->a[5]);
  launch_upcat(n->s, n->X / 2, n->Y / 2, n->Z / 2, n->B, n->a[5], 64, n->a[3], 32, n->u2);
  conv(n, 1, n->u2, 96, n->wf[6], n->p + L[6].b, 32, CONV_RELU_BF16, nullptr, n->a[6]);
  conv(n, 1, n->a[6], 32, n->wf[7], n->p + L[7].b, 32, CONV_RELU_BF16, nullptr, n->a[7]);
  launch_upcat(n->s, n->X, n->Y, n->Z, n->B, n->a[7], 32, n->a[1], 16, n->u1);
  conv(n, 0, n->u1, 48, n->wf[8], n->p + L[8].b, 16, CONV_RELU_BF16, nullptr, n->a[8]);
  conv(n, 0, n->a[8], 16, n->wf[9], n->p + L[9].b, 16, CONV_RELU_BF16, nullptr, n->a[9]);
  launch_head(n->s, n->V[0], n->a[9], 16, n->p + TAB.head_w, n->p + TAB.head_b, n->y);
}

// weight and bias gradients of layer l from its input x and output grad dyl
void layer_grads(cadmas_unet *n, int l, const void *x, const void *dyl) {
  const Layer &L = TAB.L[l];
  int X, Y, Z;
  dims(n, L.res, X, Y, Z);
  launch_wgrad(n->s, X, Y, Z, n->B, x, L.cin, dyl, L.cout, n->slice, n->part, n->g + L.w, n->err);
  launch_bias_grad(n->s, n->V[L.res], dyl, L.cout, n->bpart, n->g + L.b);
}

// backward from n->dy (FP32 loss gradient of the output) into n->g
void backward(cadmas_unet *n) {
  const int nbh = (int)((n->V[0] + 1023) / 1024);
  launch_head_bwd(n->s, n->V[0], n->dy, n->a[9], 16, n->p + TAB.head_w, n->d[9], n->bpart);
  launch_bias_reduce(n->s, n->bpart, nbh, 17, n->g + TAB.head_w);
  // c52, c51
  layer_grads(n, 9, n->a[8], n->d[9]);
  conv(n, 0, n->d[9], 16, n->wt[9], nullptr, 16, CONV_MASK_BF16, n->a[8], n->d[8]);
  layer_grads(n, 8, n->u1, n->d[8]);
  conv(n, 0, n->d[8], 16, n->wt[8], nullptr, 48, CONV_MASK_BF16, n->u1, n->du1);
  // split: d of c42's output (coarse, 32) and of skip1 (16)
  launch_upcat_bwd(n->s, n->X, n->Y, n->Z, n->B, n->du1, 32, 16, n->d[7], n->d[1], 0);
  // c42, c41
  layer_grads(n, 7, n->a[6], n->d[7]);
  conv(n, 1, n->d[7], 32, n->wt[7], nullptr, 32, CONV_MASK_BF16, n->a[6], n->d[6]);
  layer_grads(n, 6, n->u2, n->d[6]);
  conv(n, 1, n->d[6], 32, n->wt[6], nullptr, 96, CONV_MASK_BF16, n->u2, n->du2);
  launch_upcat_bwd(n->s, n->X / 2, n->Y / 2, n->Z / 2, n->B, n->du2, 64, 32, n->d[5], n->d[3], 0);
  // c32, c31
  layer_grads(n, 5, n->a[4], n->d[5]);
  conv(n, 2, n->d[5], 64, n->wt[5], nullptr, 64, CONV_MASK_BF16, n->a[4], n->d[4]);
  layer_grads(n, 4, n->p2, n->d[4]);
  conv(n, 2, n->d[4], 64, n->wt[4], nullptr, 32, CONV_BF16, nullptr, n->dp2);
  // skip2 gets the pooled path too, then the ReLU of c22
  launch_pool_bwd(n->s, n->X / 4, n->Y / 4, n->Z / 4, n->B, n->dp2, 32, n->d[3], 1);
  launch_relu_mask(n->s, n->V[1] * 32, n->a[3], n->d[3]);
  // c22, c21
  layer_grads(n, 3, n->a[2], n->d[3]);
  conv(n, 1, n->d[3], 32, n->wt[3], nullptr, 32, CONV_MASK_BF16, n->a[2], n->d[2]);
  layer_grads(n, 2, n->p1, n->d[2]);
  conv(n, 1, n->d[2], 32, n->wt[2], nullptr, 16, CONV_BF16, nullptr, n->dp1);
  launch_pool_bwd(n->s, n->X / 2, n->Y / 2, n->Z / 2, n->B, n->dp1, 16, n->d[1], 1);
  launch_relu_mask(n->s, n->V[0] * 16, n->a[1], n->d[1]);
  // c12, c11
  layer_grads(n, 1, n->a[0], n->d[1]);
  conv(n, 0, n->d[1], 16, n->wt[1], nullptr, 16, CONV_MASK_BF16, n->a[0], n->d[0]);
  layer_grads(n, 0, n->xin, n->d[0]);
}

// loss of n->y against t on mask m (host arrays already on the device)
int loss_and_dy(cadmas_unet *n, float *loss) {
  const long long V = n->V[0];
  std::vector<float> mh((size_t)V);
  if (cudaMemcpyAsync(mh.data(), n->mk, V * sizeof(float), cudaMemcpyDeviceToHost, n->s) != cudaSuccess)
    return CADMAS_ECUDA;
  if (cudaStreamSynchronize(n->s) != cudaSuccess) return CADMAS_ECUDA;
  double cnt = 0.0;
  for (float q : mh) cnt += q;
  const float inv = cnt > 0.0 ? (float)(1.0 / cnt) : 0.0f;
  launch_mse(n->s, V, n->y, n->t, n->mk, inv, n->dy, n->lpart);
  const int nbk = (int)((V + 255) / 256);
  n->hl.resize((size_t)nbk);
  if (cudaMemcpyAsync(n->hl.data(), n->lpart, nbk * sizeof(float), cudaMemcpyDeviceToHost, n->s) != cudaSuccess)
    return CADMAS_ECUDA;
  if (cudaStreamSynchronize(n->s) != cudaSuccess) return CADMAS_ECUDA;
  double l = 0.0;
  for (float q : n->hl) l += q;
  *loss = (float)(l * inv);
  return CADMAS_OK;
}

int upload(cadmas_unet *n, const float *x, const float *t, const float *m) {
  const long long V = n->V[0];
  if (cudaMemcpyAsync(n->x4, x, V * 4 * sizeof(float), cudaMemcpyHostToDevice, n->s) != cudaSuccess)
    return CADMAS_ECUDA;
  if (t && cudaMemcpyAsync(n->t, t, V * sizeof(float), cudaMemcpyHostToDevice, n->s) != cudaSuccess)
    return CADMAS_ECUDA;
  if (m && cudaMemcpyAsync(n->mk, m, V * sizeof(float), cudaMemcpyHostToDevice, n->s) != cudaSuccess)
    return CADMAS_ECUDA;
  return CADMAS_OK;
}

}  // namespace

extern "C" {

size_t cadmas_unet_param_count(void) { return TAB.n; }

int cadmas_unet_destroy(cadmas_unet *n) {
  if (!n) return CADMAS_OK;
  for (float *q : {n->p, n->g, n->m, n->v, n->x4, n->y, n->t, n->mk, n->dy, n->part, n->bpart, n->lpart, n->a7, n->r})
    if (q) cudaFree(q);
  for (int l = 0; l < NL; ++l)
    for (void *q : {n->wf[l], n->wt[l], n->a[l], n->d[l]})
      if (q) cudaFree(q);
  for (void *q : {n->xin, n->p1, n->p2, n->u2, n->u1, n->du2, n->du1, n->dp1, n->dp2})
    if (q) cudaFree(q);
  if (n->err) cudaFree(n->err);
  if (n->s && n->own_stream) cudaStreamDestroy(n->s);
  delete n;
  return CADMAS_OK;
}

int cadmas_unet_create(int nx, int ny, int nz, int batch, cadmas_unet **out) {
  return cadmas::unet_new(nx, ny, nz, batch, nullptr, out);
}

}  // extern "C"

namespace cadmas {

// A network on the given stream (its own stream when null).
int unet_new(int nx, int ny, int nz, int batch, cudaStream_t stream, cadmas_unet **out) {
  if (!out || nx < 4 || ny < 4 || nz < 4 || batch < 1 || nx % 4 || ny % 4 || nz % 4) return CADMAS_EINVAL;
  if (!unet_kernels_configure()) return CADMAS_ECUDA;
  cadmas_unet *n = new cadmas_unet();
  n->X = nx; n->Y = ny; n->Z = nz; n->B = batch;
  for (int r = 0; r < 3; ++r) n->V[r] = (long long)(nx >> r) * (ny >> r) * (nz >> r) * batch;
  int rc = CADMAS_OK;
  if (stream) {
    n->s = stream;
    n->own_stream = false;
  } else if (cudaStreamCreateWithFlags(&n->s, cudaStreamNonBlocking) != cudaSuccess) {
    rc = CADMAS_ECUDA;
  }
  const size_t P = TAB.n;
#define AL(ptr, cnt) if (!rc) rc = dmalloc(&(ptr), (cnt))
  AL(n->p, P); AL(n->g, P); AL(n->m, P); AL(n->v, P);
  using u16 = unsigned short;
  for (int l = 0; l < NL; ++l) {
    const size_t w = (size_t)27 * TAB.L[l].cin * TAB.L[l].cout;
    AL(*(u16 **)&n->wf[l], w);
    if (l > 0) AL(*(u16 **)&n->wt[l], w);
    AL(*(u16 **)&n->a[l], (size_t)n->V[TAB.L[l].res] * TAB.L[l].cout);
    AL(*(u16 **)&n->d[l], (size_t)n->V[TAB.L[l].res] * TAB.L[l].cout);
  }
  AL(*(u16 **)&n->xin, (size_t)n->V[0] * 16);
  AL(*(u16 **)&n->p1, (size_t)n->V[1] * 16); AL(*(u16 **)&n->dp1, (size_t)n->V[1] * 16);
  AL(*(u16 **)&n->p2, (size_t)n->V[2] * 32); AL(*(u16 **)&n->dp2, (size_t)n->V[2] * 32);
  AL(*(u16 **)&n->u2, (size_t)n->V[1] * 96); AL(*(u16 **)&n->du2, (size_t)n->V[1] * 96);
  AL(*(u16 **)&n->u1, (size_t)n->V[0] * 48); AL(*(u16 **)&n->du1, (size_t)n->V[0] * 48);
  AL(n->x4, (size_t)n->V[0] * 4); AL(n->y, (size_t)n->V[0]); AL(n->t, (size_t)n->V[0]);
  AL(n->mk, (size_t)n->V[0]); AL(n->dy, (size_t)n->V[0]);
  // wgrad partial sums: the largest (slices x 27 Cin x Cout) of any layer
  for (int l = 0; l < NL; ++l) {
    const long long ns = (n->V[TAB.L[l].res] + n->slice - 1) / n->slice;
    n->part_n = std::max(n->part_n, (size_t)ns * 27 * TAB.L[l].cin * TAB.L[l].cout);
  }
  AL(n->part, n->part_n);
  AL(n->bpart, (size_t)((n->V[0] + 1023) / 1024) * 128);
  AL(n->lpart, (size_t)((n->V[0] + 255) / 256));
  if (!rc && cudaMalloc((void **)&n->err, sizeof(int)) != cudaSuccess) rc = CADMAS_ENOMEM;
#undef AL
  if (rc) { cadmas_unet_destroy(n); return rc; }
  cudaMemsetAsync(n->err, 0, sizeof(int), n->s);
  cudaMemsetAsync(n->p, 0, P * sizeof(float), n->s);
  cudaMemsetAsync(n->m, 0, P * sizeof(float), n->s);
  cudaMemsetAsync(n->v, 0, P * sizeof(float), n->s);
  cast_weights(n);
  if (cudaStreamSynchronize(n->s) != cudaSuccess) { cadmas_unet_destroy(n); return CADMAS_ECUDA; }
  *out = n;
  return CADMAS_OK;
}

void unet_dims(const cadmas_unet *n, int &X, int &Y, int &Z) { X = n->X; Y = n->Y; Z = n->Z; }
float *unet_input(cadmas_unet *n) { return n->x4; }
const float *unet_output(const cadmas_unet *n) { return n->y; }
const int *unet_error(const cadmas_unet *n) { return n->err; }
void unet_run_forward(cadmas_unet *n) { forward(n); }
int unet_error_host(cadmas_unet *n) { return check(n); }

}  // namespace cadmas

extern "C" {

int cadmas_unet_set_params(cadmas_unet *n, const float *p) {
  if (!n || !p) return CADMAS_EINVAL;
  if (cudaMemcpyAsync(n->p, p, TAB.n * sizeof(float), cudaMemcpyHostToDevice, n->s) != cudaSuccess)
    return CADMAS_ECUDA;
  cudaMemsetAsync(n->m, 0, TAB.n * sizeof(float), n->s);
  cudaMemsetAsync(n->v, 0, TAB.n * sizeof(float), n->s);
  n->step = 0;
  cast_weights(n);
  return check(n);
}

int cadmas_unet_get_params(cadmas_unet *n, float *p) {
  if (!n || !p) return CADMAS_EINVAL;
  if (cudaMemcpyAsync(p, n->p, TAB.n * sizeof(float), cudaMemcpyDeviceToHost, n->s) != cudaSuccess)
    return CADMAS_ECUDA;
  return check(n);
}

int cadmas_unet_forward(cadmas_unet *n, const float *x, float *y) {
  if (!n || !x || !y) return CADMAS_EINVAL;
  int rc = upload(n, x, nullptr, nullptr);
  if (rc) return rc;
  forward(n);
  if (cudaMemcpyAsync(y, n->y, n->V[0] * sizeof(float), cudaMemcpyDeviceToHost, n->s) != cudaSuccess)
    return CADMAS_ECUDA;
  return check(n);
}

int cadmas_unet_time_forward(cadmas_unet *n, int reps, float *ms) {
  if (!n || reps < 1 || !ms) return CADMAS_EINVAL;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return CADMAS_ECUDA;
  cudaEventRecord(e0, n->s);
  for (int r = 0; r < reps; ++r) forward(n);
  cudaEventRecord(e1, n->s);
  int rc = check(n);
  float t = 0.0f;
  if (!rc && cudaEventElapsedTime(&t, e0, e1) != cudaSuccess) rc = CADMAS_ECUDA;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = t / reps;
  return rc;
}

int cadmas_unet_grad(cadmas_unet *n, const float *x, const float *t, const float *m, float *loss, float *grad) {
  if (!n || !x || !t || !m || !loss) return CADMAS_EINVAL;
  int rc = upload(n, x, t, m);
  if (rc) return rc;
  forward(n);
  rc = loss_and_dy(n, loss);
  if (rc) return rc;
  backward(n);
  if (grad && cudaMemcpyAsync(grad, n->g, TAB.n * sizeof(float), cudaMemcpyDeviceToHost, n->s) != cudaSuccess)
    return CADMAS_ECUDA;
  return check(n);
}

// Sum of the per-block loss partials of the last loss kernel, in order.
static int lsum(cadmas_unet *n, double &out) {
  const int nbk = (int)((n->V[0] + 255) / 256);
  n->hl.resize((size_t)nbk);
  if (cudaMemcpyAsync(n->hl.data(), n->lpart, nbk * sizeof(float), cudaMemcpyDeviceToHost, n->s) != cudaSuccess)
    return CADMAS_ECUDA;
  if (cudaStreamSynchronize(n->s) != cudaSuccess) return CADMAS_ECUDA;
  out = 0.0;
  for (float q : n->hl) out += q;
  return CADMAS_OK;
}

int cadmas_unet_train_sys(cadmas_unet *n, const float *x, const float *t, const float *m, const float *a7, float c,
                          float w_mse, float w_res, float lr, int update, float *loss, float *grad) {
  if (!n || !x || !t || !m || !a7 || !loss || !(c > 0.0f)) return CADMAS_EINVAL;
  const long long V = n->V[0];
  if (!n->a7 && (dmalloc(&n->a7, (size_t)V * 7) || dmalloc(&n->r, (size_t)V))) return CADMAS_ENOMEM;
  int rc = upload(n, x, t, m);
  if (rc) return rc;
  if (cudaMemcpyAsync(n->a7, a7, V * 7 * sizeof(float), cudaMemcpyHostToDevice, n->s) != cudaSuccess)
    return CADMAS_ECUDA;
  forward(n);
  // counted cells
  std::vector<float> mh((size_t)V);
  if (cudaMemcpyAsync(mh.data(), n->mk, V * sizeof(float), cudaMemcpyDeviceToHost, n->s) != cudaSuccess)
    return CADMAS_ECUDA;
  if (cudaStreamSynchronize(n->s) != cudaSuccess) return CADMAS_ECUDA;
  double cnt = 0.0;
  for (float q : mh) cnt += q;
  const double inv = cnt > 0.0 ? 1.0 / cnt : 0.0;
  // mean-square error of y against t, weighted by w_mse in the gradient
  launch_mse(n->s, V, n->y, n->t, n->mk, (float)(inv * w_mse), n->dy, n->lpart);
  double lm, lr2;
  if ((rc = lsum(n, lm))) return rc;
  // residual |m (b - c A y)|^2 / n, weighted by w_res
  launch_res_fwd(n->s, n->X, n->Y, n->Z, n->B, n->y, n->a7, n->x4, n->mk, c, n->r, n->lpart);
  if ((rc = lsum(n, lr2))) return rc;
  launch_res_bwd(n->s, n->X, n->Y, n->Z, n->B, n->a7, n->r, n->mk, (float)(-2.0 * c * w_res * inv), n->dy);
  *loss = (float)(w_mse * lm * inv + w_res * lr2 * inv);
  backward(n);
  if (grad && cudaMemcpyAsync(grad, n->g, TAB.n * sizeof(float), cudaMemcpyDeviceToHost, n->s) != cudaSuccess)
    return CADMAS_ECUDA;
  if (update) {
    n->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - std::pow(b1, (float)n->step), c2 = 1.0f - std::pow(b2, (float)n->step);
    launch_adam(n->s, (long long)TAB.n, n->p, n->g, n->m, n->v, lr, b1, b2, 1.0e-8f, c1, c2);
    cast_weights(n);
  }
  return check(n);
}

int cadmas_unet_train_step(cadmas_unet *n, const float *x, const float *t, const float *m, float lr, float *loss) {
  int rc = cadmas_unet_grad(n, x, t, m, loss, nullptr);
  if (rc) return rc;
  n->step += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f - std::pow(b1, (float)n->step), c2 = 1.0f - std::pow(b2, (float)n->step);
  launch_adam(n->s, (long long)TAB.n, n->p, n->g, n->m, n->v, lr, b1, b2, 1.0e-8f, c1, c2);
  cast_weights(n);
  return check(n);
}

}  // extern "C"
