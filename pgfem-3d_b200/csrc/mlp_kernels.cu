// mlp_kernels.cu -- host side of the warm-start network (C ABI pgfem_mlp_*).
//
// The model owns its device buffers: FP32 master parameters, Adam moments,
// the gradient accumulator, the packed BF16 weights / FP32 biases that the
// tcgen05 kernels stage into shared memory, and the feature/target scaling.
// Training runs entirely on the GPU with this file's kernels: per step one
// k_mlp_train launch (one CTA per 128-sample tile, fused forward + backward,
// gradients reduced with FP32 atomics) and one k_mlp_adam launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "mlp_kernels.cuh"
#include "pgfem_gpu.h"

using namespace pgb::mlp;

struct pgfem_mlp {
  int dev = 0;
  float *params = nullptr, *grad = nullptr, *mom = nullptr, *vel = nullptr;
  __nv_bfloat16 *w = nullptr;
  float *bias = nullptr, *scale = nullptr;
  unsigned *err = nullptr;
  double *loss = nullptr;
  float h_scale[kScale];
  long adam_t = 0;
  uint64_t wait_ns = pgb::mlp::kWaitNs;
  int stall = 0;  // the next forward pass withholds its first MMA chain (failure-path tests)
  pgb::mlp::MlpDev dev_view() const { return {w, bias, scale, err, wait_ns, 0}; }
};

namespace {

#define MCK(x)                                                                          \
  do {                                                                                  \
    cudaError_t _e = (x);                                                               \
    if (_e != cudaSuccess) {                                                            \
      std::fprintf(stderr, "pgfem_mlp: %s failed: %s (%s:%d)\n", #x, cudaGetErrorString(_e), \
                   __FILE__, __LINE__);                                                 \
      return PGFEM_GPU_ECUDA;                                                           \
    }                                                                                   \
  } while (0)

uint64_t splitmix64(uint64_t &s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
double uniform01(uint64_t &s) { return (double)(splitmix64(s) >> 11) * (1.0 / 9007199254740992.0); }

int check_dev() {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return PGFEM_GPU_ENODEV;
  }
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, dev) != cudaSuccess || p.major != 10) return PGFEM_GPU_ENODEV;
  return PGFEM_GPU_OK;
}

int set_smem_attrs() {
  static bool done = false;
  if (done) return PGFEM_GPU_OK;
  MCK(cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kInfSmem));
  MCK(cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrainSmem));
  done = true;
  return PGFEM_GPU_OK;
}

int num_sms() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

int pack(pgfem_mlp *m) {
  k_mlp_adam<<<(kNParam + 255) / 256, 256>>>(m->params, m->grad, m->mom, m->vel, m->w, m->bias, 0.f, 0.f, 0.f,
                                             0.f, 0.f, 0.f, 0);
  MCK(cudaGetLastError());
  return PGFEM_GPU_OK;
}

int read_err(pgfem_mlp *m) {
  unsigned e = 0;
  MCK(cudaMemcpy(&e, m->err, sizeof(e), cudaMemcpyDeviceToHost));
  if (e) {
    MCK(cudaMemset(m->err, 0, sizeof(unsigned)));
    std::fprintf(stderr, "pgfem_mlp: a tensor-core completion wait ran out\n");
    return PGFEM_GPU_ETIMEOUT;
  }
  return PGFEM_GPU_OK;
}

// launches the tiles of one gradient evaluation over rows perm[first .. first+count)
int launch_grad(pgfem_mlp *m, long count, long first, const int *perm, const float *x, const float *t,
                float inv_batch, cudaStream_t s) {
  const long tiles = (count + kTile - 1) / kTile;
  if (tiles > 0x7fffffffL) return PGFEM_GPU_ELIMIT;
  k_mlp_train<<<(unsigned)tiles, kThreads, kTrainSmem, s>>>(m->dev_view(), count, first, perm, x, t, inv_batch,
                                                            m->grad, m->loss);
  MCK(cudaGetLastError());
  return PGFEM_GPU_OK;
}

}  // namespace

extern "C" {

long pgfem_mlp_num_params(void) { return kNParam; }

int pgfem_mlp_create(unsigned long long seed, pgfem_mlp **out) {
  if (!out) return PGFEM_GPU_EINVAL;
  *out = nullptr;
  int r = check_dev();
  if (r) return r;
  if ((r = set_smem_attrs())) return r;
  pgfem_mlp *m = new pgfem_mlp();
  cudaGetDevice(&m->dev);
  auto fail = [&](int code) {
    pgfem_mlp_destroy(m);
    return code;
  };
  if (cudaMalloc(&m->params, sizeof(float) * kNParam) || cudaMalloc(&m->grad, sizeof(float) * kNParam) ||
      cudaMalloc(&m->mom, sizeof(float) * kNParam) || cudaMalloc(&m->vel, sizeof(float) * kNParam) ||
      cudaMalloc(&m->w, sizeof(__nv_bfloat16) * kNPW) || cudaMalloc(&m->bias, sizeof(float) * kNPB) ||
      cudaMalloc(&m->scale, sizeof(float) * kScale) || cudaMalloc(&m->err, sizeof(unsigned)) ||
      cudaMalloc(&m->loss, sizeof(double))) {
    cudaGetLastError();
    return fail(PGFEM_GPU_ENOMEM);
  }
  if (cudaMemset(m->grad, 0, sizeof(float) * kNParam) || cudaMemset(m->mom, 0, sizeof(float) * kNParam) ||
      cudaMemset(m->vel, 0, sizeof(float) * kNParam) || cudaMemset(m->w, 0, sizeof(__nv_bfloat16) * kNPW) ||
      cudaMemset(m->bias, 0, sizeof(float) * kNPB) || cudaMemset(m->err, 0, sizeof(unsigned)) ||
      cudaMemset(m->loss, 0, sizeof(double)))
    return fail(PGFEM_GPU_ECUDA);
  // Glorot-uniform weights, zero biases, from a splitmix64 stream
  std::vector<float> p(kNParam, 0.0f);
  uint64_t st = seed;
  auto fill = [&](int off, int rows, int cols) {
    const double lim = std::sqrt(6.0 / (rows + cols));
    for (int i = 0; i < rows * cols; i++) p[off + i] = (float)((2.0 * uniform01(st) - 1.0) * lim);
  };
  fill(oW1, kH, kIn);
  fill(oW2, kH, kH);
  fill(oW3, kH, kH);
  fill(oW4, kOut, kH);
  for (int j = 0; j < kScale; j++) m->h_scale[j] = (j >= kIn && j < 2 * kIn) || j >= 2 * kIn ? 1.0f : 0.0f;
  if (cudaMemcpy(m->scale, m->h_scale, sizeof(m->h_scale), cudaMemcpyHostToDevice)) return fail(PGFEM_GPU_ECUDA);
  if ((r = pgfem_mlp_set_params(m, p.data()))) return fail(r);
  *out = m;
  return PGFEM_GPU_OK;
}

int pgfem_mlp_destroy(pgfem_mlp *m) {
  if (!m) return PGFEM_GPU_OK;
  cudaFree(m->params);
  cudaFree(m->grad);
  cudaFree(m->mom);
  cudaFree(m->vel);
  cudaFree(m->w);
  cudaFree(m->bias);
  cudaFree(m->scale);
  cudaFree(m->err);
  cudaFree(m->loss);
  delete m;
  return PGFEM_GPU_OK;
}

int pgfem_mlp_set_params(pgfem_mlp *m, const float *p) {
  if (!m || !p) return PGFEM_GPU_EINVAL;
  MCK(cudaMemcpy(m->params, p, sizeof(float) * kNParam, cudaMemcpyHostToDevice));
  MCK(cudaMemset(m->mom, 0, sizeof(float) * kNParam));
  MCK(cudaMemset(m->vel, 0, sizeof(float) * kNParam));
  m->adam_t = 0;
  int r = pack(m);
  if (r) return r;
  MCK(cudaDeviceSynchronize());
  return PGFEM_GPU_OK;
}

int pgfem_mlp_get_params(const pgfem_mlp *m, float *p) {
  if (!m || !p) return PGFEM_GPU_EINVAL;
  MCK(cudaMemcpy(p, m->params, sizeof(float) * kNParam, cudaMemcpyDeviceToHost));
  return PGFEM_GPU_OK;
}

int pgfem_mlp_set_scaling(pgfem_mlp *m, const float *x_mean, const float *x_std, const float *y_std) {
  if (!m || !x_mean || !x_std || !y_std) return PGFEM_GPU_EINVAL;
  for (int j = 0; j < kIn; j++) {
    if (!(x_std[j] > 0.0f)) return PGFEM_GPU_EINVAL;
    m->h_scale[j] = x_mean[j];
    m->h_scale[kIn + j] = 1.0f / x_std[j];
  }
  for (int j = 0; j < kOut; j++) {
    if (!(y_std[j] > 0.0f)) return PGFEM_GPU_EINVAL;
    m->h_scale[2 * kIn + j] = y_std[j];
  }
  MCK(cudaMemcpy(m->scale, m->h_scale, sizeof(m->h_scale), cudaMemcpyHostToDevice));
  return PGFEM_GPU_OK;
}

int pgfem_mlp_get_scaling(const pgfem_mlp *m, float *x_mean, float *x_inv_std, float *y_std) {
  if (!m) return PGFEM_GPU_EINVAL;
  for (int j = 0; j < kIn; j++) {
    if (x_mean) x_mean[j] = m->h_scale[j];
    if (x_inv_std) x_inv_std[j] = m->h_scale[kIn + j];
  }
  for (int j = 0; j < kOut; j++)
    if (y_std) y_std[j] = m->h_scale[2 * kIn + j];
  return PGFEM_GPU_OK;
}

int pgfem_mlp_fit_scaling(pgfem_mlp *m, long n, const float *d_x, const float *d_t) {
  if (!m || n < 2 || !d_x || !d_t) return PGFEM_GPU_EINVAL;
  double *acc = nullptr;
  if (cudaMalloc(&acc, sizeof(double) * 2 * (kIn + kOut))) {
    cudaGetLastError();
    return PGFEM_GPU_ENOMEM;
  }
  std::vector<double> h(2 * (kIn + kOut));
  int r = PGFEM_GPU_OK;
  if (cudaMemset(acc, 0, sizeof(double) * 2 * (kIn + kOut))) r = PGFEM_GPU_ECUDA;
  if (!r) {
    const unsigned grid = (unsigned)std::min<long>((n + 255) / 256, 4L * num_sms());
    k_col_stats<kIn><<<grid, 256>>>(d_x, n, acc);
    k_col_stats<kOut><<<grid, 256>>>(d_t, n, acc + 2 * kIn);
    if (cudaGetLastError() || cudaMemcpy(h.data(), acc, sizeof(double) * h.size(), cudaMemcpyDeviceToHost))
      r = PGFEM_GPU_ECUDA;
  }
  cudaFree(acc);
  if (r) return r;
  float xm[kIn], xs[kIn], ys[kOut];
  for (int j = 0; j < kIn; j++) {
    const double mu = h[j] / n, var = std::max(0.0, h[kIn + j] / n - mu * mu);
    xm[j] = (float)mu;
    xs[j] = (float)std::max(std::sqrt(var), 1e-6 * std::max(1.0, std::fabs(mu)));
  }
  for (int j = 0; j < kOut; j++) {
    // targets keep their sign and zero: scale only, by the root mean square
    const double rms = std::sqrt(h[2 * kIn + kOut + j] / n);
    ys[j] = (float)std::max(rms, 1e-30);
  }
  return pgfem_mlp_set_scaling(m, xm, xs, ys);
}

int pgfem_mlp_set_wait_test(pgfem_mlp *m, double limit_s, int stall_next_forward) {
  if (!m || !(limit_s > 0.0) || limit_s > 60.0) return PGFEM_GPU_EINVAL;
  m->wait_ns = (uint64_t)(limit_s * 1e9);
  m->stall = stall_next_forward ? 1 : 0;
  return PGFEM_GPU_OK;
}

int pgfem_mlp_predict_device(pgfem_mlp *m, long n, const float *d_x, float *d_y, void *stream) {
  if (!m || n < 0 || (n && (!d_x || !d_y))) return PGFEM_GPU_EINVAL;
  if (n == 0) return PGFEM_GPU_OK;
  int r = set_smem_attrs();
  if (r) return r;
  const long tiles = (n + kTile - 1) / kTile;
  const unsigned grid = (unsigned)std::min<long>(tiles, num_sms());
  pgb::mlp::MlpDev dv = m->dev_view();
  dv.stall = m->stall;
  m->stall = 0;
  k_mlp_forward<<<grid, kThreads, kInfSmem, (cudaStream_t)stream>>>(dv, n, d_x, d_y);
  MCK(cudaGetLastError());
  return PGFEM_GPU_OK;
}

int pgfem_mlp_predict(pgfem_mlp *m, long n, const float *x, float *y) {
  if (!m || n < 0 || (n && (!x || !y))) return PGFEM_GPU_EINVAL;
  if (n == 0) return PGFEM_GPU_OK;
  float *dx = nullptr, *dy = nullptr;
  if (cudaMalloc(&dx, sizeof(float) * n * kIn) || cudaMalloc(&dy, sizeof(float) * n * kOut)) {
    cudaGetLastError();
    cudaFree(dx);
    return PGFEM_GPU_ENOMEM;
  }
  int r = PGFEM_GPU_OK;
  if (cudaMemcpy(dx, x, sizeof(float) * n * kIn, cudaMemcpyHostToDevice)) r = PGFEM_GPU_ECUDA;
  if (!r) r = pgfem_mlp_predict_device(m, n, dx, dy, nullptr);
  if (!r && cudaMemcpy(y, dy, sizeof(float) * n * kOut, cudaMemcpyDeviceToHost)) r = PGFEM_GPU_ECUDA;
  cudaFree(dx);
  cudaFree(dy);
  if (!r) r = read_err(m);
  return r;
}

int pgfem_mlp_loss_grad(pgfem_mlp *m, long n, const float *x, const float *t, float *grad, double *loss) {
  if (!m || n < 1 || !x || !t || !grad) return PGFEM_GPU_EINVAL;
  float *dx = nullptr, *dt = nullptr;
  if (cudaMalloc(&dx, sizeof(float) * n * kIn) || cudaMalloc(&dt, sizeof(float) * n * kOut)) {
    cudaGetLastError();
    cudaFree(dx);
    return PGFEM_GPU_ENOMEM;
  }
  int r = PGFEM_GPU_OK;
  if (cudaMemcpy(dx, x, sizeof(float) * n * kIn, cudaMemcpyHostToDevice) ||
      cudaMemcpy(dt, t, sizeof(float) * n * kOut, cudaMemcpyHostToDevice) ||
      cudaMemset(m->grad, 0, sizeof(float) * kNParam) || cudaMemset(m->loss, 0, sizeof(double)))
    r = PGFEM_GPU_ECUDA;
  if (!r) r = set_smem_attrs();
  if (!r) r = launch_grad(m, n, 0, nullptr, dx, dt, 1.0f / (float)n, nullptr);
  if (!r && (cudaMemcpy(grad, m->grad, sizeof(float) * kNParam, cudaMemcpyDeviceToHost) ||
             (loss && cudaMemcpy(loss, m->loss, sizeof(double), cudaMemcpyDeviceToHost))))
    r = PGFEM_GPU_ECUDA;
  cudaMemset(m->grad, 0, sizeof(float) * kNParam);
  cudaFree(dx);
  cudaFree(dt);
  if (!r) r = read_err(m);
  return r;
}

int pgfem_mlp_train_device(pgfem_mlp *m, long n, const float *d_x, const float *d_t,
                           const pgfem_mlp_train_opts *o, double *epoch_loss) {
  if (!m || n < 1 || !d_x || !d_t || !o || o->epochs < 0 || o->batch < kTile) return PGFEM_GPU_EINVAL;
  if (n > 0x7fffffffL) return PGFEM_GPU_ELIMIT;
  int r = set_smem_attrs();
  if (r) return r;
  int *perm = nullptr;
  double *losses = nullptr;
  if (cudaMalloc(&perm, sizeof(int) * n) || cudaMalloc(&losses, sizeof(double) * std::max(1, o->epochs))) {
    cudaGetLastError();
    cudaFree(perm);
    return PGFEM_GPU_ENOMEM;
  }
  std::vector<int> h(n);
  uint64_t st = o->seed;
  const long nb = n / o->batch;  // full batches per epoch (the remainder rotates with the shuffle)
  const long total = (long)o->epochs * std::max<long>(nb, 1);
  long step = 0;
  cudaMemset(m->grad, 0, sizeof(float) * kNParam);
  for (int ep = 0; ep < o->epochs && !r; ep++) {
    for (long i = 0; i < n; i++) h[i] = (int)i;
    for (long i = n - 1; i > 0; i--) std::swap(h[i], h[(long)(uniform01(st) * (double)(i + 1)) % (i + 1)]);
    if (cudaMemcpy(perm, h.data(), sizeof(int) * n, cudaMemcpyHostToDevice) ||
        cudaMemset(m->loss, 0, sizeof(double))) {
      r = PGFEM_GPU_ECUDA;
      break;
    }
    const long nbe = std::max<long>(nb, 1);
    for (long b = 0; b < nbe && !r; b++, step++) {
      const long cnt = nb ? o->batch : n;
      r = launch_grad(m, cnt, b * (nb ? o->batch : 0), perm, d_x, d_t, 1.0f / (float)cnt, nullptr);
      if (r) break;
      // cosine decay from lr to lr_min over all steps
      const double frac = total > 1 ? (double)step / (double)(total - 1) : 0.0;
      const float lr = (float)(o->lr_min + 0.5 * (o->lr - o->lr_min) * (1.0 + std::cos(M_PI * frac)));
      m->adam_t++;
      const float c1 = (float)(1.0 / (1.0 - std::pow((double)o->beta1, (double)m->adam_t)));
      const float c2 = (float)(1.0 / (1.0 - std::pow((double)o->beta2, (double)m->adam_t)));
      k_mlp_adam<<<(kNParam + 255) / 256, 256>>>(m->params, m->grad, m->mom, m->vel, m->w, m->bias, lr, o->beta1,
                                                 o->beta2, o->eps, c1, c2, 1);
      if (cudaGetLastError()) r = PGFEM_GPU_ECUDA;
    }
    // mean batch loss of the epoch
    if (!r && cudaMemcpyAsync(losses + ep, m->loss, sizeof(double), cudaMemcpyDeviceToDevice))
      r = PGFEM_GPU_ECUDA;
  }
  if (!r && cudaDeviceSynchronize()) r = PGFEM_GPU_ECUDA;
  if (!r && epoch_loss && o->epochs > 0) {
    std::vector<double> hl(o->epochs);
    if (cudaMemcpy(hl.data(), losses, sizeof(double) * o->epochs, cudaMemcpyDeviceToHost)) r = PGFEM_GPU_ECUDA;
    for (int ep = 0; ep < o->epochs && !r; ep++) epoch_loss[ep] = hl[ep] / (double)std::max<long>(nb, 1);
  }
  cudaFree(perm);
  cudaFree(losses);
  if (!r) r = read_err(m);
  return r;
}

}  // extern "C"
