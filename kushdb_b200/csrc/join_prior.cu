// Kernels of the learned join-order prior (join_prior.h): fused forward over
// all layers, fused backward with deterministic per-CTA gradient partials,
// and a reduce + Adam update.  The MLP is tiny (41,473 fp32 parameters), so
// the kernels run on CUDA cores: each CTA of 128 threads owns a tile of 16
// rows, thread j computes hidden unit j for every row of the tile, and the
// activations of the tile stay in shared memory between layers.
#include "join_prior.h"

#include <algorithm>
#include <cmath>
#include <cstring>

#include "capi_internal.h"

namespace kdb {
namespace {

constexpr int kIn = JoinPrior::kIn;
constexpr int kHid = JoinPrior::kHid;
constexpr int kRows = 16;      // rows per CTA
constexpr int kThreads = kHid;  // one thread per hidden unit
constexpr int64_t kParams = JoinPrior::kParams;

// out[r][j] = relu(b[j] + sum_k in[r][k] * W[k][j]) for the tile; saved to
// global for the backward pass.
template <int K>
__device__ __forceinline__ void Dense(const float* __restrict__ W, const float* __restrict__ b, const float* in,
                                      float* out, float* __restrict__ save, int64_t row0, int64_t n) {
  const int j = threadIdx.x;
  float acc[kRows];
  const float bj = b[j];
#pragma unroll
  for (int r = 0; r < kRows; r++) acc[r] = bj;
  for (int k = 0; k < K; k++) {
    const float w = W[k * kHid + j];
#pragma unroll
    for (int r = 0; r < kRows; r++) acc[r] = fmaf(in[r * K + k], w, acc[r]);
  }
#pragma unroll
  for (int r = 0; r < kRows; r++) {
    const float v = fmaxf(acc[r], 0.f);
    out[r * kHid + j] = v;
    if (row0 + r < n) save[(row0 + r) * kHid + j] = v;
  }
}

__device__ __forceinline__ float WarpSum(float s) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

template <int K>
__device__ __forceinline__ void LoadTile(float* dst, const float* __restrict__ src, int64_t row0, int64_t n) {
  for (int i = threadIdx.x; i < kRows * K; i += kThreads) {
    const int r = i / K;
    dst[i] = row0 + r < n ? src[(row0 + r) * K + i % K] : 0.f;
  }
}

__global__ void __launch_bounds__(kThreads) PriorForward(const float* __restrict__ P, const float* __restrict__ X,
                                                         int64_t n, float* __restrict__ Y, float* __restrict__ H) {
  __shared__ float xs[kRows * kIn];
  __shared__ float ha[kRows * kHid];
  __shared__ float hb[kRows * kHid];
  __shared__ float red[kThreads / 32][kRows];
  const int64_t row0 = static_cast<int64_t>(blockIdx.x) * kRows;
  float* H1 = H;
  float* H2 = H + static_cast<int64_t>(JoinPrior::kMaxRows) * kHid;
  float* H3 = H + 2 * static_cast<int64_t>(JoinPrior::kMaxRows) * kHid;
  LoadTile<kIn>(xs, X, row0, n);
  __syncthreads();
  Dense<kIn>(P + JoinPrior::kOffW1, P + JoinPrior::kOffB1, xs, ha, H1, row0, n);
  __syncthreads();
  Dense<kHid>(P + JoinPrior::kOffW2, P + JoinPrior::kOffB2, ha, hb, H2, row0, n);
  __syncthreads();
  Dense<kHid>(P + JoinPrior::kOffW3, P + JoinPrior::kOffB3, hb, ha, H3, row0, n);
  __syncthreads();
  const int j = threadIdx.x;
  const float w = P[JoinPrior::kOffW4 + j];
#pragma unroll
  for (int r = 0; r < kRows; r++) {
    const float s = WarpSum(ha[r * kHid + j] * w);
    if ((j & 31) == 0) red[j >> 5][r] = s;
  }
  __syncthreads();
  if (j < kRows && row0 + j < n)
    Y[row0 + j] = ((red[0][j] + red[1][j]) + (red[2][j] + red[3][j])) + P[JoinPrior::kOffB4];
}

// outW[k][j] = sum_r in[r][k] * dz[r][j], outB[j] = sum_r dz[r][j]
template <int K>
__device__ __forceinline__ void WeightGrad(const float* in, const float* dz, float* __restrict__ outW,
                                           float* __restrict__ outB) {
  const int j = threadIdx.x;
  float d[kRows];
  float sb = 0.f;
#pragma unroll
  for (int r = 0; r < kRows; r++) {
    d[r] = dz[r * kHid + j];
    sb += d[r];
  }
  outB[j] = sb;
  for (int k = 0; k < K; k++) {
    float s = 0.f;
#pragma unroll
    for (int r = 0; r < kRows; r++) s = fmaf(in[r * K + k], d[r], s);
    outW[k * kHid + j] = s;
  }
}

// dst[r][k] = (act[r][k] > 0) * sum_j dz[r][j] * W[k][j]  (W is kHid x kHid)
__device__ __forceinline__ void InputGrad(const float* __restrict__ W, const float* dz, const float* act,
                                          float* dst) {
  const int k = threadIdx.x;
  float s[kRows];
#pragma unroll
  for (int r = 0; r < kRows; r++) s[r] = 0.f;
  const float4* row = reinterpret_cast<const float4*>(W + k * kHid);
  for (int j4 = 0; j4 < kHid / 4; j4++) {
    const float4 w = row[j4];
#pragma unroll
    for (int r = 0; r < kRows; r++) {
      const float* z = dz + r * kHid + 4 * j4;
      s[r] = fmaf(z[0], w.x, s[r]);
      s[r] = fmaf(z[1], w.y, s[r]);
      s[r] = fmaf(z[2], w.z, s[r]);
      s[r] = fmaf(z[3], w.w, s[r]);
    }
  }
#pragma unroll
  for (int r = 0; r < kRows; r++) dst[r * kHid + k] = act[r * kHid + k] > 0.f ? s[r] : 0.f;
}

// Gradient of mean((y - t)^2) for this CTA's rows into partial[blockIdx.x].
__global__ void __launch_bounds__(kThreads) PriorBackward(const float* __restrict__ P, const float* __restrict__ X,
                                                          const float* __restrict__ H, const float* __restrict__ Y,
                                                          const float* __restrict__ T, int64_t n,
                                                          float* __restrict__ partial) {
  __shared__ float dy[kRows];
  __shared__ float ga[kRows * kHid];
  __shared__ float gb[kRows * kHid];
  __shared__ float hs[kRows * kHid];
  __shared__ float xs[kRows * kIn];
  const int64_t row0 = static_cast<int64_t>(blockIdx.x) * kRows;
  const float* H1 = H;
  const float* H2 = H + static_cast<int64_t>(JoinPrior::kMaxRows) * kHid;
  const float* H3 = H + 2 * static_cast<int64_t>(JoinPrior::kMaxRows) * kHid;
  float* out = partial + static_cast<int64_t>(blockIdx.x) * kParams;
  const int j = threadIdx.x;
  if (j < kRows) dy[j] = row0 + j < n ? 2.f * (Y[row0 + j] - T[row0 + j]) / static_cast<float>(n) : 0.f;
  LoadTile<kHid>(hs, H3, row0, n);
  __syncthreads();
  // head: y = w4 . h3 + b4
  {
    float g = 0.f, sb = 0.f;
#pragma unroll
    for (int r = 0; r < kRows; r++) {
      g = fmaf(dy[r], hs[r * kHid + j], g);
      sb += dy[r];
    }
    out[JoinPrior::kOffW4 + j] = g;
    if (j == 0) out[JoinPrior::kOffB4] = sb;
    const float w4 = P[JoinPrior::kOffW4 + j];
#pragma unroll
    for (int r = 0; r < kRows; r++) ga[r * kHid + j] = hs[r * kHid + j] > 0.f ? dy[r] * w4 : 0.f;
  }
  __syncthreads();
  // layer 3 (input H2, pre-activation delta ga)
  LoadTile<kHid>(hs, H2, row0, n);
  __syncthreads();
  WeightGrad<kHid>(hs, ga, out + JoinPrior::kOffW3, out + JoinPrior::kOffB3);
  InputGrad(P + JoinPrior::kOffW3, ga, hs, gb);
  __syncthreads();
  // layer 2 (input H1, delta gb)
  LoadTile<kHid>(hs, H1, row0, n);
  __syncthreads();
  WeightGrad<kHid>(hs, gb, out + JoinPrior::kOffW2, out + JoinPrior::kOffB2);
  InputGrad(P + JoinPrior::kOffW2, gb, hs, ga);
  __syncthreads();
  // layer 1 (input X, delta ga)
  LoadTile<kIn>(xs, X, row0, n);
  __syncthreads();
  WeightGrad<kIn>(xs, ga, out + JoinPrior::kOffW1, out + JoinPrior::kOffB1);
}

// grad = sum of the CTA partials (fixed order); optional Adam step
// (Kingma & Ba, beta1 0.9, beta2 0.999, eps 1e-8).
__global__ void PriorAdam(float* __restrict__ P, const float* __restrict__ partial, int nblk, float* __restrict__ m,
                          float* __restrict__ v, float* __restrict__ grad, float lr, float c1, float c2) {
  for (int64_t p = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; p < kParams;
       p += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    float g = 0.f;
    for (int b = 0; b < nblk; b++) g += partial[b * kParams + p];
    grad[p] = g;
    if (lr > 0.f) {
      const float mp = 0.9f * m[p] + 0.1f * g;
      const float vp = 0.999f * v[p] + 0.001f * g * g;
      m[p] = mp;
      v[p] = vp;
      P[p] -= lr * (mp / c1) / (sqrtf(vp / c2) + 1e-8f);
    }
  }
}

uint64_t SplitMix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

}  // namespace

JoinPrior::JoinPrior(int device, uint32_t seed) : device_(device) {
  KDB_CUDA(cudaSetDevice(device));
  KDB_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  const int64_t nblk = kMaxRows / kRows;
  KDB_CUDA(cudaMalloc(&p_, sizeof(float) * kParams));
  KDB_CUDA(cudaMalloc(&m_, sizeof(float) * kParams));
  KDB_CUDA(cudaMalloc(&v_, sizeof(float) * kParams));
  KDB_CUDA(cudaMalloc(&grad_, sizeof(float) * kParams));
  KDB_CUDA(cudaMalloc(&x_, sizeof(float) * kMaxRows * kIn));
  KDB_CUDA(cudaMalloc(&t_, sizeof(float) * kMaxRows));
  KDB_CUDA(cudaMalloc(&y_, sizeof(float) * kMaxRows));
  KDB_CUDA(cudaMalloc(&h_, sizeof(float) * 3 * kMaxRows * kHid));
  KDB_CUDA(cudaMalloc(&partial_, sizeof(float) * nblk * kParams));
  KDB_CUDA(cudaMallocHost(&pinned_, sizeof(float) * (kMaxRows * (kIn + 2) + kParams)));
  // He-uniform initialisation (bound sqrt(6 / fan_in)), zero biases
  std::vector<float> init(kParams, 0.f);
  uint64_t s = 0x6A09E667F3BCC909ULL ^ seed;
  auto fill = [&](int64_t off, int64_t count, int fan_in) {
    const double a = std::sqrt(6.0 / fan_in);
    for (int64_t i = 0; i < count; i++)
      init[off + i] = static_cast<float>((static_cast<double>(SplitMix(s) >> 11) * 0x1.0p-53 * 2.0 - 1.0) * a);
  };
  fill(kOffW1, kIn * kHid, kIn);
  fill(kOffW2, kHid * kHid, kHid);
  fill(kOffW3, kHid * kHid, kHid);
  fill(kOffW4, kHid, kHid);
  SetParams(init.data());
}

JoinPrior::~JoinPrior() {
  cudaSetDevice(device_);
  cudaStreamSynchronize(stream_);
  for (float* p : {p_, m_, v_, grad_, x_, t_, y_, h_, partial_}) cudaFree(p);
  cudaFreeHost(pinned_);
  cudaStreamDestroy(stream_);
}

void JoinPrior::SetParams(const float* p) {
  std::lock_guard<std::mutex> lock(mu_);
  KDB_CUDA(cudaSetDevice(device_));
  std::memcpy(pinned_, p, sizeof(float) * kParams);
  KDB_CUDA(cudaMemcpyAsync(p_, pinned_, sizeof(float) * kParams, cudaMemcpyHostToDevice, stream_));
  KDB_CUDA(cudaMemsetAsync(m_, 0, sizeof(float) * kParams, stream_));
  KDB_CUDA(cudaMemsetAsync(v_, 0, sizeof(float) * kParams, stream_));
  KDB_CUDA(cudaStreamSynchronize(stream_));
  step_ = 0;
}

void JoinPrior::GetParams(float* p) {
  std::lock_guard<std::mutex> lock(mu_);
  KDB_CUDA(cudaSetDevice(device_));
  KDB_CUDA(cudaMemcpyAsync(pinned_, p_, sizeof(float) * kParams, cudaMemcpyDeviceToHost, stream_));
  KDB_CUDA(cudaStreamSynchronize(stream_));
  std::memcpy(p, pinned_, sizeof(float) * kParams);
}

double JoinPrior::Run(const float* x, const float* t, int64_t n, float* grad, float lr, float* y) {
  if (n <= 0 || n > kMaxRows) throw Error(KDB_ERR_INVALID, "join prior batch must hold 1.." +
                                                              std::to_string(kMaxRows) + " rows");
  std::lock_guard<std::mutex> lock(mu_);
  KDB_CUDA(cudaSetDevice(device_));
  const int nblk = static_cast<int>((n + kRows - 1) / kRows);
  float* px = pinned_;
  float* pt = pinned_ + kMaxRows * kIn;
  float* py = pt + kMaxRows;
  std::memcpy(px, x, sizeof(float) * n * kIn);
  KDB_CUDA(cudaMemcpyAsync(x_, px, sizeof(float) * n * kIn, cudaMemcpyHostToDevice, stream_));
  if (t) {
    std::memcpy(pt, t, sizeof(float) * n);
    KDB_CUDA(cudaMemcpyAsync(t_, pt, sizeof(float) * n, cudaMemcpyHostToDevice, stream_));
  }
  PriorForward<<<nblk, kThreads, 0, stream_>>>(p_, x_, n, y_, h_);
  KDB_CUDA(cudaGetLastError());
  if (t) {
    PriorBackward<<<nblk, kThreads, 0, stream_>>>(p_, x_, h_, y_, t_, n, partial_);
    KDB_CUDA(cudaGetLastError());
    float c1 = 1.f, c2 = 1.f;
    if (lr > 0.f) {
      step_++;
      c1 = static_cast<float>(1.0 - std::pow(0.9, static_cast<double>(step_)));
      c2 = static_cast<float>(1.0 - std::pow(0.999, static_cast<double>(step_)));
    }
    PriorAdam<<<static_cast<int>((kParams + 255) / 256), 256, 0, stream_>>>(p_, partial_, nblk, m_, v_, grad_, lr,
                                                                              c1, c2);
    KDB_CUDA(cudaGetLastError());
    if (grad) KDB_CUDA(cudaMemcpyAsync(pinned_ + kMaxRows * (kIn + 2), grad_, sizeof(float) * kParams,
                                       cudaMemcpyDeviceToHost, stream_));
  }
  KDB_CUDA(cudaMemcpyAsync(py, y_, sizeof(float) * n, cudaMemcpyDeviceToHost, stream_));
  KDB_CUDA(cudaStreamSynchronize(stream_));
  if (grad) std::memcpy(grad, pinned_ + kMaxRows * (kIn + 2), sizeof(float) * kParams);
  double loss = 0;
  if (t)
    for (int64_t i = 0; i < n; i++) {
      const double d = static_cast<double>(py[i]) - t[i];
      loss += d * d;
    }
  if (y) std::memcpy(y, py, sizeof(float) * n);
  return t ? loss / static_cast<double>(n) : 0.0;
}

void JoinPrior::Forward(const float* x, int64_t n, float* y) {
  Run(x, nullptr, n, nullptr, 0.f, y);
}

double JoinPrior::Gradient(const float* x, const float* t, int64_t n, float* grad) {
  return Run(x, t, n, grad, 0.f, nullptr);
}

double JoinPrior::TrainStep(const float* x, const float* t, int64_t n, float lr) {
  if (!(lr > 0.f)) throw Error(KDB_ERR_INVALID, "learning rate must be positive");
  return Run(x, t, n, nullptr, lr, nullptr);
}

}  // namespace kdb

struct kdb_mlp {
  std::unique_ptr<kdb::JoinPrior> p;
  std::string err;
};

namespace {

template <typename F>
int MGuard(kdb_mlp* m, F&& f) {
  if (!m) return KDB_ERR_INVALID;
  try {
    f();
    return KDB_OK;
  } catch (const kdb::Error& e) {
    m->err = e.what();
    return e.code;
  } catch (const std::exception& e) {
    m->err = e.what();
    return KDB_ERR_CUDA;
  }
}

}  // namespace

extern "C" {

int32_t kdb_mlp_num_features(void) { return kdb::JoinPrior::kIn; }
int64_t kdb_mlp_num_params(void) { return kdb::JoinPrior::kParams; }

int kdb_mlp_create(kdb_ctx* ctx, uint32_t seed, kdb_mlp** out) {
  if (!ctx || !out) return KDB_ERR_INVALID;
  *out = nullptr;
  try {
    kdb::Context& c = *kdb_ctx_context(ctx);
    if (c.dry) throw kdb::Error(KDB_ERR_UNSUPPORTED, "the join prior needs a GPU context");
    auto m = std::make_unique<kdb_mlp>();
    m->p = std::make_unique<kdb::JoinPrior>(c.device, seed);
    *out = m.release();
    return KDB_OK;
  } catch (const kdb::Error& e) {
    kdb_ctx_set_error(ctx, e.what());
    return e.code;
  } catch (const std::exception& e) {
    kdb_ctx_set_error(ctx, e.what());
    return KDB_ERR_CUDA;
  }
}

const char* kdb_mlp_last_error(kdb_mlp* m) { return m ? m->err.c_str() : "null model"; }

int kdb_mlp_set_params(kdb_mlp* m, const float* params, int64_t n) {
  return MGuard(m, [&] {
    if (!params || n != kdb::JoinPrior::kParams) throw kdb::Error(KDB_ERR_INVALID, "wrong parameter count");
    m->p->SetParams(params);
  });
}

int kdb_mlp_get_params(kdb_mlp* m, float* params, int64_t n) {
  return MGuard(m, [&] {
    if (!params || n != kdb::JoinPrior::kParams) throw kdb::Error(KDB_ERR_INVALID, "wrong parameter count");
    m->p->GetParams(params);
  });
}

int kdb_mlp_forward(kdb_mlp* m, const float* x, int64_t n, float* y) {
  return MGuard(m, [&] {
    if (!x || !y) throw kdb::Error(KDB_ERR_INVALID, "null buffer");
    m->p->Forward(x, n, y);
  });
}

int kdb_mlp_gradient(kdb_mlp* m, const float* x, const float* t, int64_t n, float* grad, double* loss) {
  return MGuard(m, [&] {
    if (!x || !t || !grad) throw kdb::Error(KDB_ERR_INVALID, "null buffer");
    double l = m->p->Gradient(x, t, n, grad);
    if (loss) *loss = l;
  });
}

int kdb_mlp_train_step(kdb_mlp* m, const float* x, const float* t, int64_t n, float lr, double* loss) {
  return MGuard(m, [&] {
    if (!x || !t) throw kdb::Error(KDB_ERR_INVALID, "null buffer");
    double l = m->p->TrainStep(x, t, n, lr);
    if (loss) *loss = l;
  });
}

void kdb_mlp_free(kdb_mlp* m) { delete m; }

int kdb_ctx_set_skinner_policy(kdb_ctx* ctx, int32_t policy, kdb_mlp* prior, int32_t log_samples) {
  if (!ctx || policy < 0 || policy > 2) return KDB_ERR_INVALID;
  kdb::Context& c = *kdb_ctx_context(ctx);
  if (policy == 1 && !prior) {
    kdb_ctx_set_error(ctx, "the prior policy needs a model");
    return KDB_ERR_INVALID;
  }
  if (prior && prior->p->device() != c.device) {
    kdb_ctx_set_error(ctx, "the model lives on another device");
    return KDB_ERR_INVALID;
  }
  c.skinner_policy = policy;
  c.join_prior = prior ? prior->p.get() : nullptr;
  c.skinner_log = log_samples != 0;
  return KDB_OK;
}

}  // extern "C"
