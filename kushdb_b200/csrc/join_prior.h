// Learned join-order prior for the Skinner join: a 64 -> 128 -> 128 -> 128
// -> 1 ReLU MLP (fp32) that predicts the episode reward of appending a
// candidate table to a join-order prefix.  Forward, backward and the Adam
// update are hand-written CUDA kernels (join_prior.cu); the reference has
// no counterpart (its UctJoinAgent, runtime/skinner_join_executor.cc:779-838,
// searches without a prior).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <vector>

namespace kdb {

class Context;

class JoinPrior {
 public:
  static constexpr int kIn = 64;
  static constexpr int kHid = 128;
  static constexpr int kMaxRows = 4096;  // rows per forward / gradient call
  // parameter layout: W1[kIn][kHid] b1 W2[kHid][kHid] b2 W3[kHid][kHid] b3 w4[kHid] b4
  static constexpr int64_t kOffW1 = 0;
  static constexpr int64_t kOffB1 = kOffW1 + kIn * kHid;
  static constexpr int64_t kOffW2 = kOffB1 + kHid;
  static constexpr int64_t kOffB2 = kOffW2 + kHid * kHid;
  static constexpr int64_t kOffW3 = kOffB2 + kHid;
  static constexpr int64_t kOffB3 = kOffW3 + kHid * kHid;
  static constexpr int64_t kOffW4 = kOffB3 + kHid;
  static constexpr int64_t kOffB4 = kOffW4 + kHid;
  static constexpr int64_t kParams = kOffB4 + 1;

  JoinPrior(int device, uint32_t seed);
  ~JoinPrior();
  JoinPrior(const JoinPrior&) = delete;
  JoinPrior& operator=(const JoinPrior&) = delete;

  void SetParams(const float* p);
  void GetParams(float* p);
  // y[i] = MLP(x[i]) for n host rows of kIn features.
  void Forward(const float* x, int64_t n, float* y);
  // Gradient of the mean squared error over the n rows (no update); returns
  // the loss.
  double Gradient(const float* x, const float* t, int64_t n, float* grad);
  // One Adam step on the mean squared error; returns the loss before it.
  double TrainStep(const float* x, const float* t, int64_t n, float lr);
  int device() const { return device_; }

 private:
  double Run(const float* x, const float* t, int64_t n, float* grad, float lr, float* y);
  int device_;
  std::mutex mu_;
  cudaStream_t stream_ = nullptr;
  float* p_ = nullptr;  // parameters
  float* m_ = nullptr;  // Adam moments
  float* v_ = nullptr;
  float* x_ = nullptr;
  float* t_ = nullptr;
  float* y_ = nullptr;
  float* h_ = nullptr;        // saved activations H1, H2, H3
  float* partial_ = nullptr;  // per-CTA gradient partials
  float* grad_ = nullptr;
  float* pinned_ = nullptr;
  int64_t step_ = 0;
};

}  // namespace kdb
