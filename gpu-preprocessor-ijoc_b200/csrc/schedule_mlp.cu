// Learned round schedule: a small FP32 MLP (kScheduleFeatures -> 64 -> 64 ->
// kGatedRules + 1) with hand-written training and inference kernels, and the
// SchedulePolicy that consults it once per round of the phase machine.
//
// Outputs are logits: output g < kGatedRules says "gated rule g will change
// the model this round", the last one says "stop now".  Training minimises
// the masked binary cross-entropy of those logits against labels taken from
// traces of the plain phase machine.  Everything is dense and tiny (a 64-wide
// layer), so plain FP32 SIMT kernels are used; there is nothing here for the
// tensor cores to speed up.
#include <cmath>
#include <numeric>
#include <random>
#include <stdexcept>
#include <vector>

#include "presolve.hpp"
#include "schedule_mlp.hpp"

namespace gpp {

namespace {

constexpr int F = kScheduleFeatures, H = kScheduleHidden, O = kScheduleOutputs;
// Offsets of the parameter blocks in the flat parameter vector.
constexpr int64_t kW1 = 0, kB1 = kW1 + int64_t(F) * H, kW2 = kB1 + H, kB2 = kW2 + int64_t(H) * H, kW3 = kB2 + H,
                  kB3 = kW3 + int64_t(H) * O;
static_assert(kB3 + O == kScheduleParams, "parameter layout");

// Y[r][j] = act(b[j] + sum_k X[r][k] W[k][j]); one thread per (r, j).
__global__ void dense_forward(const float* __restrict__ X, int64_t rows, int K, const float* __restrict__ W,
                              const float* __restrict__ b, int N, int relu, float* __restrict__ Y) {
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= rows * N) return;
  const int64_t r = t / N;
  const int j = int(t % N);
  float acc = b[j];
  for (int k = 0; k < K; ++k) acc = fmaf(X[r * K + k], W[int64_t(k) * N + j], acc);
  Y[t] = relu ? fmaxf(acc, 0.0f) : acc;
}

// Masked binary cross-entropy on logits: dZ = scale * M (sigmoid(Z) - Y) and
// the summed loss (numerically stable form).
__global__ void bce_grad(const float* __restrict__ Z, const float* __restrict__ Y, const float* __restrict__ M,
                         int64_t count, float scale, float* __restrict__ dZ, float* __restrict__ loss) {
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  float l = 0.0f;
  if (t < count) {
    const float z = Z[t], y = Y[t], m = M[t];
    const float p = 1.0f / (1.0f + expf(-z));
    dZ[t] = scale * m * (p - y);
    l = m * (fmaxf(z, 0.0f) - z * y + log1pf(expf(-fabsf(z))));
  }
  for (int off = 16; off; off >>= 1) l += __shfl_down_sync(0xffffffffu, l, off);
  if ((threadIdx.x & 31) == 0 && l != 0.0f) atomicAdd(loss, l);
}

// dX[r][k] = sum_j dY[r][j] W[k][j], times (X[r][k] > 0) when X is a ReLU
// output; one thread per (r, k).
__global__ void dense_backward_input(const float* __restrict__ dY, int64_t rows, int N, const float* __restrict__ W,
                                     int K, const float* __restrict__ Xrelu, float* __restrict__ dX) {
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= rows * K) return;
  const int64_t r = t / K;
  const int k = int(t % K);
  float acc = 0.0f;
  for (int j = 0; j < N; ++j) acc = fmaf(dY[r * N + j], W[int64_t(k) * N + j], acc);
  dX[t] = Xrelu && Xrelu[t] <= 0.0f ? 0.0f : acc;
}

// dW[k][j] = sum_r X[r][k] dY[r][j] and db[j] = sum_r dY[r][j], summed over the
// rows in order (deterministic); one thread per parameter.
__global__ void dense_backward_params(const float* __restrict__ X, const float* __restrict__ dY, int64_t rows, int K,
                                      int N, float* __restrict__ dW, float* __restrict__ db) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < K * N) {
    const int k = t / N, j = t % N;
    float acc = 0.0f;
    for (int64_t r = 0; r < rows; ++r) acc = fmaf(X[r * K + k], dY[r * N + j], acc);
    dW[t] = acc;
  } else if (t < K * N + N) {
    const int j = t - K * N;
    float acc = 0.0f;
    for (int64_t r = 0; r < rows; ++r) acc += dY[r * N + j];
    db[j] = acc;
  }
}

// Adam (Kingma & Ba, 2015) with bias correction.
__global__ void adam_step(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                          const float* __restrict__ g, int64_t count, float lr, float beta1, float beta2, float eps,
                          float c1, float c2) {
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= count) return;
  const float gt = g[t];
  const float mt = beta1 * m[t] + (1.0f - beta1) * gt;
  const float vt = beta2 * v[t] + (1.0f - beta2) * gt * gt;
  m[t] = mt;
  v[t] = vt;
  w[t] -= lr * (mt / c1) / (sqrtf(vt / c2) + eps);
}

__global__ void gather_rows(const float* __restrict__ src, const int32_t* __restrict__ rows, int64_t count, int width,
                            float* __restrict__ dst) {
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= count * width) return;
  dst[t] = src[int64_t(rows[t / width]) * width + t % width];
}

__global__ void sigmoid_kernel(float* z, int64_t count) {
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t < count) z[t] = 1.0f / (1.0f + expf(-z[t]));
}

// Inference on one feature vector: one block of H threads, layer by layer in
// shared memory; out[o] = sigmoid(logit o).
__global__ void __launch_bounds__(kScheduleHidden) forward_one(const float* __restrict__ params,
                                                               const float* __restrict__ x, float* __restrict__ out) {
  __shared__ float in[kScheduleFeatures], h1[kScheduleHidden], h2[kScheduleHidden];
  const int j = threadIdx.x;
  if (j < F) in[j] = x[j];
  __syncthreads();
  float a = params[kB1 + j];
  for (int k = 0; k < F; ++k) a = fmaf(in[k], params[kW1 + int64_t(k) * H + j], a);
  h1[j] = fmaxf(a, 0.0f);
  __syncthreads();
  a = params[kB2 + j];
  for (int k = 0; k < H; ++k) a = fmaf(h1[k], params[kW2 + int64_t(k) * H + j], a);
  h2[j] = fmaxf(a, 0.0f);
  __syncthreads();
  if (j < O) {
    a = params[kB3 + j];
    for (int k = 0; k < H; ++k) a = fmaf(h2[k], params[kW3 + int64_t(k) * O + j], a);
    out[j] = 1.0f / (1.0f + expf(-a));
  }
}

int grid_for(int64_t n) { return int(std::max<int64_t>(1, (n + kThreads - 1) / kThreads)); }

// Activations and gradients of one batch of `rows` samples.
struct Workspace {
  DBuf<float> a1, a2, z3, d3, d2, d1, grads, loss;
  void ensure(int64_t rows, cudaStream_t s) {
    if (a1.n < size_t(rows * H)) {
      a1.alloc(size_t(rows * H), s); a2.alloc(size_t(rows * H), s);
      d2.alloc(size_t(rows * H), s); d1.alloc(size_t(rows * H), s);
      z3.alloc(size_t(rows * O), s); d3.alloc(size_t(rows * O), s);
    }
    if (grads.n < size_t(kScheduleParams)) grads.alloc(size_t(kScheduleParams), s);
    if (loss.n < 1) loss.alloc(1, s);
  }
};

void forward_batch(const float* w, const float* X, int64_t rows, Workspace& ws, cudaStream_t s) {
  GPP_LAUNCH(dense_forward, grid_for(rows * H), kThreads, 0, s, X, rows, F, w + kW1, w + kB1, H, 1, ws.a1.p);
  GPP_LAUNCH(dense_forward, grid_for(rows * H), kThreads, 0, s, ws.a1.p, rows, H, w + kW2, w + kB2, H, 1, ws.a2.p);
  GPP_LAUNCH(dense_forward, grid_for(rows * O), kThreads, 0, s, ws.a2.p, rows, H, w + kW3, w + kB3, O, 0, ws.z3.p);
}

// Gradients of the mean (over rows) masked loss into ws.grads; the summed
// loss into ws.loss[0] (added to).
void backward_batch(const float* w, const float* X, const float* Y, const float* M, int64_t rows, Workspace& ws,
                    cudaStream_t s) {
  const float scale = 1.0f / float(rows);
  GPP_LAUNCH(bce_grad, grid_for(rows * O), kThreads, 0, s, ws.z3.p, Y, M, rows * O, scale, ws.d3.p, ws.loss.p);
  float* g = ws.grads.p;
  GPP_LAUNCH(dense_backward_params, grid_for(H * O + O), kThreads, 0, s, ws.a2.p, ws.d3.p, rows, H, O, g + kW3,
             g + kB3);
  GPP_LAUNCH(dense_backward_input, grid_for(rows * H), kThreads, 0, s, ws.d3.p, rows, O, w + kW3, H, ws.a2.p, ws.d2.p);
  GPP_LAUNCH(dense_backward_params, grid_for(H * H + H), kThreads, 0, s, ws.a1.p, ws.d2.p, rows, H, H, g + kW2,
             g + kB2);
  GPP_LAUNCH(dense_backward_input, grid_for(rows * H), kThreads, 0, s, ws.d2.p, rows, H, w + kW2, H, ws.a1.p, ws.d1.p);
  GPP_LAUNCH(dense_backward_params, grid_for(F * H + H), kThreads, 0, s, X, ws.d1.p, rows, F, H, g + kW1, g + kB1);
}

}  // namespace

void mlp_gradients(const float* params, const float* X, const float* Y, const float* M, int64_t n, float* grads,
                   float* loss) {
  if (n <= 0) throw std::invalid_argument("mlp_gradients: no samples");
  auto s = ctx().stream;
  DBuf<float> w(size_t(kScheduleParams), s), dx(size_t(n * F), s), dy(size_t(n * O), s), dm(size_t(n * O), s);
  check(cudaMemcpyAsync(w.p, params, sizeof(float) * kScheduleParams, cudaMemcpyHostToDevice, s), "params");
  check(cudaMemcpyAsync(dx.p, X, sizeof(float) * size_t(n * F), cudaMemcpyHostToDevice, s), "X");
  check(cudaMemcpyAsync(dy.p, Y, sizeof(float) * size_t(n * O), cudaMemcpyHostToDevice, s), "Y");
  check(cudaMemcpyAsync(dm.p, M, sizeof(float) * size_t(n * O), cudaMemcpyHostToDevice, s), "M");
  Workspace ws;
  ws.ensure(n, s);
  ws.loss.zero();
  forward_batch(w.p, dx.p, n, ws, s);
  backward_batch(w.p, dx.p, dy.p, dm.p, n, ws, s);
  check(cudaMemcpyAsync(grads, ws.grads.p, sizeof(float) * kScheduleParams, cudaMemcpyDeviceToHost, s), "grads");
  float l = 0.0f;
  check(cudaMemcpyAsync(&l, ws.loss.p, sizeof(float), cudaMemcpyDeviceToHost, s), "loss");
  ctx().sync("mlp gradients");
  if (loss) *loss = l / float(n);
}

void mlp_forward(const float* params, const float* X, int64_t n, float* probs) {
  if (n <= 0) return;
  auto s = ctx().stream;
  DBuf<float> w(size_t(kScheduleParams), s), dx(size_t(n * F), s);
  check(cudaMemcpyAsync(w.p, params, sizeof(float) * kScheduleParams, cudaMemcpyHostToDevice, s), "params");
  check(cudaMemcpyAsync(dx.p, X, sizeof(float) * size_t(n * F), cudaMemcpyHostToDevice, s), "X");
  Workspace ws;
  ws.ensure(n, s);
  forward_batch(w.p, dx.p, n, ws, s);
  GPP_LAUNCH(sigmoid_kernel, grid_for(n * O), kThreads, 0, s, ws.z3.p, n * O);
  check(cudaMemcpyAsync(probs, ws.z3.p, sizeof(float) * size_t(n * O), cudaMemcpyDeviceToHost, s), "probs");
  ctx().sync("mlp forward");
}

void mlp_train(float* params, const float* X, const float* Y, const float* M, int64_t n, int epochs, int batch,
               float lr, uint64_t seed, float* loss_per_epoch) {
  if (n <= 0 || epochs < 0 || batch <= 0) throw std::invalid_argument("mlp_train: empty data or bad settings");
  auto s = ctx().stream;
  DBuf<float> w(size_t(kScheduleParams), s), m(size_t(kScheduleParams), s), v(size_t(kScheduleParams), s);
  DBuf<float> dx(size_t(n * F), s), dy(size_t(n * O), s), dm(size_t(n * O), s);
  DBuf<float> bx(size_t(batch) * F, s), by(size_t(batch) * O, s), bm(size_t(batch) * O, s);
  DBuf<int32_t> rows_d(size_t(n), s);
  check(cudaMemcpyAsync(w.p, params, sizeof(float) * kScheduleParams, cudaMemcpyHostToDevice, s), "params");
  check(cudaMemcpyAsync(dx.p, X, sizeof(float) * size_t(n * F), cudaMemcpyHostToDevice, s), "X");
  check(cudaMemcpyAsync(dy.p, Y, sizeof(float) * size_t(n * O), cudaMemcpyHostToDevice, s), "Y");
  check(cudaMemcpyAsync(dm.p, M, sizeof(float) * size_t(n * O), cudaMemcpyHostToDevice, s), "M");
  m.zero();
  v.zero();
  Workspace ws;
  ws.ensure(batch, s);
  std::vector<int32_t> order(static_cast<size_t>(n));
  std::iota(order.begin(), order.end(), 0);
  std::mt19937_64 rng(seed);
  const float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
  int step = 0;
  for (int e = 0; e < epochs; ++e) {
    std::shuffle(order.begin(), order.end(), rng);
    check(cudaMemcpyAsync(rows_d.p, order.data(), sizeof(int32_t) * size_t(n), cudaMemcpyHostToDevice, s), "order");
    ws.loss.zero();
    for (int64_t b0 = 0; b0 < n; b0 += batch) {
      const int64_t rows = std::min<int64_t>(batch, n - b0);
      GPP_LAUNCH(gather_rows, grid_for(rows * F), kThreads, 0, s, dx.p, rows_d.p + b0, rows, F, bx.p);
      GPP_LAUNCH(gather_rows, grid_for(rows * O), kThreads, 0, s, dy.p, rows_d.p + b0, rows, O, by.p);
      GPP_LAUNCH(gather_rows, grid_for(rows * O), kThreads, 0, s, dm.p, rows_d.p + b0, rows, O, bm.p);
      forward_batch(w.p, bx.p, rows, ws, s);
      backward_batch(w.p, bx.p, by.p, bm.p, rows, ws, s);
      ++step;
      const float c1 = 1.0f - std::pow(beta1, float(step)), c2 = 1.0f - std::pow(beta2, float(step));
      GPP_LAUNCH(adam_step, grid_for(kScheduleParams), kThreads, 0, s, w.p, m.p, v.p, ws.grads.p,
                 int64_t(kScheduleParams), lr, beta1, beta2, eps, c1, c2);
    }
    if (loss_per_epoch) {
      float l = 0.0f;
      check(cudaMemcpyAsync(&l, ws.loss.p, sizeof(float), cudaMemcpyDeviceToHost, s), "loss");
      ctx().sync("mlp epoch");
      loss_per_epoch[e] = l / float(n);
    }
    // The shuffled order uploaded for this epoch must not be overwritten
    // before its gathers ran.
    ctx().sync("mlp epoch order");
  }
  check(cudaMemcpyAsync(params, w.p, sizeof(float) * kScheduleParams, cudaMemcpyDeviceToHost, s), "params out");
  ctx().sync("mlp train");
}

// ---- the policy ---------------------------------------------------------------

MlpSchedule::MlpSchedule(const float* params, const double* skip_below, double stop_above) : stop_above_(stop_above) {
  std::copy(skip_below, skip_below + kGatedRules, skip_below_);
  auto s = ctx().stream;
  weights_.alloc(size_t(kScheduleParams), s);
  check(cudaMemcpyAsync(weights_.p, params, sizeof(float) * kScheduleParams, cudaMemcpyHostToDevice, s), "weights");
  ctx().sync("schedule weights");
}

uint32_t MlpSchedule::decide(const float* features, bool* stop) {
  auto& c = ctx();
  // Features in, probabilities out, through the context's pinned status
  // block (kScheduleFeatures + kScheduleOutputs floats fit in it).
  static_assert(kScheduleFeatures + kScheduleOutputs <= Context::kStatusWords, "pinned block too small");
  float* host = reinterpret_cast<float*>(c.host_status);
  std::copy(features, features + kScheduleFeatures, host);
  DBuf<float> io(size_t(kScheduleFeatures + kScheduleOutputs), c.stream);
  check(cudaMemcpyAsync(io.p, host, sizeof(float) * kScheduleFeatures, cudaMemcpyHostToDevice, c.stream), "features");
  GPP_LAUNCH(forward_one, 1, kScheduleHidden, 0, c.stream, weights_.p, io.p, io.p + kScheduleFeatures);
  check(cudaMemcpyAsync(host + kScheduleFeatures, io.p + kScheduleFeatures, sizeof(float) * kScheduleOutputs,
                        cudaMemcpyDeviceToHost, c.stream),
        "decision");
  c.sync("schedule decision");
  const float* p = host + kScheduleFeatures;
  uint32_t skip = 0;
  for (int g = 0; g < kGatedRules; ++g)
    if (double(p[g]) < skip_below_[g]) skip |= 1u << g;
  *stop = stop_above_ < 1.0 && double(p[kGatedRules]) > stop_above_;
  ++decisions_;
  return skip;
}

}  // namespace gpp
