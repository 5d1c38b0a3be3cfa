// Learned round schedule: the FP32 MLP and the policy that uses it.
#pragma once

#include "presolve.hpp"

namespace gpp {

constexpr int kScheduleHidden = 64;
constexpr int kScheduleOutputs = kGatedRules + 1;   // per gated rule "will change the model", then "stop"
// Flat parameter vector: W1[F][H], b1[H], W2[H][H], b2[H], W3[H][O], b3[O]
// (W[k][j] row-major: input k, unit j).
constexpr int64_t kScheduleParams = int64_t(kScheduleFeatures) * kScheduleHidden + kScheduleHidden +
                                    int64_t(kScheduleHidden) * kScheduleHidden + kScheduleHidden +
                                    int64_t(kScheduleHidden) * kScheduleOutputs + kScheduleOutputs;

// Host arrays in, host arrays out; the work runs on the engine stream.
// X: n x kScheduleFeatures, Y and M (labels, 0/1 masks): n x kScheduleOutputs.
void mlp_train(float* params, const float* X, const float* Y, const float* M, int64_t n, int epochs, int batch,
               float lr, uint64_t seed, float* loss_per_epoch);
void mlp_forward(const float* params, const float* X, int64_t n, float* probs);
// Gradient of the mean masked loss over the n samples, and that loss.
void mlp_gradients(const float* params, const float* X, const float* Y, const float* M, int64_t n, float* grads,
                   float* loss);

// Skips gated rule g when its probability is below `skip_below[g]`; stops
// when the stop probability is above `stop_above` (never when stop_above >= 1).
class MlpSchedule final : public SchedulePolicy {
 public:
  MlpSchedule(const float* params, const double* skip_below, double stop_above);
  uint32_t decide(const float* features, bool* stop) override;
  int64_t decisions() const { return decisions_; }

 private:
  DBuf<float> weights_;
  double skip_below_[kGatedRules];
  double stop_above_;
  int64_t decisions_ = 0;
};

}  // namespace gpp
