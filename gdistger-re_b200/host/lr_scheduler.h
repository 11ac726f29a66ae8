// Per-round learning-rate schedules of the SGNS trainer.
//
// Same classes, constructor arguments and arithmetic types as the reference's
// include/lr_scheduler.hpp:5-81: get_lr() is called once per walk round and
// advances the step counter.  word2vec.cu:1279 drives training with
// ExponentialDecayLR(0.025, 0.1).
#pragma once

#include <cmath>

namespace dg_host {

class LR {
  public:
    explicit LR(float initial_lr) : initial_lr(initial_lr), step(0) {}
    virtual ~LR() = default;
    virtual float get_lr() = 0;

  protected:
    float initial_lr;
    int step;
};

class FixedLR : public LR {
  public:
    explicit FixedLR(float initial_lr) : LR(initial_lr) {}
    float get_lr() override { return initial_lr; }
};

// initial_lr * exp(-decay_rate * step), evaluated in float (lr_scheduler.hpp:23-31).
class ExponentialDecayLR : public LR {
  public:
    ExponentialDecayLR(float initial_lr, float decay_rate) : LR(initial_lr), decay_rate(decay_rate) {}
    float get_lr() override { return initial_lr * std::exp(-decay_rate * static_cast<float>(step++)); }

  private:
    float decay_rate;
};

// min_lr + (initial_lr - min_lr) * (1 + cos(pi * step / T_max)) / 2 (lr_scheduler.hpp:33-45).
class CosineAnnealingLR : public LR {
  public:
    CosineAnnealingLR(float initial_lr, float min_lr, int t_max) : LR(initial_lr), min_lr(min_lr), t_max(t_max) {}
    float get_lr() override {
        const float cosine = static_cast<float>(std::cos(M_PI * step / t_max));
        const float lr = static_cast<float>(min_lr + 0.5 * (initial_lr - min_lr) * (1 + cosine));
        ++step;
        return lr;
    }

  private:
    double min_lr;
    int t_max;
};

// initial_lr * decay_factor ^ (step / step_size) (lr_scheduler.hpp:47-62).
class StepDecayLR : public LR {
  public:
    StepDecayLR(float initial_lr, float decay_factor, int step_size)
        : LR(initial_lr), decay_factor(decay_factor), step_size(step_size) {}
    float get_lr() override {
        const int factor = step / step_size;
        ++step;
        return static_cast<float>(initial_lr * std::pow(decay_factor, factor));
    }

  private:
    float decay_factor;
    int step_size;
};

// x0.8 every fifth call, starting with the first (lr_scheduler.hpp:64-77).
class CustomLR : public LR {
  public:
    explicit CustomLR(float initial_lr) : LR(initial_lr) {}
    float get_lr() override {
        if (step % 5 == 0) initial_lr = static_cast<float>(initial_lr * 0.8);
        ++step;
        return initial_lr;
    }
};

}  // namespace dg_host
