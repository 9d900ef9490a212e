// The device engine behind a CKKSContext (internal to the reference-API layer).
#pragma once
#include <random>
#include <vector>

#include "../../../include/walsh_gpu.h"
#include "ckks_context.hpp"

struct CKKSContext::Engine {
    explicit Engine(CKKSParams p) : params(std::move(p)) {}
    ~Engine();
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    CKKSParams params;
    wg_context* ctx = nullptr;
    std::vector<wg_lt_stage*> s2c, s2c_x2, c2s;  // SlotToCoeff (x1, x2 input scale), CoeffToSlot
    double c2s_transform_scale = 1.0;
    PolynomialApproximation evalmod;
    bool has_evalmod = false, has_plans = false, has_switch_keys = false;
    std::vector<int8_t> secret, low_secret;  // dense and sparse (bootstrapping) secrets
    std::vector<int64_t> rotations;          // installed rotation keys, normalised
    std::random_device rd;

    uint64_t next_seed();
    std::vector<wg_lt_stage*> make_plan(bool c2s_plan, double transform_scale);
    wg_bootstrap_params bootstrap_params() const;
};
