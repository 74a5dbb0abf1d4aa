/*
 * sforacle.h — internal declarations of the CPU restatement (test infrastructure only).
 * The extern "C" entry points are bound from Python with ctypes (tests/oracle_binding.py).
 */
#ifndef SFORACLE_H
#define SFORACLE_H

#include "../include/rgbdflow.h"

#ifdef __cplusplus
namespace sfo {
struct LevelTrace {
    int outer = 0;
    int sor[RGBDFLOW_MAX_OUTER] = {0};
    float maxdiff[RGBDFLOW_MAX_OUTER] = {0};
    float stat[RGBDFLOW_MAX_OUTER] = {0};
};
struct Trace {
    int n_levels = 0;
    int w[RGBDFLOW_MAX_LEVELS] = {0}, h[RGBDFLOW_MAX_LEVELS] = {0};
    LevelTrace lev[RGBDFLOW_MAX_LEVELS];
};
} // namespace sfo
extern "C" {
#endif

/* Same values as rgbdflow_params_default() of the library, restated so the oracle links alone:
 * sceneFlowParams() (OpticalFlow.h:107-109) + setUpSceneFlowParams (runFlowTwoFrames.cpp:66-100)
 * + the solver constants of sceneFlowSingleScaleJacobiCUDA.cu. */
static inline void rgbdflow_params_default_oracle(rgbdflow_params* p)
{
    p->regularization = RGBDFLOW_REG_HPB;
    p->color_data_weight = 1;
    p->depth_vs_color_data_weight = 1;
    p->alpha = 0.02;
    p->gamma = 1e-5;
    p->pyramid_ratio = 0.75;
    p->min_width = 60;
    p->n_outer = 50;
    p->n_inner = 1;
    p->n_sor = 10000;
    p->depth_boundary_dist = 4;
    p->fill_holes = 1;
    p->fixed_schedule = 0;
    p->storage = RGBDFLOW_STORE_FP32;
    p->compute = RGBDFLOW_COMPUTE_FP32;
    p->omega = 0.7;
    p->max_flow_step = 0.3;
    p->eps_d = 1e-6;
    p->eps_z = 1e-10;
    p->eps_s = 1e-6;
    p->sor_tol = 1e-5;
    p->sor_check_period = 25;
    p->outer_tol = 4e-4;
    p->occ_margin = 0.02;
    p->occ_penalty = 0.01;
    p->max_depth_grad = 0.04;
    p->sweeps_per_launch = 0;
}

#ifdef __cplusplus
}
#endif
#endif
