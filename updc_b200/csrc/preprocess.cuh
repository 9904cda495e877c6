// Per-exposure weight preprocessing drivers (preprocess.cu).
#pragma once

#include <string>

#include "../../include/updc_b200.h"
#include "common.cuh"

namespace updc {

void preprocess_exposure(const float *sci, const uint32_t *dq, const double *vp, const double *vr,
                         const double *vf, size_t n, int mode, uint32_t bad, double pedestal_sigma,
                         const std::string &source, float *wht, uint8_t *sky, updc_preprocess_metrics *M,
                         bool device_pointers, cudaStream_t st);

void robust_background(const float *sci, const uint8_t *base_valid, size_t n, int max_iter, uint8_t *mask,
                       double *background, double *sigma, int *passes, bool device_pointers, cudaStream_t st);

}  // namespace updc
