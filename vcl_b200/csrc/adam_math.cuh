// Adam update of one parameter, shared by the per-operator Adam and the
// fused optimizer kernels.
#pragma once
#include "common.cuh"

// optimize.cu:95-106: moments rounded to FP32, update in FP64, NaN-guarded.
DEV void adam_one(float& p, float g, float& m, float& v, double b1, double b2, double lr, double eps, double c1,
                  double c2) {
    m = (float)__dadd_rn(__dmul_rn(b1, (double)m), __dmul_rn(1.0 - b1, (double)g));
    v = (float)__dadd_rn(__dmul_rn(b2, (double)v), __dmul_rn(__dmul_rn(1.0 - b2, (double)g), (double)g));
    double mh = (double)m / c1;
    double vh = (double)v / c2;
    add_nan_check(p, (float)(-mh * lr / (sqrt(vh) + eps)));
}

