// Per-cell arithmetic shared by the standalone collision kernels and the
// fused schedules: the SRD rotation matrix (src/mpcd.f90:163-171), the
// rotation about the cell mean (src/mpcd.f90:173-175) and the per-cell sums.
//
// FP64: sums are sequential in particle order and every expression keeps the
// reference association, so results equal the reference's single-thread
// arithmetic.  FP32: sums use Neumaier's compensated two-sum, so the cell
// mean carries ~1 ulp of float error independent of the cell population.
#pragma once
#include "rmpcd_common.cuh"

namespace rmpcd {

template <typename R>
struct CellSum;

template <>
struct CellSum<double> {
    double s = 0;
    __device__ inline void add(double v) { s = s + v; }
    __device__ inline double value() const { return s; }
};

template <>
struct CellSum<float> {
    float s = 0.f, c = 0.f;
    __device__ inline void add(float v)
    {
        float t = s + v;
        if (fabsf(s) >= fabsf(v)) c += (s - t) + v;
        else c += (v - t) + s;
        s = t;
    }
    __device__ inline float value() const { return s + c; }
};

// omega(r, c) of src/mpcd.f90:163-171 (the reshape is column-major)
struct Rot {
    double m[3][3];
};

__host__ __device__ inline Rot srd_matrix(double v0, double v1, double v2, double sin_a, double cos_a)
{
    Rot o;
    double omc = 1 - cos_a;
    o.m[0][0] = cos_a + v0 * v0 * omc;
    o.m[1][0] = v0 * v1 * omc - v2 * sin_a;
    o.m[2][0] = v0 * v2 * omc + v1 * sin_a;
    o.m[0][1] = v1 * v0 * omc + v2 * sin_a;
    o.m[1][1] = cos_a + v1 * v1 * omc;
    o.m[2][1] = v1 * v2 * omc - v0 * sin_a;
    o.m[0][2] = v2 * v0 * omc - v1 * sin_a;
    o.m[1][2] = v2 * v1 * omc + v0 * sin_a;
    o.m[2][2] = cos_a + v2 * v2 * omc;
    return o;
}

// v = lv + matmul(omega, v - lv), matmul accumulating over k = 1, 2, 3
template <typename R>
__device__ inline void srd_rotate(R &x, R &y, R &z, const R lv[3], const Rot &o)
{
    R d0 = x - lv[0], d1 = y - lv[1], d2 = z - lv[2];
    R r0 = (R)o.m[0][0] * d0 + (R)o.m[0][1] * d1 + (R)o.m[0][2] * d2;
    R r1 = (R)o.m[1][0] * d0 + (R)o.m[1][1] * d1 + (R)o.m[1][2] * d2;
    R r2 = (R)o.m[2][0] * d0 + (R)o.m[2][1] * d1 + (R)o.m[2][2] * d2;
    x = lv[0] + r0;
    y = lv[1] + r1;
    z = lv[2] + r2;
}

}  // namespace rmpcd
