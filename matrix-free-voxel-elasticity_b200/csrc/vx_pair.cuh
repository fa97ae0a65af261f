// Pairs of values processed in lockstep: the two elements (or two node columns) a thread of the
// streaming operator owns.  FP32 pairs are float2 registers driven by sm_100's packed f32x2
// arithmetic (one instruction per pair); FP64 pairs are two scalar operations.
#pragma once
#include <cuda_runtime.h>

namespace vx {

template <typename T> struct V2;
template <> struct V2<double> {
    double x, y;
    __device__ __forceinline__ double lo() const { return x; }
    __device__ __forceinline__ double hi() const { return y; }
};
template <> struct V2<float> {
    float2 v;
    __device__ __forceinline__ float lo() const { return v.x; }
    __device__ __forceinline__ float hi() const { return v.y; }
};

__device__ __forceinline__ V2<double> mk2(double a, double b) { return {a, b}; }
__device__ __forceinline__ V2<float> mk2(float a, float b) { return {make_float2(a, b)}; }

__device__ __forceinline__ V2<double> add2(V2<double> a, V2<double> b) { return {a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ V2<double> sub2(V2<double> a, V2<double> b) { return {a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ V2<double> mul2(V2<double> a, V2<double> b) { return {a.x * b.x, a.y * b.y}; }
__device__ __forceinline__ V2<double> fma2(V2<double> a, V2<double> b, V2<double> c) {
    return {fma(a.x, b.x, c.x), fma(a.y, b.y, c.y)};
}

__device__ __forceinline__ V2<float> add2(V2<float> a, V2<float> b) { return {__fadd2_rn(a.v, b.v)}; }
__device__ __forceinline__ V2<float> sub2(V2<float> a, V2<float> b) {
    return {__ffma2_rn(b.v, make_float2(-1.f, -1.f), a.v)};             // exact a - b
}
__device__ __forceinline__ V2<float> mul2(V2<float> a, V2<float> b) { return {__fmul2_rn(a.v, b.v)}; }
__device__ __forceinline__ V2<float> fma2(V2<float> a, V2<float> b, V2<float> c) {
    return {__ffma2_rn(a.v, b.v, c.v)};
}

// coefficient broadcast to both lanes of a pair (FP32: a pre-duplicated float2 constant)
template <typename T> struct Coef;
template <> struct Coef<double> { using type = double; };
template <> struct Coef<float> { using type = float2; };
__device__ __forceinline__ V2<double> cmul2(double c, V2<double> a) { return {c * a.x, c * a.y}; }
__device__ __forceinline__ V2<double> cfma2(double c, V2<double> a, V2<double> acc) {
    return {fma(c, a.x, acc.x), fma(c, a.y, acc.y)};
}
__device__ __forceinline__ V2<float> cmul2(float2 c, V2<float> a) { return {__fmul2_rn(c, a.v)}; }
__device__ __forceinline__ V2<float> cfma2(float2 c, V2<float> a, V2<float> acc) { return {__ffma2_rn(c, a.v, acc.v)}; }

// whole-pair shuffles: an FP32 pair moves as one 64-bit value, so both halves land in an aligned
// register pair; an FP64 pair is two 64-bit shuffles
__device__ __forceinline__ V2<float> shfl_down2(V2<float> a, int d) {
    const unsigned long long b = __shfl_down_sync(0xffffffffu, *reinterpret_cast<const unsigned long long*>(&a.v), d);
    return {*reinterpret_cast<const float2*>(&b)};
}
__device__ __forceinline__ V2<float> shfl_up2(V2<float> a, int d) {
    const unsigned long long b = __shfl_up_sync(0xffffffffu, *reinterpret_cast<const unsigned long long*>(&a.v), d);
    return {*reinterpret_cast<const float2*>(&b)};
}
__device__ __forceinline__ V2<double> shfl_down2(V2<double> a, int d) {
    return {__shfl_down_sync(0xffffffffu, a.x, d), __shfl_down_sync(0xffffffffu, a.y, d)};
}
__device__ __forceinline__ V2<double> shfl_up2(V2<double> a, int d) {
    return {__shfl_up_sync(0xffffffffu, a.x, d), __shfl_up_sync(0xffffffffu, a.y, d)};
}

}  // namespace vx
