// common.cuh - precision traits, complex helpers and small device utilities shared by the
// sm_100a kernels of the GP stepper.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace gp5 {

// Complex element type per precision: double2 for complex128, float2 for complex64.
template <typename R> struct CT;
template <> struct CT<double> { using T = double2; };
template <> struct CT<float> { using T = float2; };

template <typename R> using cpx = typename CT<R>::T;

template <typename R> __host__ __device__ __forceinline__ cpx<R> mk(R re, R im) {
    cpx<R> v;
    v.x = re;
    v.y = im;
    return v;
}
template <typename V> __host__ __device__ __forceinline__ V cadd(V a, V b) {
    V r; r.x = a.x + b.x; r.y = a.y + b.y; return r;
}
template <typename V> __host__ __device__ __forceinline__ V csub(V a, V b) {
    V r; r.x = a.x - b.x; r.y = a.y - b.y; return r;
}
// complex64 sums and differences as one packed two-lane FP32 instruction (add/sub.rn.f32x2 of
// sm_100a, each lane rounded as the scalar operation is).  Default on: the complex64 step is
// issue-bound and measured 4.6% faster at 256^3 (every pass gained).  The packed forms are not
// contracted with a neighbouring multiply, so results differ from GP5_F32X2=0 in the last bits.
#ifndef GP5_F32X2
#define GP5_F32X2 1
#endif
#if GP5_F32X2
template <> __host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) {
#ifdef __CUDA_ARCH__
    unsigned long long x, y, d;
    asm("mov.b64 %0, {%1, %2};" : "=l"(x) : "f"(a.x), "f"(a.y));
    asm("mov.b64 %0, {%1, %2};" : "=l"(y) : "f"(b.x), "f"(b.y));
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(x), "l"(y));
    float2 r;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(d));
    return r;
#else
    return float2{a.x + b.x, a.y + b.y};
#endif
}
template <> __host__ __device__ __forceinline__ float2 csub(float2 a, float2 b) {
#ifdef __CUDA_ARCH__
    unsigned long long x, y, d;
    asm("mov.b64 %0, {%1, %2};" : "=l"(x) : "f"(a.x), "f"(a.y));
    asm("mov.b64 %0, {%1, %2};" : "=l"(y) : "f"(b.x), "f"(b.y));
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(x), "l"(y));
    float2 r;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(d));
    return r;
#else
    return float2{a.x - b.x, a.y - b.y};
#endif
}
#endif
// (a+ib)(c+id) = (ac - bd) + i(ad + bc), the order std::complex uses
template <typename V> __host__ __device__ __forceinline__ V cmul(V a, V b) {
    V r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
// a * conj(b)
template <typename V> __host__ __device__ __forceinline__ V cmulc(V a, V b) {
    V r; r.x = a.x * b.x + a.y * b.y; r.y = a.y * b.x - a.x * b.y; return r;
}
template <typename V, typename S> __host__ __device__ __forceinline__ V cscale(V a, S s) {
    V r; r.x = a.x * s; r.y = a.y * s; return r;
}
// multiply by -i (DIR=-1) or +i (DIR=+1)
template <int DIR, typename V> __host__ __device__ __forceinline__ V mul_i(V a) {
    V r;
    if (DIR < 0) { r.x = a.y; r.y = -a.x; }
    else { r.x = -a.y; r.y = a.x; }
    return r;
}
template <typename V> __host__ __device__ __forceinline__ V cconj(V a) {
    V r; r.x = a.x; r.y = -a.y; return r;
}

// ---- programmatic dependent launch ----------------------------------------------------
// Every kernel of the stepper path starts here.  The wait returns once the grid this launch
// depends on has completed and its writes are visible (at once when the launch has no
// programmatic dependency), so nothing below reads a predecessor's output early; the trigger
// then lets the next launch of the stream be scheduled while this grid drains.  The next
// grid starts only after every CTA of this one has triggered, i.e. is resident or done.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// ---- status words shared with the host ------------------------------------------------
enum DevStatus : unsigned { DS_OK = 0u, DS_NONFINITE = 1u, DS_TIMEOUT = 2u };

}  // namespace gp5
