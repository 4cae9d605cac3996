// pd_pack.cuh -- packed FP32 pair arithmetic (sm_100 f32x2: one instruction for two FP32
// operations, flush-to-zero as the FP32 force path) and compensated sums of pairs, shared by
// the packed force kernels.
#pragma once
#include <cuda_runtime.h>

namespace pd {
namespace pack {

// packed FP32 pairs (sm_100 f32x2): flush-to-zero as the rest of the FP32 force path
__device__ __forceinline__ unsigned long long pk(float2 v) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(v.x), "f"(v.y));
  return r;
}
__device__ __forceinline__ float2 upk(unsigned long long r) {
  float2 v;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(r));
  return v;
}
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
  unsigned long long d;
  asm("add.rn.ftz.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pk(a)), "l"(pk(b)));
  return upk(d);
}
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
  unsigned long long d;
  asm("sub.rn.ftz.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pk(a)), "l"(pk(b)));
  return upk(d);
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) {
  unsigned long long d;
  asm("mul.rn.ftz.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pk(a)), "l"(pk(b)));
  return upk(d);
}

// Kahan sum of pairs with the negated compensation n = -c: y = x + n, t = s + y,
// n = (s - t) + y, s = t (the value is s + n)
struct KSum2 {
  float2 s, n;
  __device__ __forceinline__ KSum2() : s(make_float2(0.f, 0.f)), n(make_float2(0.f, 0.f)) {}
  __device__ __forceinline__ void add(float2 x) {
    const float2 y = add2(x, n);
    const float2 t = add2(s, y);
    n = add2(sub2(s, t), y);
    s = t;
  }
  __device__ __forceinline__ float2 value() const { return add2(s, n); }
};

struct KSum1 {
  float s, n;
  __device__ __forceinline__ KSum1() : s(0.f), n(0.f) {}
  __device__ __forceinline__ void add(float x) {
    const float y = x + n;
    const float t = s + y;
    n = (s - t) + y;
    s = t;
  }
  __device__ __forceinline__ float value() const { return s + n; }
};

__device__ __forceinline__ float2 xy(const float4& v) { return make_float2(v.x, v.y); }

// a load of the bond stream: read once per phase, so it is marked as streaming (evict first)
// and leaves L2 to the neighbours' point records, which the gathers reuse. Measured on the
// 8M-point OSB block: step 8.90 -> 8.73 ms; 1M-point CMat block: 1.444 -> 1.407 ms.
template <typename T>
__device__ __forceinline__ T ld_stream(const T* p) {
  return __ldcs(p);
}

}  // namespace pack
}  // namespace pd
