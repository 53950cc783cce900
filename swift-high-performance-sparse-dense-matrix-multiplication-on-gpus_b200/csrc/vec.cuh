// vec.cuh -- 16-byte vector loads/stores of the dense operands with conversion to the
// accumulator type, and vector reductions into C.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace swift {

template <class T> struct VecWidth { static constexpr int value = 16 / sizeof(T); };
// 32-byte vectors (sm_100 256-bit global loads / stores)
template <class T> struct WideWidth { static constexpr int value = 32 / sizeof(T); };

__device__ __forceinline__ void ld_nc_v8(const void *p, unsigned (&r)[8]) {
  asm volatile("ld.global.nc.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                 "=r"(r[6]), "=r"(r[7])
               : "l"(p));
}

__device__ __forceinline__ void st_cs_v8(void *p, const unsigned (&r)[8]) {
  asm volatile("st.global.cs.v8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(p), "r"(r[0]),
               "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
               : "memory");
}

template <class ACC, class T> __device__ __forceinline__ ACC to_acc(T x) { return (ACC)x; }
template <> __device__ __forceinline__ float to_acc<float, __nv_bfloat16>(__nv_bfloat16 x) { return __bfloat162float(x); }
template <> __device__ __forceinline__ float to_acc<float, __half>(__half x) { return __half2float(x); }

template <class T, class ACC> __device__ __forceinline__ T from_acc(ACC x) { return (T)x; }
template <> __device__ __forceinline__ __nv_bfloat16 from_acc<__nv_bfloat16, float>(float x) { return __float2bfloat16_rn(x); }
template <> __device__ __forceinline__ __half from_acc<__half, float>(float x) { return __float2half_rn(x); }

// Read-only load of VB elements (one 16-byte vector when VB * sizeof(T) == 16).
template <class T, class ACC, int VB>
__device__ __forceinline__ void vload(const T *__restrict__ p, ACC (&o)[VB]) {
  if constexpr (VB == 1) {
    o[0] = to_acc<ACC>(__ldg(p));
  } else if constexpr (sizeof(T) * VB == 32) {
    unsigned r[8];
    ld_nc_v8(p, r);
    const T *h = reinterpret_cast<const T *>(r);
#pragma unroll
    for (int i = 0; i < VB; ++i) o[i] = to_acc<ACC>(h[i]);
  } else if constexpr (sizeof(T) == 4 && VB == 4) {
    float4 f = __ldg(reinterpret_cast<const float4 *>(p));
    o[0] = f.x; o[1] = f.y; o[2] = f.z; o[3] = f.w;
  } else if constexpr (sizeof(T) == 8 && VB == 2) {
    double2 d = __ldg(reinterpret_cast<const double2 *>(p));
    o[0] = d.x; o[1] = d.y;
  } else {
    static_assert(sizeof(T) == 2 && VB == 8, "unsupported vector shape");
    uint4 u = __ldg(reinterpret_cast<const uint4 *>(p));
    const T *h = reinterpret_cast<const T *>(&u);
#pragma unroll
    for (int i = 0; i < 8; ++i) o[i] = to_acc<ACC>(h[i]);
  }
}

// Streaming store (evict-first): each C row is written once.
template <class T, class ACC, int VB>
__device__ __forceinline__ void vstore(T *__restrict__ p, const ACC (&a)[VB]) {
  if constexpr (VB == 1) {
    if constexpr (sizeof(T) >= 4) __stcs(p, from_acc<T>(a[0]));
    else *p = from_acc<T>(a[0]);
  } else if constexpr (sizeof(T) * VB == 32) {
    unsigned r[8];
    T *h = reinterpret_cast<T *>(r);
#pragma unroll
    for (int i = 0; i < VB; ++i) h[i] = from_acc<T>(a[i]);
    st_cs_v8(p, r);
  } else if constexpr (sizeof(T) == 4 && VB == 4) {
    __stcs(reinterpret_cast<float4 *>(p), make_float4(a[0], a[1], a[2], a[3]));
  } else if constexpr (sizeof(T) == 8 && VB == 2) {
    __stcs(reinterpret_cast<double2 *>(p), make_double2(a[0], a[1]));
  } else {
    static_assert(sizeof(T) == 2 && VB == 8, "unsupported vector shape");
    uint4 u;
    T *h = reinterpret_cast<T *>(&u);
#pragma unroll
    for (int i = 0; i < 8; ++i) h[i] = from_acc<T>(a[i]);
    __stcs(reinterpret_cast<uint4 *>(p), u);
  }
}

// acc += w * b over one vector.  FP32 pairs go through the packed two-lane FMA of sm_100
// (fma.rn.f32x2: each lane an IEEE fused multiply-add, so results equal the scalar form) to
// halve the FMA instructions per gathered element.
template <class ACC, int VB>
__device__ __forceinline__ void fma_vec(ACC (&acc)[VB], ACC w, const ACC (&b)[VB]) {
  if constexpr (sizeof(ACC) == 4 && VB % 2 == 0) {
    unsigned long long ww;
    asm("mov.b64 %0, {%1, %1};" : "=l"(ww) : "f"(w));
#pragma unroll
    for (int e = 0; e < VB; e += 2) {
      unsigned long long a2, b2;
      asm("mov.b64 %0, {%1, %2};" : "=l"(a2) : "f"(acc[e]), "f"(acc[e + 1]));
      asm("mov.b64 %0, {%1, %2};" : "=l"(b2) : "f"(b[e]), "f"(b[e + 1]));
      asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(a2) : "l"(ww), "l"(b2));
      asm("mov.b64 {%0, %1}, %2;" : "=f"(acc[e]), "=f"(acc[e + 1]) : "l"(a2));
    }
  } else {
#pragma unroll
    for (int e = 0; e < VB; ++e) acc[e] = fma(w, b[e], acc[e]);
  }
}

// One gathered B vector held until it is consumed.  FP32/FP64 keep the converted values;
// 16-bit types keep the raw packed words (half the registers while loads are in flight) and
// convert a pair at a time when accumulating.
template <class T, class ACC, int VB>
struct BVec {
  ACC v[VB];
  __device__ __forceinline__ void load(const T *p) { vload<T, ACC, VB>(p, v); }
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int e = 0; e < VB; ++e) v[e] = ACC(0);
  }
  template <bool PK>
  __device__ __forceinline__ void fma_into(ACC (&acc)[VB], ACC w) const {
    if constexpr (PK) {
      fma_vec<ACC, VB>(acc, w, v);
    } else {
#pragma unroll
      for (int e = 0; e < VB; ++e) acc[e] = fma(w, v[e], acc[e]);
    }
  }
};

template <class T> __device__ __forceinline__ float2 unpack2(unsigned u);
template <> __device__ __forceinline__ float2 unpack2<__nv_bfloat16>(unsigned u) {
  return make_float2(__uint_as_float(u << 16), __uint_as_float(u & 0xffff0000u));
}
template <> __device__ __forceinline__ float2 unpack2<__half>(unsigned u) {
  return __half22float2(*reinterpret_cast<const __half2 *>(&u));
}

template <class T, int VB>
struct BVec16 {
  static_assert(VB == 8 || VB == 16, "16-bit vectors of 16 or 32 bytes");
  unsigned u[VB / 2];
  __device__ __forceinline__ void load(const T *p) {
    if constexpr (VB == 16) {
      ld_nc_v8(p, u);
    } else {
      const uint4 q = __ldg(reinterpret_cast<const uint4 *>(p));
      u[0] = q.x; u[1] = q.y; u[2] = q.z; u[3] = q.w;
    }
  }
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int i = 0; i < VB / 2; ++i) u[i] = 0u;
  }
  template <bool PK>
  __device__ __forceinline__ void fma_into(float (&acc)[VB], float w) const {
#pragma unroll
    for (int i = 0; i < VB / 2; ++i) {
      const float2 f = unpack2<T>(u[i]);
      if constexpr (PK) {
        const float b[2] = {f.x, f.y};
        float a[2] = {acc[2 * i], acc[2 * i + 1]};
        fma_vec<float, 2>(a, w, b);
        acc[2 * i] = a[0];
        acc[2 * i + 1] = a[1];
      } else {
        acc[2 * i] = fma(w, f.x, acc[2 * i]);
        acc[2 * i + 1] = fma(w, f.y, acc[2 * i + 1]);
      }
    }
  }
};
template <int VB> struct BVec<__nv_bfloat16, float, VB> : BVec16<__nv_bfloat16, VB> {};
template <int VB> struct BVec<__half, float, VB> : BVec16<__half, VB> {};
template <> struct BVec<__nv_bfloat16, float, 1> {
  float v[1];
  __device__ __forceinline__ void load(const __nv_bfloat16 *p) { v[0] = __bfloat162float(p[0]); }
  __device__ __forceinline__ void zero() { v[0] = 0.f; }
  template <bool PK> __device__ __forceinline__ void fma_into(float (&acc)[1], float w) const {
    acc[0] = fma(w, v[0], acc[0]);
  }
};
template <> struct BVec<__half, float, 1> {
  float v[1];
  __device__ __forceinline__ void load(const __half *p) { v[0] = __half2float(p[0]); }
  __device__ __forceinline__ void zero() { v[0] = 0.f; }
  template <bool PK> __device__ __forceinline__ void fma_into(float (&acc)[1], float w) const {
    acc[0] = fma(w, v[0], acc[0]);
  }
};

// C += a (vector reduction in L2).  FP32: one 16-byte float4 atomic (sm_90+); FP64: scalar.
template <class T, class ACC, int VB>
__device__ __forceinline__ void vatomic_add(T *__restrict__ p, const ACC (&a)[VB]) {
  if constexpr (sizeof(T) == 4 && VB == 4) {
    atomicAdd(reinterpret_cast<float4 *>(p), make_float4(a[0], a[1], a[2], a[3]));
  } else {
#pragma unroll
    for (int i = 0; i < VB; ++i) atomicAdd(p + i, (T)a[i]);
  }
}

}  // namespace swift
