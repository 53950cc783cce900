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
