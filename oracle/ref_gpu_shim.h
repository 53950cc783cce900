/*
 * ref_gpu_shim.h -- force-included (nvcc -include) ahead of the reference's GPU headers when
 * oracle/Makefile compiles them in place for sm_100a.  TEST INFRASTRUCTURE ONLY.
 *
 * The reference's warp reductions (src/Swift.h:46-50, src/Swift_gpu_col_major.h:40-44 and the
 * FP32 copies under test/k-32/FP32/) call the pre-Volta intrinsic __shfl_down, which CUDA 9+
 * no longer provides for sm_70 and newer.  Every such call sits in warp-uniform control flow
 * (a loop over width/32 chunks, or a branch on threadIdx.x / 32), so the full-mask
 * __shfl_down_sync is the same operation.  No reference line is changed.  The CUDA headers
 * that declare their own __shfl_down overloads come first, so the macro does not touch them.
 */
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#define __shfl_down(v, d) __shfl_down_sync(0xffffffffu, (v), (d))
