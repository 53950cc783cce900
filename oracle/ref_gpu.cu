/*
 * ref_gpu.cu -- C entry points over the REFERENCE's own GPU SpMM wrappers, compiled in place
 * from the reference checkout for sm_100a by oracle/Makefile into oracle/_ref/.  TEST AND
 * MEASUREMENT INFRASTRUCTURE ONLY: it times the reference's kernels on the same GPU as this
 * library, as a context figure beside the library's own; nothing in the package loads it.
 * No reference source is copied here: the headers are included from the checkout
 * (-I<ref>/test/k-32/FP32 or -I<ref>/src) with ref_gpu_shim.h force-included.
 *
 *   variant 0  Swift_GPU    src/Swift.h:184            (column-major B and C)
 *   variant 1  Swift_gpu1   src/Swift_gpu_col_major.h:171
 *   variant 2  Swift_gpu2   src/Swift_gpu_row_major.h:136   (row-major B and C)
 *   variant 3  Swift_GPU_3  src/Swift_3.h:216
 *   variant 4  Swift_GPU_4  src/Swift_4.h:305          (after row_idx_sort)
 *
 * Each wrapper uploads the format and B, runs its kernels between two CUDA events on the
 * legacy stream, downloads C and checks it against `golden` (|C - golden| <= 1e-2,
 * src/auxiliary.h:156-165), setting its time to -1 when the check fails.
 *
 * Only inputs whose launches were read to stay in bounds are accepted (anything else returns
 * REFGPU_REFUSED without touching the GPU):
 *   - width a positive multiple of 32, tilenum > 0 and reside_nnz > 0: the branch every
 *     wrapper takes for the R-MAT workloads.  The FP32 Swift_GPU_3 / Swift_GPU_4 branch for
 *     reside_nnz == 0 sizes its grid with (width + 32) / 32 (test/k-32/FP32/Swift_3.h:369,
 *     Swift_4.h:486), one 32-column chunk past B and C;
 *   - Swift_GPU_4 only in FP32 and only when tilenum % 8 == 0: its kernel calls
 *     __syncthreads() inside `if (rid < tilenum)` (src/Swift_4.h:33-75), which is uniform
 *     across the block only when every block holds 8 tiles.  The FP64 launch passes
 *     32*8*(sizeof(int)+sizeof(double)) = 3072 bytes of dynamic shared memory
 *     (src/Swift_4.h:433) while the kernel addresses 4096 (two int arrays of 256, then 256
 *     doubles at byte 2048, src/Swift_4.h:20-23), so FP64 Swift_GPU_4 is never run.
 */
#include <cuda_runtime.h>
#include <sys/time.h>  // the reference's driver includes it before its headers (src/main.cu:3)

#include "coo2csc.h"  // auxiliary.h (ResultVerify, dense_mtx2dense_mtx_spmm), format.h
#include "Swift_gpu_row_major.h"  // defines CHECK_CUDA_ERROR used by the other wrappers
#include "Swift_gpu_col_major.h"
#include "Swift.h"
#include "Swift_3.h"
#include "Swift_4.h"

#include "swift_oracle.h"

#if defined(REF_FP32)
typedef float ref_t;
typedef float gflops_t;  // test/k-32/FP32/Swift.h:219
typedef or_slide_f32 or_slide_t;
#define REFN(name) name##_f32
#elif defined(REF_FP64)
typedef double ref_t;
typedef double gflops_t;  // src/Swift.h:186
typedef or_slide_f64 or_slide_t;
#define REFN(name) name##_f64
#else
#error "define REF_FP32 or REF_FP64"
#endif

enum { REFGPU_OK = 0, REFGPU_CHECK_FAILED = 1, REFGPU_REFUSED = 2, REFGPU_CUDA_ERROR = 3 };

extern "C" {

/* Runs one reference wrapper on the format `s` (arrays as the reference's preprocessing
 * leaves them; variant 4 needs row_idx_sort's sortrowidx, val_position and val_offset).
 * B: sorted dense operand (column-major colA x width for variants 0, 1, 3, 4; row-major for
 * variant 2); C: result in the same layout; golden: row-major rowA x width.  *ms receives the
 * wrapper's own CUDA-event time (kernels only). */
__attribute__((visibility("default"))) int REFN(refgpu_spmm)(int variant, const or_slide_t *s, int rowA,
                                                            int colA, int width, int nnz, ref_t *B, ref_t *C,
                                                            ref_t *golden, float *ms) {
  if (!s || !B || !C || !golden || !ms || variant < 0 || variant > 4) return REFGPU_REFUSED;
  if (width <= 0 || width % 32 != 0 || s->tilenum <= 0 || s->reside_nnz <= 0) return REFGPU_REFUSED;
#if defined(REF_FP64)
  if (variant == 4) return REFGPU_REFUSED;
#endif
  if (variant == 4 && (s->tilenum % 8 != 0 || !s->val_position || !s->val_offset)) return REFGPU_REFUSED;
  if (variant != 1 && (!s->colorblk || s->numblk <= 0)) return REFGPU_REFUSED;

  slide_matrix m;
  memset(&m, 0, sizeof(m));
  m.sortval = s->sortval;
  m.sortrowidx = s->sortrowidx;
  m.tile_ptr = s->tile_ptr;
  m.tile_len = s->tile_len;
  m.tile_colidx = s->tile_colidx;
  m.tile_tall = s->tile_tall;
  m.tile_format = s->tile_format;
  m.countrow = s->countrow;
  m.segmentoffset = s->segmentoffset;
  m.sortrowindex = s->sortrowindex;
  m.val_position = s->val_position;
  m.val_offset = s->val_offset;
  m.tilenum = s->tilenum;
  m.segsum = s->segsum;
  m.regular_nnz = s->regular_nnz;
  m.reside_col = s->reside_col;
  m.reside_nnz = s->reside_nnz;
  m.reside_cscptr = s->reside_cscptr;
  m.reside_cscrowidx = s->reside_cscrowidx;
  m.reside_val = s->reside_val;
  m.numblk = s->numblk;
  m.colorblk = s->colorblk;
  m.blkstart = s->blkstart;
  m.blkstop = s->blkstop;
  m.blkptr = s->blkptr;

  char name[] = "synthetic";
  float t = 0.f;
  gflops_t gf = 0;
  cudaGetLastError();
  switch (variant) {
    case 0: Swift_GPU(name, t, gf, &m, rowA, colA, width, nnz, B, C, golden); break;
    case 1: Swift_gpu1(name, t, gf, &m, rowA, colA, width, nnz, B, C, golden); break;
    case 2: Swift_gpu2(name, t, gf, &m, rowA, colA, width, nnz, B, C, golden); break;
    case 3: Swift_GPU_3(name, t, gf, &m, rowA, colA, width, nnz, B, C, golden); break;
    default: Swift_GPU_4(name, t, gf, &m, rowA, colA, width, nnz, B, C, golden); break;
  }
  if (cudaDeviceSynchronize() != cudaSuccess || cudaGetLastError() != cudaSuccess) return REFGPU_CUDA_ERROR;
  *ms = t;
  return t < 0 ? REFGPU_CHECK_FAILED : REFGPU_OK;
}

}  // extern "C"
