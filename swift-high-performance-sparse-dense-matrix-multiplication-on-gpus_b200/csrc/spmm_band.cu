// spmm_band.cu -- dense diagonal tiles (the band engine).
//
// Matrices whose nonzeros crowd the diagonal (banded stencils, the |i-j| < 32 band of the
// precision workload) waste the row walk's per-nonzero B-row gather: neighbouring rows gather
// almost the same B rows.  The band engine splits A once per plan:
//   * tiles: for every 8-row group g, a dense 8 x TW tile of the columns
//     [8g - W, 8g - W + TW), TW = 8 + 2W rounded up to 4 (values only, zeros where A has none);
//   * rest:  the nonzeros outside their group's tile, as a CSR operand for the row walk.
// A product runs the row walk over the rest (writing every C row), then the tile kernel adds
// the tiles' product: persistent blocks, each over a contiguous range of 64-row groups and one
// 128-column slice, keep the B rows their tiles touch in a shared-memory ring of 64-row chunks
// filled by TMA tile loads one group ahead (consecutive groups share all but 64 of those rows),
// with the groups' tile values double-buffered by bulk copies.  FP32 B: each warp keeps the
// 8 x 128 slice of its C rows in registers, so every B row read from shared memory feeds eight
// rows' FMAs (a loaded B vector is used 8 times, a loaded tile vector 4 times).  BF16 / FP16 B:
// the tiles run on the tensor cores (mma.sync m16n8k16, FP32 accumulation; A's FP32 values
// split into hi + lo parts of B's type after a power-of-two row scale), with the C tile moved
// by TMA in and out of shared memory.
//
// The half-width W is chosen from the plan's distance profile (nonzeros per |col - row|, one
// GPU pass): the W that saves the most gathered rows for the dense work it adds, if it saves at
// least a twentieth of the walk's gathers.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <type_traits>

#include "common.cuh"
#include "vec.cuh"

namespace swift {

namespace {

constexpr int kGroup = 8;          // rows per tile (one warp)
constexpr int kCtaRows = 64;       // rows per block (eight warps)
constexpr int kSlice = 128;        // dense columns per block (32 lanes x 4)
constexpr int kChunk = 64;         // B rows per TMA load (one ring slot)
constexpr int kMaxDist = 128;      // |col - row| profiled up to this distance
constexpr int kWidths[] = {3, 7, 15, 31, 47, 63};

__device__ int g_band_timeout;     // set when a block's copy wait ran out

constexpr int tile_width(int w) { return (kGroup + 2 * w + 3) / 4 * 4; }
constexpr int panel_rows(int tw) { return kCtaRows - kGroup + tw; }

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Bounded wait on phase `parity` of an mbarrier: about two seconds of SM clock at most.
__device__ __forceinline__ bool wait_phase(uint32_t bar, uint32_t parity) {
  const long long t0 = clock64();
  while (true) {
    uint32_t ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
    if (ok) return true;
    if (clock64() - t0 > 4000000000LL) return false;
  }
}

// |col - row| histogram (distances above kMaxDist are not counted).
__global__ void band_profile_kernel(const int *__restrict__ rowptr, const int *__restrict__ colidx, int M,
                                    unsigned long long *__restrict__ hist) {
  __shared__ unsigned int sh[kMaxDist + 1];
  for (int t = threadIdx.x; t <= kMaxDist; t += blockDim.x) sh[t] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < M; i += (gridDim.x * blockDim.x) >> 5) {
    const int e1 = __ldg(rowptr + i + 1);
    for (int e = __ldg(rowptr + i) + lane; e < e1; e += 32) {
      const int d = abs(__ldg(colidx + e) - i);
      if (d <= kMaxDist) atomicAdd(&sh[d], 1u);
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t <= kMaxDist; t += blockDim.x)
    if (sh[t]) atomicAdd(hist + t, (unsigned long long)sh[t]);
}

// Per row: nonzeros outside the row's group tile.
__global__ void band_count_kernel(const int *__restrict__ rowptr, const int *__restrict__ colidx, int M, int W,
                                  int TW, int *__restrict__ rest_cnt) {
  const int lane = threadIdx.x & 31;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < M; i += (gridDim.x * blockDim.x) >> 5) {
    const int c0 = (i & ~(kGroup - 1)) - W;
    const int e0 = __ldg(rowptr + i), e1 = __ldg(rowptr + i + 1);
    int cnt = 0;
    for (int b = e0; b < e1; b += 32) {
      const int e = b + lane;
      bool out = false;
      if (e < e1) {
        const int j = __ldg(colidx + e);
        out = j < c0 || j >= c0 + TW;
      }
      cnt += __popc(__ballot_sync(0xffffffffu, out));
    }
    if (lane == 0) rest_cnt[i] = cnt;
  }
}

// Per row: tile entries into the tiles, the others (in row order) into the rest CSR; dst[e]
// records where nonzero e went (>= 0: rest position, < 0: -1 - tile position) for value updates.
template <class TV>
__global__ void band_split_kernel(const int *__restrict__ rowptr, const int *__restrict__ colidx,
                                  const TV *__restrict__ val, int M, int W, int TW, const int *__restrict__ rest_ptr,
                                  int *__restrict__ rest_idx, TV *__restrict__ rest_val, float *__restrict__ tiles,
                                  int *__restrict__ dst) {
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < M; i += (gridDim.x * blockDim.x) >> 5) {
    const int c0 = (i & ~(kGroup - 1)) - W;
    const int e0 = __ldg(rowptr + i), e1 = __ldg(rowptr + i + 1);
    int base = __ldg(rest_ptr + i);
    for (int b = e0; b < e1; b += 32) {
      const int e = b + lane;
      bool out = false;
      int j = 0;
      if (e < e1) {
        j = __ldg(colidx + e);
        out = j < c0 || j >= c0 + TW;
      }
      const unsigned m = __ballot_sync(0xffffffffu, out);
      if (e < e1) {
        if (out) {
          const int pos = base + __popc(m & below);
          rest_idx[pos] = j;
          rest_val[pos] = val[e];
          dst[e] = pos;
        } else {
          const int tpos = i * TW + (j - c0);
          tiles[tpos] = (float)val[e];
          dst[e] = -1 - tpos;
        }
      }
      base += __popc(m);
    }
  }
}

// New values for the fixed pattern: scatter through dst.
template <class TV>
__global__ void band_refill_kernel(const TV *__restrict__ val, int64_t nnz, const int *__restrict__ dst,
                                   TV *__restrict__ rest_val, float *__restrict__ tiles) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += (int64_t)gridDim.x * blockDim.x) {
    const int d = dst[e];
    if (d >= 0) rest_val[d] = val[e];
    else tiles[-1 - d] = (float)val[e];
  }
}

// C[rows, this 128-column slice] += tiles x B, one persistent block per contiguous range of
// 64-row groups.  The B rows a group's tiles touch (64 + TW - 8 of them, starting W rows above
// the group) overlap the next group's by TW - 8 rows, so B lives in a ring of 64-row chunks:
// each group adds one chunk.  Chunk c holds B rows [rbase + 64c, rbase + 64c + 64) in slot
// c % NR, NR = (chunks one group touches) + 1, so the chunk of the group after next loads while
// this group computes; the groups' tile values are double-buffered the same way.  TMA tile
// loads fill the ring (rows outside B are zero-filled), bulk copies the values, one mbarrier
// per slot.  The old C rows (the rest walk's result) are loaded into registers before the
// waits.  Waits are bounded; a block that gives up sets g_band_timeout and leaves.
template <int TW, int MINB>
__global__ void __launch_bounds__(256, MINB) band_tile_kernel(const __grid_constant__ CUtensorMap bmap,
                                                              const float *__restrict__ tiles, int M, int N, int W,
                                                              int ngroups, int per_block, float *__restrict__ C,
                                                              int64_t ldc) {
  constexpr int PR = panel_rows(TW);
  constexpr int NCH = (PR + kChunk - 1) / kChunk;
  constexpr int NR = NCH + 1;
  constexpr int RING_ROWS = NR * kChunk;
  constexpr uint32_t CHUNK_BYTES = (uint32_t)kChunk * kSlice * 4;
  constexpr uint32_t VAL_BYTES = (uint32_t)kCtaRows * TW * 4;
  extern __shared__ __align__(1024) unsigned char sm[];
  float *ring = reinterpret_cast<float *>(sm);
  float *vals = reinterpret_cast<float *>(sm + NR * CHUNK_BYTES);
  uint64_t *bar = reinterpret_cast<uint64_t *>(sm + NR * CHUNK_BYTES + 2 * VAL_BYTES);  // NR chunks, 2 values
  const int g0 = blockIdx.x * per_block;
  const int g1 = min(g0 + per_block, ngroups);
  if (g0 >= g1) return;
  const int nb = g1 - g0, nchunks = nb - 1 + NCH;
  const int col0 = blockIdx.y * kSlice;
  const int rbase = g0 * kCtaRows - W;
  int issued_chunks = 0, issued_vals = 0;  // producer (thread 0) state
  auto issue_chunk = [&](int c) {
    const uint32_t b = smem_addr(bar + c % NR);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(CHUNK_BYTES) : "memory");
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(smem_addr(ring + (size_t)(c % NR) * kChunk * kSlice)), "l"(reinterpret_cast<uint64_t>(&bmap)),
        "r"(col0), "r"(rbase + kChunk * c), "r"(b)
        : "memory");
    issued_chunks = c + 1;
  };
  auto issue_vals = [&](int k) {
    const uint32_t b = smem_addr(bar + NR + (k & 1));
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(VAL_BYTES) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_addr(vals + (size_t)(k & 1) * kCtaRows * TW)),
                 "l"(tiles + (size_t)(g0 + k) * kCtaRows * TW), "r"(VAL_BYTES), "r"(b)
                 : "memory");
    issued_vals = k + 1;
  };
  if (threadIdx.x == 0) {
    for (int s = 0; s < NR + 2; ++s) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar + s)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (int c = 0; c < NR && c < nchunks; ++c) issue_chunk(c);
    for (int k = 0; k < 2 && k < nb; ++k) issue_vals(k);
  }
  __syncthreads();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int col = col0 + lane * 4;
  for (int k = 0; k < nb; ++k) {
    const int rw = (g0 + k) * kCtaRows + kGroup * w;  // first C row of this warp
    // the rest walk's C rows, in their own registers so that no FMA waits on them
    float4 old[kGroup];
#pragma unroll
    for (int r = 0; r < kGroup; ++r)
      old[r] = (rw + r < M && col < N) ? __ldcs(reinterpret_cast<const float4 *>(C + (int64_t)(rw + r) * ldc + col))
                                       : make_float4(0.f, 0.f, 0.f, 0.f);
    float acc[kGroup][4];
#pragma unroll
    for (int r = 0; r < kGroup; ++r) acc[r][0] = acc[r][1] = acc[r][2] = acc[r][3] = 0.f;
    bool bad = false;
#pragma unroll
    for (int j = 0; j < NCH; ++j) bad |= !wait_phase(smem_addr(bar + (k + j) % NR), (uint32_t)(((k + j) / NR) & 1));
    bad |= !wait_phase(smem_addr(bar + NR + (k & 1)), (uint32_t)((k >> 1) & 1));
    if (__syncthreads_or(bad)) {
      if (threadIdx.x == 0) {
        atomicExch(&g_band_timeout, 1);
        // give the copies still in flight a bounded chance to land before the block leaves
        for (int c = max(0, issued_chunks - NR); c < issued_chunks; ++c)
          wait_phase(smem_addr(bar + c % NR), (uint32_t)((c / NR) & 1));
        for (int v = max(0, issued_vals - 2); v < issued_vals; ++v)
          wait_phase(smem_addr(bar + NR + (v & 1)), (uint32_t)((v >> 1) & 1));
      }
      return;
    }
    const int rb = (k % NR) * kChunk + kGroup * w;  // ring row of this warp's tile column 0
    const float *E = vals + (size_t)(k & 1) * kCtaRows * TW + (size_t)(kGroup * w) * TW;
#pragma unroll 2
    for (int c = 0; c < TW; c += 4) {
      int rr = rb + c;
      if (rr >= RING_ROWS) rr -= RING_ROWS;  // four rows never straddle the wrap (all multiples of 4)
      const float *bp = ring + (size_t)rr * kSlice + lane * 4;
      float bv[4][4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float4 f = *reinterpret_cast<const float4 *>(bp + q * kSlice);
        bv[q][0] = f.x; bv[q][1] = f.y; bv[q][2] = f.z; bv[q][3] = f.w;
      }
      float4 v[kGroup];
#pragma unroll
      for (int r = 0; r < kGroup; ++r) v[r] = *reinterpret_cast<const float4 *>(E + r * TW + c);
      // rows inner: consecutive FMAs update different accumulators
#pragma unroll
      for (int r = 0; r < kGroup; ++r) fma_vec<float, 4>(acc[r], v[r].x, bv[0]);
#pragma unroll
      for (int r = 0; r < kGroup; ++r) fma_vec<float, 4>(acc[r], v[r].y, bv[1]);
#pragma unroll
      for (int r = 0; r < kGroup; ++r) fma_vec<float, 4>(acc[r], v[r].z, bv[2]);
#pragma unroll
      for (int r = 0; r < kGroup; ++r) fma_vec<float, 4>(acc[r], v[r].w, bv[3]);
    }
    if (col < N) {
#pragma unroll
      for (int r = 0; r < kGroup; ++r)
        if (rw + r < M)
          __stcs(reinterpret_cast<float4 *>(C + (int64_t)(rw + r) * ldc + col),
                 make_float4(acc[r][0] + old[r].x, acc[r][1] + old[r].y, acc[r][2] + old[r].z, acc[r][3] + old[r].w));
    }
    __syncthreads();  // chunk k's slot and value slot k & 1 are free again
    if (threadIdx.x == 0) {
      if (k + NR < nchunks) issue_chunk(k + NR);
      if (k + 2 < nb) issue_vals(k + 2);
    }
  }
}

// ---------------------------------------------------------------- tensor-core tiles (16-bit B)
// For BF16 and FP16 B the tiles run on the tensor cores.  A 16-row group h pairs the 8-row tiles
// 2h and 2h + 1 in one 16 x TWM window starting at column 16h - W (tile 2h at window columns
// [0, TW), tile 2h + 1 at [8, 8 + TW); TWM = 8 + TW rounded up to 16), multiplied with mma.sync
// m16n8k16 (16-bit inputs of B's type, FP32 accumulation) against the B rows of the window.
// Each FP32 tile value, first scaled by its row's power of two 2^e (e puts the row's largest
// magnitude in [2^13, 2^14): no FP16 overflow, and small values keep their bits), is split into
// hi + lo parts of B's type (hi = the value rounded, lo = the remainder rounded), so A keeps
// about 16 (BF16) or 22 (FP16) significant bits; the epilogue multiplies each row's sum by
// 2^-e, which is exact.
//
// The window values are stored in the mma's A-fragment order: per 64-row block, per 16-row group
// (4), per 16-column k-step (KS = TWM / 16), per part (hi, lo), 32 lanes x 16 bytes -- lane
// l = 4g + t holds rows g and g + 8 at columns 2t, 2t + 1, 2t + 8, 2t + 9 of the k-step -- then
// the block's 64 row factors 2^-e.  One block's values are one contiguous bulk copy, and each
// lane reads its fragment with one conflict-free 16-byte shared load.
constexpr int mma_width(int tw) { return (kGroup + tw + 15) / 16 * 16; }  // TWM
constexpr int kFragBytes = 32 * 16;                                      // one 16 x 16 fragment
constexpr int mma_block_bytes(int ks) { return 4 * ks * 2 * kFragBytes + kCtaRows * 4; }

template <class T>
__device__ __forceinline__ T to16(float x);
template <> __device__ __forceinline__ __nv_bfloat16 to16<__nv_bfloat16>(float x) { return __float2bfloat16_rn(x); }
template <> __device__ __forceinline__ __half to16<__half>(float x) { return __float2half_rn(x); }
template <class T>
__device__ __forceinline__ float from16(T x);
template <> __device__ __forceinline__ float from16<__nv_bfloat16>(__nv_bfloat16 x) { return __bfloat162float(x); }
template <> __device__ __forceinline__ float from16<__half>(__half x) { return __half2float(x); }
template <class T>
__device__ __forceinline__ uint32_t pack2(float a, float b);
template <> __device__ __forceinline__ uint32_t pack2<__nv_bfloat16>(float a, float b) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t *>(&v);
}
template <> __device__ __forceinline__ uint32_t pack2<__half>(float a, float b) {
  const __half2 v = __floats2half2_rn(a, b);
  return *reinterpret_cast<const uint32_t *>(&v);
}

__device__ __forceinline__ float pow2f(int e) { return __int_as_float((127 + e) << 23); }  // e in [-126, 127]

// Per row: e with the row's largest |tile value| x 2^e in [2^13, 2^14) (0 for an all-zero row),
// read off the IEEE exponent field and clamped so that 2^e and 2^-e stay normal.
__global__ void band_row_exp_kernel(const float *__restrict__ tiles, int64_t rows, int TW, int *__restrict__ rexp) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x) {
    float m = 0.f;
    for (int c = 0; c < TW; ++c) m = fmaxf(m, fabsf(tiles[r * TW + c]));
    int e = 0;
    if (m > 0.f) {
      const int ex = (__float_as_int(m) >> 23) & 0xff;  // m in [2^(ex-127), 2^(ex-126)); 0 for subnormals
      e = min(126, max(-126, 140 - ex));                 // 2^(ex - 127 + e) = 2^13
    }
    rexp[r] = e;
  }
}

template <class T>
__global__ void band_mma_fill_kernel(const float *__restrict__ tiles, const int *__restrict__ rexp, int nblocks,
                                     int TW, int KS, unsigned char *__restrict__ frags) {
  const int64_t total = (int64_t)nblocks * 4 * KS * 32;
  const int64_t bb = mma_block_bytes(KS);
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int lane = (int)(e & 31);
    const int64_t q = e >> 5;  // (block, group, k-step)
    const int s = (int)(q % KS);
    const int64_t bg = q / KS;  // block * 4 + group
    const int64_t blk = bg >> 2;
    const int g = lane >> 2, t = lane & 3;
    const int64_t r0 = bg * 16 + g;  // rows r0 (tile 2h, window column = tile column) and r0 + 8
    const float sc[2] = {pow2f(rexp[r0]), pow2f(rexp[r0 + 8])};
    T hi[8], lo[8];
#pragma unroll
    for (int x = 0; x < 8; ++x) {
      // element order of the fragment: (r0, c) (r0, c+1) (r0+8, c) (r0+8, c+1) then c + 8
      const int c = 16 * s + 2 * t + (x & 1) + ((x & 4) ? 8 : 0);
      const int h = (x & 2) ? 1 : 0;
      const int tc = c - h * kGroup;
      const float v = (tc >= 0 && tc < TW) ? tiles[(r0 + 8 * h) * TW + tc] * sc[h] : 0.f;
      hi[x] = to16<T>(v);
      lo[x] = to16<T>(v - from16<T>(hi[x]));
    }
    uint4 *out = reinterpret_cast<uint4 *>(frags + blk * bb) + (q - blk * 4 * KS) * 64 + lane;
    out[0] = *reinterpret_cast<const uint4 *>(hi);
    out[32] = *reinterpret_cast<const uint4 *>(lo);
    if (s == 0 && lane < 16) {  // the row factors 2^-e of this group's 16 rows
      float *inv = reinterpret_cast<float *>(frags + blk * bb + 4 * KS * 2 * kFragBytes);
      inv[(bg & 3) * 16 + lane] = pow2f(-rexp[bg * 16 + lane]);
    }
  }
}

__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3) : "r"(addr) : "memory");
}
__device__ __forceinline__ void ldsm_x4_trans(uint32_t addr, uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0, %1, %2, %3}, [%4];"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3) : "r"(addr) : "memory");
}
__device__ __forceinline__ void stsm_x4(uint32_t addr, uint32_t r0, uint32_t r1, uint32_t r2, uint32_t r3) {
  asm volatile("stmatrix.sync.aligned.m8n8.x4.shared.b16 [%0], {%1, %2, %3, %4};"
               ::"r"(addr), "r"(r0), "r"(r1), "r"(r2), "r"(r3) : "memory");
}

// acc += A (16 x 16, row-major fragment) x B (16 x 8, column fragment), 16-bit in, FP32 accumulation
template <class T>
__device__ __forceinline__ void mma16(float (&acc)[4], const uint4 &a, uint32_t b0, uint32_t b1) {
  if constexpr (std::is_same<T, __nv_bfloat16>::value) {
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
                 "{%0, %1, %2, %3};"
                 : "+f"(acc[0]), "+f"(acc[1]), "+f"(acc[2]), "+f"(acc[3])
                 : "r"(a.x), "r"(a.y), "r"(a.z), "r"(a.w), "r"(b0), "r"(b1));
  } else {
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
                 "{%0, %1, %2, %3};"
                 : "+f"(acc[0]), "+f"(acc[1]), "+f"(acc[2]), "+f"(acc[3])
                 : "r"(a.x), "r"(a.y), "r"(a.z), "r"(a.w), "r"(b0), "r"(b1));
  }
}

// C[rows, this 128-column slice] += tiles x B on the tensor cores; the same persistent walk as
// band_tile_kernel (ring of 64-row B chunks one group ahead, values double-buffered, bounded
// waits).  Each B chunk arrives as two 64-column TMA boxes with the 128-byte swizzle: 16-byte
// unit u of ring row r sits at unit u ^ (r & 7) of its 128-byte row, so the eight row addresses
// of an ldmatrix hit eight different bank groups.  Warp w computes the 16-row group w & 3 over
// the 64 columns (w >> 2): eight n-tiles, each one mma per part and k-step.  The group's C tile
// (the rest walk's result) comes in by TMA, in the same swizzled layout, while the group is
// computed; the epilogue reads it with ldmatrix (which yields the accumulator's fragment layout),
// adds, writes the sums back with stmatrix, and one TMA store writes the tile out -- eight
// shared-memory wavefronts per warp and group instead of 32-bit global accesses spread over
// eight rows each.  The tile is single-buffered: the next group's C load is issued once the
// store has read it.
template <class T, int TW, int MINB>
__global__ void __launch_bounds__(256, MINB) band_mma_kernel(const __grid_constant__ CUtensorMap bmap,
                                                             const __grid_constant__ CUtensorMap cmap,
                                                             const unsigned char *__restrict__ frags, int W,
                                                             int ngroups, int per_block) {
  constexpr int TWM = mma_width(TW);
  constexpr int KS = TWM / 16;
  constexpr int NCH = (kCtaRows - 16 + TWM + kChunk - 1) / kChunk;  // chunks one block's windows touch
  constexpr int NR = NCH + 1;
  constexpr int RING_ROWS = NR * kChunk;
  constexpr uint32_t HALF_BYTES = (uint32_t)kChunk * 128;             // 64 rows x 64 16-bit columns
  constexpr uint32_t CHUNK_BYTES = 2 * HALF_BYTES;
  constexpr uint32_t VAL_BYTES = (uint32_t)mma_block_bytes(KS);
  extern __shared__ unsigned char sm_raw[];
  // the 128-byte swizzle repeats every 1024 bytes: align the ring and the C tile to that
  unsigned char *sm = sm_raw + ((1024u - (smem_addr(sm_raw) & 1023u)) & 1023u);
  unsigned char *ring = sm;
  unsigned char *ctile = sm + NR * CHUNK_BYTES;
  unsigned char *vals = ctile + CHUNK_BYTES;
  uint64_t *bar = reinterpret_cast<uint64_t *>(vals + 2 * VAL_BYTES);  // NR chunks, 2 values, C tile
  const int g0 = blockIdx.x * per_block;
  const int g1 = min(g0 + per_block, ngroups);
  if (g0 >= g1) return;
  const int nb = g1 - g0, nchunks = nb - 1 + NCH;
  const int col0 = blockIdx.y * kSlice;
  const int rbase = g0 * kCtaRows - W;
  const uint64_t bmap_p = reinterpret_cast<uint64_t>(&bmap), cmap_p = reinterpret_cast<uint64_t>(&cmap);
  int issued_chunks = 0, issued_vals = 0, issued_c = 0;  // producer (thread 0) state
  auto issue_chunk = [&](int c) {
    const uint32_t b = smem_addr(bar + c % NR);
    const uint32_t dst = smem_addr(ring + (size_t)(c % NR) * CHUNK_BYTES);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(CHUNK_BYTES) : "memory");
#pragma unroll
    for (int hf = 0; hf < 2; ++hf)
      asm volatile(
          "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
          "[%4];" ::"r"(dst + hf * HALF_BYTES),
          "l"(bmap_p), "r"(col0 + 64 * hf), "r"(rbase + kChunk * c), "r"(b)
          : "memory");
    issued_chunks = c + 1;
  };
  auto issue_vals = [&](int k) {
    const uint32_t b = smem_addr(bar + NR + (k & 1));
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(VAL_BYTES) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_addr(vals + (size_t)(k & 1) * VAL_BYTES)),
                 "l"(frags + (size_t)(g0 + k) * VAL_BYTES), "r"(VAL_BYTES), "r"(b)
                 : "memory");
    issued_vals = k + 1;
  };
  auto issue_c = [&](int k) {  // the rest walk's C rows of group k into the C tile
    const uint32_t b = smem_addr(bar + NR + 2);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(CHUNK_BYTES) : "memory");
#pragma unroll
    for (int hf = 0; hf < 2; ++hf)
      asm volatile(
          "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
          "[%4];" ::"r"(smem_addr(ctile) + hf * HALF_BYTES),
          "l"(cmap_p), "r"(col0 + 64 * hf), "r"((g0 + k) * kCtaRows), "r"(b)
          : "memory");
    issued_c = k + 1;
  };
  if (threadIdx.x == 0) {
    for (int s = 0; s < NR + 3; ++s) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar + s)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (int c = 0; c < NR && c < nchunks; ++c) issue_chunk(c);
    for (int k = 0; k < 2 && k < nb; ++k) issue_vals(k);
    issue_c(0);
  }
  __syncthreads();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int grp = w & 3, nh = w >> 2;
  const int g = lane >> 2;
  // ldmatrix / stmatrix addresses: lanes 0-15 give rows 0-15 of n-tile 2jj, lanes 16-31 of 2jj + 1
  const int lrow = lane & 15, lunit = lane >> 4;
  const uint32_t ring_s = smem_addr(ring) + nh * HALF_BYTES;
  const int crow = 16 * grp + lrow;  // C tile row of this lane's address
  const uint32_t crow_s = smem_addr(ctile) + nh * HALF_BYTES + (uint32_t)crow * 128;
  bool timed_out = false;
  for (int k = 0; k < nb; ++k) {
    float acc[8][4];
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
    bool bad = false;
#pragma unroll
    for (int j = 0; j < NCH; ++j) bad |= !wait_phase(smem_addr(bar + (k + j) % NR), (uint32_t)(((k + j) / NR) & 1));
    bad |= !wait_phase(smem_addr(bar + NR + (k & 1)), (uint32_t)((k >> 1) & 1));
    if ((timed_out = __syncthreads_or(bad))) break;
    const unsigned char *vk = vals + (size_t)(k & 1) * VAL_BYTES;
    const uint4 *A = reinterpret_cast<const uint4 *>(vk) + (size_t)grp * KS * 64 + lane;
#pragma unroll
    for (int s = 0; s < KS; ++s) {
      const uint4 ahi = A[s * 64], alo = A[s * 64 + 32];
      int rr = (k % NR) * kChunk + 16 * grp + 16 * s + lrow;  // ring row of this lane's address
      if (rr >= RING_ROWS) rr -= RING_ROWS;                      // 16-row steps never straddle the wrap
      const uint32_t rowaddr = ring_s + (uint32_t)(rr / kChunk) * CHUNK_BYTES + (uint32_t)(rr % kChunk) * 128;
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) {
        uint32_t b0, b1, b2, b3;
        ldsm_x4_trans(rowaddr + ((uint32_t)((2 * jj + lunit) ^ (rr & 7)) << 4), b0, b1, b2, b3);
        mma16<T>(acc[2 * jj], ahi, b0, b1);
        mma16<T>(acc[2 * jj + 1], ahi, b2, b3);
        mma16<T>(acc[2 * jj], alo, b0, b1);
        mma16<T>(acc[2 * jj + 1], alo, b2, b3);
      }
    }
    const float *inv = reinterpret_cast<const float *>(vk + 4 * KS * 2 * kFragBytes);
    const float i0 = inv[16 * grp + g], i1 = inv[16 * grp + g + 8];
    bad = !wait_phase(smem_addr(bar + NR + 2), (uint32_t)(k & 1));
    if ((timed_out = __syncthreads_or(bad))) break;
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
      const uint32_t a = crow_s + ((uint32_t)((2 * jj + lunit) ^ (crow & 7)) << 4);
      uint32_t o[4];
      ldsm_x4(a, o[0], o[1], o[2], o[3]);  // (rows g, n-tile 2jj) (g + 8, 2jj) (g, 2jj + 1) (g + 8, 2jj + 1)
      uint32_t v[4];
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        const float *ac = acc[2 * jj + (m >> 1)] + 2 * (m & 1);
        const float sc = (m & 1) ? i1 : i0;
        const float2 old = unpack2<T>(o[m]);
        v[m] = pack2<T>(ac[0] * sc + old.x, ac[1] * sc + old.y);
      }
      stsm_x4(a, v[0], v[1], v[2], v[3]);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // the tile's writes, before the TMA store reads it
    __syncthreads();  // chunk k's slot, value slot k & 1 and the C tile are done with
    if (threadIdx.x == 0) {
      if (k + NR < nchunks) issue_chunk(k + NR);
      if (k + 2 < nb) issue_vals(k + 2);
#pragma unroll
      for (int hf = 0; hf < 2; ++hf)
        asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];"
                     ::"l"(cmap_p), "r"(col0 + 64 * hf), "r"((g0 + k) * kCtaRows), "r"(smem_addr(ctile) + hf * HALF_BYTES)
                     : "memory");
      asm volatile("cp.async.bulk.commit_group;" ::: "memory");
      if (k + 1 < nb) {
        asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");  // the store has read the tile
        issue_c(k + 1);
      }
    }
  }
  if (threadIdx.x == 0) {
    if (timed_out) {
      atomicExch(&g_band_timeout, 1);
      // give the copies still in flight a bounded chance to land before the block leaves
      for (int c = max(0, issued_chunks - NR); c < issued_chunks; ++c)
        wait_phase(smem_addr(bar + c % NR), (uint32_t)((c / NR) & 1));
      for (int v = max(0, issued_vals - 2); v < issued_vals; ++v)
        wait_phase(smem_addr(bar + NR + (v & 1)), (uint32_t)((v >> 1) & 1));
      wait_phase(smem_addr(bar + NR + 2), (uint32_t)((issued_c - 1) & 1));
    }
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");  // the last stores are complete
  }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }();
  return fn;
}

template <int TW>
swift_status launch_tile(const CUtensorMap &map, const float *tiles, int M, int N, int W, void *C, int64_t ldc,
                         int sm_count, cudaStream_t st) {
  constexpr int NR = (panel_rows(TW) + kChunk - 1) / kChunk + 1;
  constexpr size_t smem = (size_t)NR * kChunk * kSlice * 4 + 2 * (size_t)kCtaRows * TW * 4 + (NR + 2) * 8;
  // one block per SM: its old-C rows and accumulators (64 registers) would spill at the 128
  // registers of two blocks
  static_assert(smem <= 227 * 1024, "band tile kernel: shared memory above the per-block limit");
  auto k = band_tile_kernel<TW, 1>;
  SW_CHECK_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  SW_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, 256, smem));
  const int ngroups = (M + kCtaRows - 1) / kCtaRows, nslices = (N + kSlice - 1) / kSlice;
  // one resident block per row range: contiguous ranges of 64-row groups, every SM filled
  int ranges = std::max(1, std::min(ngroups, sm_count * std::max(occ, 1) / nslices));
  const int per = (ngroups + ranges - 1) / ranges;
  ranges = (ngroups + per - 1) / per;
  k<<<dim3((unsigned)ranges, (unsigned)nslices), 256, smem, st>>>(map, tiles, M, N, W, ngroups, per,
                                                                 static_cast<float *>(C), ldc);
  SW_CHECK_LAUNCH();
  return SWIFT_OK;
}

swift_status launch_tile_w(const CUtensorMap &map, const float *tiles, int M, int N, int W, void *C, int64_t ldc,
                           int sm_count, cudaStream_t st) {
  switch (W) {
    case 3: return launch_tile<tile_width(3)>(map, tiles, M, N, W, C, ldc, sm_count, st);
    case 7: return launch_tile<tile_width(7)>(map, tiles, M, N, W, C, ldc, sm_count, st);
    case 15: return launch_tile<tile_width(15)>(map, tiles, M, N, W, C, ldc, sm_count, st);
    case 31: return launch_tile<tile_width(31)>(map, tiles, M, N, W, C, ldc, sm_count, st);
    case 47: return launch_tile<tile_width(47)>(map, tiles, M, N, W, C, ldc, sm_count, st);
    case 63: return launch_tile<tile_width(63)>(map, tiles, M, N, W, C, ldc, sm_count, st);
  }
  return SWIFT_ERR_UNSUPPORTED;
}

template <class T, int TW>
swift_status launch_mma(const CUtensorMap &bmap, const CUtensorMap &cmap, const unsigned char *frags, int M, int N,
                        int W, int sm_count, cudaStream_t st) {
  constexpr int KS = mma_width(TW) / 16;
  constexpr int NR = (kCtaRows - 16 + mma_width(TW) + kChunk - 1) / kChunk + 1;
  constexpr size_t smem = (size_t)(NR + 1) * 2 * kChunk * 128 + 2 * (size_t)mma_block_bytes(KS) + (NR + 3) * 8 + 1024;
  constexpr int minb = smem * 2 + 2048 <= 227 * 1024 ? 2 : 1;
  static_assert(smem <= 227 * 1024, "band mma kernel: shared memory above the per-block limit");
  auto k = band_mma_kernel<T, TW, minb>;
  SW_CHECK_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  SW_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, 256, smem));
  const int ngroups = (M + kCtaRows - 1) / kCtaRows, nslices = (N + kSlice - 1) / kSlice;
  int ranges = std::max(1, std::min(ngroups, sm_count * std::max(occ, 1) / nslices));
  const int per = (ngroups + ranges - 1) / ranges;
  ranges = (ngroups + per - 1) / per;
  k<<<dim3((unsigned)ranges, (unsigned)nslices), 256, smem, st>>>(bmap, cmap, frags, W, ngroups, per);
  SW_CHECK_LAUNCH();
  return SWIFT_OK;
}

template <class T>
swift_status launch_mma_w(const CUtensorMap &bmap, const CUtensorMap &cmap, const unsigned char *frags, int M, int N,
                          int W, int sm_count, cudaStream_t st) {
  switch (W) {
    case 3: return launch_mma<T, tile_width(3)>(bmap, cmap, frags, M, N, W, sm_count, st);
    case 7: return launch_mma<T, tile_width(7)>(bmap, cmap, frags, M, N, W, sm_count, st);
    case 15: return launch_mma<T, tile_width(15)>(bmap, cmap, frags, M, N, W, sm_count, st);
    case 31: return launch_mma<T, tile_width(31)>(bmap, cmap, frags, M, N, W, sm_count, st);
    case 47: return launch_mma<T, tile_width(47)>(bmap, cmap, frags, M, N, W, sm_count, st);
    case 63: return launch_mma<T, tile_width(63)>(bmap, cmap, frags, M, N, W, sm_count, st);
  }
  return SWIFT_ERR_UNSUPPORTED;
}

// A 2-D row-major 16-bit tensor (rows x cols, leading dimension ld elements) as 64 x 64 boxes
// with the 128-byte swizzle.
swift_status encode_16bit_swizzled(CUtensorMap *map, const void *base, int rows, int cols, int64_t ld, int dtype) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
  if (!enc) {
    set_last_error("cuTensorMapEncodeTiled", "driver entry point not available");
    return SWIFT_ERR_CUDA;
  }
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)std::max(rows, 1)};
  cuuint64_t strides[1] = {(cuuint64_t)(ld * 2)};
  cuuint32_t box[2] = {64, (cuuint32_t)kChunk};
  cuuint32_t es[2] = {1, 1};
  const CUresult cr = enc(map, dtype == SWIFT_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16,
                          2, const_cast<void *>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (cr != CUDA_SUCCESS) {
    set_last_error("cuTensorMapEncodeTiled", "operand cannot be described as a TMA tensor");
    return SWIFT_ERR_UNSUPPORTED;
  }
  return SWIFT_OK;
}

}  // namespace

// Distance profile and the half-width choice (p.mu held).
swift_status band_profile(Plan &p, cudaStream_t st) {
  if (p.band_w != -2) return SWIFT_OK;
  if (!p.has_csr) return SWIFT_ERR_UNSUPPORTED;
  TmpBuf h;
  SW_TRY(h.alloc(sizeof(unsigned long long) * (kMaxDist + 1), st));
  SW_CHECK_CUDA(cudaMemsetAsync(h.p, 0, sizeof(unsigned long long) * (kMaxDist + 1), st));
  if (p.M > 0) {
    const int grid = std::max(1, std::min((p.M + 7) / 8, p.sm_count * 8));
    band_profile_kernel<<<grid, 256, 0, st>>>(p.rowptr.as<int>(), p.colidx.as<int>(), p.M,
                                              static_cast<unsigned long long *>(h.p));
    SW_CHECK_LAUNCH();
  }
  unsigned long long hh[kMaxDist + 1];
  SW_CHECK_CUDA(cudaMemcpyAsync(hh, h.p, sizeof(hh), cudaMemcpyDeviceToHost, st));
  SW_CHECK_CUDA(cudaStreamSynchronize(st));
  for (int d = 0; d <= kMaxDist; ++d) p.band_hist[d] = (long long)hh[d];
  // A gathered nonzero costs the row walk about eight times what one dense tile element costs
  // the tile kernel (measured: 39 ps per FP32 nonzero at N = 128 against about 4 ps per tile
  // element); pick the width with the largest saving, if it saves a twentieth of the gathers.
  double best = 0.05 * (double)p.nnz;
  int bw = -1;
  for (int w : kWidths) {
    long long in = 0;
    for (int d = 0; d <= w; ++d) in += p.band_hist[d];
    const double gain = (double)in - (double)p.M * tile_width(w) / 8.0;
    if (gain > best && (int64_t)((p.M + kCtaRows - 1) / kCtaRows) * kCtaRows * tile_width(w) < INT32_MAX) {
      best = gain;
      bw = w;
    }
  }
  p.band_w = bw;
  return SWIFT_OK;
}

// Splits A into tiles + rest for half-width W (p.mu held).
static swift_status band_build(Plan &p, int W, cudaStream_t st) {
  const int TW = tile_width(W);
  const int64_t rows_pad = (int64_t)((p.M + kCtaRows - 1) / kCtaRows) * kCtaRows;
  if (rows_pad * TW >= INT32_MAX) return SWIFT_ERR_OVERFLOW;
  p.band_built = false;
  p.band_mma_built[0] = p.band_mma_built[1] = false;
  SW_TRY(p.band_tiles.alloc(sizeof(float) * (size_t)std::max<int64_t>(rows_pad * TW, 1)));
  SW_CHECK_CUDA(cudaMemsetAsync(p.band_tiles.p, 0, p.band_tiles.bytes, st));
  SW_TRY(p.band_ptr.alloc(sizeof(int) * ((size_t)p.M + 1)));
  SW_TRY(p.band_dst.alloc(sizeof(int) * (size_t)std::max(p.nnz, 1)));
  const int grid = std::max(1, std::min((p.M + 7) / 8, p.sm_count * 16));
  if (p.M > 0) {
    band_count_kernel<<<grid, 256, 0, st>>>(p.rowptr.as<int>(), p.colidx.as<int>(), p.M, W, TW, p.band_ptr.as<int>());
    SW_CHECK_LAUNCH();
  }
  SW_TRY(scan_exclusive_i32(p.band_ptr.as<int>(), p.band_ptr.as<int>(), p.M, st));
  int rest = 0;
  SW_CHECK_CUDA(cudaMemcpyAsync(&rest, p.band_ptr.as<int>() + p.M, sizeof(int), cudaMemcpyDeviceToHost, st));
  SW_CHECK_CUDA(cudaStreamSynchronize(st));
  SW_TRY(p.band_idx.alloc(sizeof(int) * (size_t)std::max(rest, 1)));
  SW_TRY(p.band_val.alloc(p.vsz * (size_t)std::max(rest, 1)));
  if (p.M > 0) {
    if (p.val_type == SWIFT_F64)
      band_split_kernel<double><<<grid, 256, 0, st>>>(p.rowptr.as<int>(), p.colidx.as<int>(), p.val.as<double>(), p.M, W,
                                                      TW, p.band_ptr.as<int>(), p.band_idx.as<int>(),
                                                      p.band_val.as<double>(), p.band_tiles.as<float>(),
                                                      p.band_dst.as<int>());
    else
      band_split_kernel<float><<<grid, 256, 0, st>>>(p.rowptr.as<int>(), p.colidx.as<int>(), p.val.as<float>(), p.M, W,
                                                     TW, p.band_ptr.as<int>(), p.band_idx.as<int>(),
                                                     p.band_val.as<float>(), p.band_tiles.as<float>(),
                                                     p.band_dst.as<int>());
    SW_CHECK_LAUNCH();
  }
  // the rest as a row-walk operand (merge tasks are built on its first product)
  RowLayout &L = p.band_rest;
  L = RowLayout();
  L.rows = p.M; L.cols = p.K; L.nnz = rest;
  L.ptr = p.band_ptr.as<int>(); L.idx = p.band_idx.as<int>(); L.val = p.band_val.p; L.out_row = nullptr;
  p.band_rest_nnz = rest;
  p.band_used_w = W;
  p.band_built = true;
  return SWIFT_OK;
}

// The tiles in the tensor-core kernel's fragment order for 16-bit type `dtype`, in that type's
// own buffer (p.mu held; after band_build).
static swift_status band_mma_build(Plan &p, int dtype, cudaStream_t st) {
  const int TW = tile_width(p.band_used_w);
  const int KS = mma_width(TW) / 16;
  const int nblocks = (p.M + kCtaRows - 1) / kCtaRows;
  const int64_t rows = (int64_t)nblocks * kCtaRows;
  const int ti = dtype == SWIFT_BF16 ? 0 : 1;
  DevBuf &out = p.band_mma[ti];
  p.band_mma_built[ti] = false;
  SW_TRY(out.alloc((size_t)std::max(nblocks, 1) * mma_block_bytes(KS)));
  TmpBuf rexp;
  SW_TRY(rexp.alloc(sizeof(int) * (size_t)std::max<int64_t>(rows, 1), st));
  const int rgrid = (int)std::max<int64_t>(1, std::min<int64_t>((rows + 255) / 256, (int64_t)p.sm_count * 16));
  band_row_exp_kernel<<<rgrid, 256, 0, st>>>(p.band_tiles.as<float>(), rows, TW, rexp.as<int>());
  SW_CHECK_LAUNCH();
  const int64_t threads = (int64_t)nblocks * 4 * KS * 32;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((threads + 255) / 256, (int64_t)p.sm_count * 16));
  if (dtype == SWIFT_BF16)
    band_mma_fill_kernel<__nv_bfloat16><<<grid, 256, 0, st>>>(p.band_tiles.as<float>(), rexp.as<int>(), nblocks, TW, KS,
                                                              static_cast<unsigned char *>(out.p));
  else
    band_mma_fill_kernel<__half><<<grid, 256, 0, st>>>(p.band_tiles.as<float>(), rexp.as<int>(), nblocks, TW, KS,
                                                       static_cast<unsigned char *>(out.p));
  SW_CHECK_LAUNCH();
  p.band_mma_built[ti] = true;
  return SWIFT_OK;
}

swift_status band_refill(Plan &p, cudaStream_t st) {
  if (!p.band_built || p.nnz == 0) return SWIFT_OK;
  p.band_mma_built[0] = p.band_mma_built[1] = false;  // regrouped on the next 16-bit products
  const int grid = (int)std::min<int64_t>(((int64_t)p.nnz + 255) / 256, (int64_t)p.sm_count * 16);
  if (p.val_type == SWIFT_F64)
    band_refill_kernel<double><<<grid, 256, 0, st>>>(p.val.as<double>(), p.nnz, p.band_dst.as<int>(),
                                                     p.band_val.as<double>(), p.band_tiles.as<float>());
  else
    band_refill_kernel<float><<<grid, 256, 0, st>>>(p.val.as<float>(), p.nnz, p.band_dst.as<int>(),
                                                    p.band_val.as<float>(), p.band_tiles.as<float>());
  SW_CHECK_LAUNCH();
  return SWIFT_OK;
}

bool band_operands_ok(const Plan &p, const DenseArgs &d) {
  if (!p.has_csr || p.val_type != SWIFT_F32) return false;
  if (d.dtype != SWIFT_F32 && d.dtype != SWIFT_BF16 && d.dtype != SWIFT_F16) return false;
  if (d.b_layout != SWIFT_ROW_MAJOR || d.c_layout != SWIFT_ROW_MAJOR || d.b_presorted) return false;
  if (d.b_scale || d.c_scale) return false;
  const size_t esz = d.dtype == SWIFT_F32 ? 4 : 2;
  if (d.N < kSlice || d.N % 4 != 0) return false;
  if ((uintptr_t)d.B % 16 != 0 || (d.ldb * (int64_t)esz) % 16 != 0) return false;
  if ((uintptr_t)d.C % 16 != 0 || (d.ldc * (int64_t)esz) % 16 != 0) return false;
  return true;
}

swift_status run_band(Plan &p, const DenseArgs &d, const MergeOpts &o, cudaStream_t st) {
  if (!band_operands_ok(p, d)) return SWIFT_ERR_UNSUPPORTED;
  if (p.M == 0 || d.N == 0) return SWIFT_OK;
  int W = 0;
  {
    std::lock_guard<std::mutex> g(p.mu);
    SW_TRY(band_profile(p, st));
    W = p.band_w >= 0 ? p.band_w : kWidths[0];
    if (!p.band_built || p.band_used_w != W) SW_TRY(band_build(p, W, st));
    if (d.dtype != SWIFT_F32 && !p.band_mma_built[d.dtype == SWIFT_BF16 ? 0 : 1])
      SW_TRY(band_mma_build(p, d.dtype, st));
  }
  if (d.dtype != SWIFT_F32) {
    // 16-bit B and C: the tensor-core kernel, both operands as swizzled 64 x 64 TMA boxes
    CUtensorMap bmap, cmap;
    SW_TRY(encode_16bit_swizzled(&bmap, d.B, p.K, d.N, d.ldb, d.dtype));
    SW_TRY(encode_16bit_swizzled(&cmap, d.C, p.M, d.N, d.ldc, d.dtype));
    // the rest first: the row walk writes every C row (zeros where a row has no rest nonzeros)
    SW_TRY(run_merge(p, p.band_rest, d, o, st));
    const unsigned char *frags = static_cast<const unsigned char *>(p.band_mma[d.dtype == SWIFT_BF16 ? 0 : 1].p);
    if (d.dtype == SWIFT_BF16) return launch_mma_w<__nv_bfloat16>(bmap, cmap, frags, p.M, d.N, W, p.sm_count, st);
    return launch_mma_w<__half>(bmap, cmap, frags, p.M, d.N, W, p.sm_count, st);
  }
  PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
  if (!enc) {
    set_last_error("cuTensorMapEncodeTiled", "driver entry point not available");
    return SWIFT_ERR_CUDA;
  }
  CUtensorMap map;
  cuuint64_t dims[2] = {(cuuint64_t)d.N, (cuuint64_t)std::max(p.K, 1)};
  cuuint64_t strides[1] = {(cuuint64_t)(d.ldb * (int64_t)4)};
  cuuint32_t box[2] = {(cuuint32_t)kSlice, (cuuint32_t)kChunk};
  cuuint32_t es[2] = {1, 1};
  const CUresult cr = enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void *>(d.B), dims, strides, box, es,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (cr != CUDA_SUCCESS) {
    set_last_error("cuTensorMapEncodeTiled", "B cannot be described as a TMA tensor");
    return SWIFT_ERR_UNSUPPORTED;
  }
  SW_TRY(run_merge(p, p.band_rest, d, o, st));
  return launch_tile_w(map, p.band_tiles.as<float>(), p.M, d.N, W, d.C, d.ldc, p.sm_count, st);
}

swift_status band_timeout_flag(int *flag, int reset) {
  int v = 0;
  SW_CHECK_CUDA(cudaMemcpyFromSymbol(&v, g_band_timeout, sizeof(int)));
  if (reset && v) {
    const int z = 0;
    SW_CHECK_CUDA(cudaMemcpyToSymbol(g_band_timeout, &z, sizeof(int)));
  }
  if (flag) *flag = v;
  return SWIFT_OK;
}

}  // namespace swift
