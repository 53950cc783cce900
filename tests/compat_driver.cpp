// A program written the way the reference's driver is (src/main.cu:200-450), compiled against
// include/swift_compat.h and linked with libswiftb200.so: every reference function keeps its
// name and signature, every stage runs on the GPU.  Built and run by tests/test_compat_header.py.
//
//   compat_driver M K density N seed     -> exit 0 if every wrapper's check passed
//
// Build with -DSWIFT_COMPAT_FP32 for the FP32 flavour (test/k-32/FP32 signatures).
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "swift_compat.h"

#ifdef SWIFT_COMPAT_FP32
typedef float VAL;
typedef float GFLOPS;
#else
typedef double VAL;
typedef double GFLOPS;
#endif

static uint64_t lcg(uint64_t &s) {
  s = s * 6364136223846793005ULL + 1442695040888963407ULL;
  return s >> 33;
}

int main(int argc, char **argv) {
  if (argc < 6) {
    std::fprintf(stderr, "usage: %s M K density N seed\n", argv[0]);
    return 2;
  }
  const int rowA = std::atoi(argv[1]), colA = std::atoi(argv[2]);
  const double density = std::atof(argv[3]);
  const int BN = std::atoi(argv[4]);
  uint64_t seed = (uint64_t)std::atoll(argv[5]) * 2654435761ULL + 1;

  // CSR with skewed column popularity (some long columns, many short ones)
  std::vector<int> rowptr(rowA + 1, 0), colidx;
  std::vector<VAL> val;
  for (int r = 0; r < rowA; ++r) {
    std::vector<char> used(colA, 0);
    const int want = (int)(density * colA) + (int)(lcg(seed) % 3);
    for (int t = 0; t < want; ++t) {
      const double u = (double)(lcg(seed) % 1000000) / 1e6;
      const int c = (int)(u * u * colA) % colA;
      if (!used[c]) used[c] = 1;
    }
    for (int c = 0; c < colA; ++c)
      if (used[c]) {
        colidx.push_back(c);
        val.push_back((VAL)((double)(lcg(seed) % 2000001) / 1e6 - 1.0));
      }
    rowptr[r + 1] = (int)colidx.size();
  }
  const int nnz = rowptr[rowA];
  std::vector<VAL> dense((size_t)colA * BN);
  for (auto &x : dense) x = (VAL)((double)(lcg(seed) % 2000001) / 1e6 - 1.0);

  // golden C = A * B, row-major, accumulated in double
  std::vector<VAL> golden((size_t)rowA * BN, 0);
  for (int r = 0; r < rowA; ++r)
    for (int j = 0; j < BN; ++j) {
      double acc = 0;
      for (int p = rowptr[r]; p < rowptr[r + 1]; ++p) acc += (double)val[p] * (double)dense[(size_t)colidx[p] * BN + j];
      golden[(size_t)r * BN + j] = (VAL)acc;
    }

  // src/main.cu: csr_to_csc -> col_sort -> formattransation -> block_catgory
  std::vector<VAL> cscval(nnz > 0 ? nnz : 1);
  std::vector<int> cscrow(nnz > 0 ? nnz : 1), cscptr(colA + 1), nnzpercol(colA > 0 ? colA : 1);
#ifdef SWIFT_COMPAT_FP32
  float t_csc = 0;
#else
  double t_csc = 0;
#endif
  csr_to_csc(t_csc, rowA, colA, nnz, val.data(), rowptr.data(), colidx.data(), cscval.data(), cscrow.data(),
             cscptr.data(), nnzpercol.data());
  std::vector<int> sortrowidx_tmp(nnz > 0 ? nnz : 1), sortnnz_tmp(colA > 0 ? colA : 1);
  std::vector<VAL> sortval_tmp(nnz > 0 ? nnz : 1), sort_dense((size_t)colA * BN);
  col_sort(colA, BN, nnzpercol.data(), cscptr.data(), cscrow.data(), cscval.data(), sortrowidx_tmp.data(),
           sortval_tmp.data(), sortnnz_tmp.data(), dense.data(), sort_dense.data());

  slide_matrix *matrixA = (slide_matrix *)std::malloc(sizeof(slide_matrix));
  std::memset(matrixA, 0, sizeof(slide_matrix));
#ifdef SWIFT_COMPAT_FP32
  float time_irrepart = 0;
  formattransation(time_irrepart, matrixA, sortrowidx_tmp.data(), sortval_tmp.data(), sortnnz_tmp.data(), nnz,
                   rowA, colA);
  block_catgory(matrixA);
#else
  double time_irrepart = 0, reside_ratio = 0, shuffle_ratio = 0;
  formattransation(time_irrepart, matrixA, sortrowidx_tmp.data(), sortval_tmp.data(), sortnnz_tmp.data(), nnz,
                   rowA, colA, reside_ratio);
  block_catgory(matrixA, shuffle_ratio);
#endif

  // column-major copy of the sorted dense operand (src/main.cu:338-340)
  std::vector<VAL> sort_dense1((size_t)colA * BN), result((size_t)rowA * BN);
  for (int j = 0; j < BN; ++j)
    for (int i = 0; i < colA; ++i) sort_dense1[(size_t)j * colA + i] = sort_dense[(size_t)i * BN + j];

  char filename[] = "synthetic";
  float t[5] = {0, 0, 0, 0, 0};
  GFLOPS gf[5] = {0, 0, 0, 0, 0};
  Swift_gpu1(filename, t[0], gf[0], matrixA, rowA, colA, BN, nnz, sort_dense1.data(), result.data(),
             golden.data());
  balance(matrixA, rowA, matrixA->reside_col, matrixA->reside_nnz, matrixA->reside_cscptr,
          matrixA->reside_cscrowidx);
  Swift_gpu2(filename, t[1], gf[1], matrixA, rowA, colA, BN, nnz, sort_dense.data(), result.data(),
             golden.data());
  Swift_GPU(filename, t[2], gf[2], matrixA, rowA, colA, BN, nnz, sort_dense1.data(), result.data(),
            golden.data());
  Swift_GPU_3(filename, t[3], gf[3], matrixA, rowA, colA, BN, nnz, sort_dense1.data(), result.data(),
              golden.data());
#ifdef SWIFT_COMPAT_FP32
  float blockratio = 0;
  row_idx_sort(matrixA, sort_dense1.data(), rowA, colA, BN, blockratio);
#else
  row_idx_sort(matrixA, sort_dense1.data(), rowA, colA, BN);
#endif
  Swift_GPU_4(filename, t[4], gf[4], matrixA, rowA, colA, BN, nnz, sort_dense1.data(), result.data(),
              golden.data());

  int failed = 0;
  const char *names[5] = {"Swift_gpu1", "Swift_gpu2", "Swift_GPU", "Swift_GPU_3", "Swift_GPU_4"};
  for (int i = 0; i < 5; ++i) {
    std::printf("%s %.4f ms %.2f GFLOP/s\n", names[i], t[i], (double)gf[i]);
    if (t[i] < 0) failed = 1;
  }
  std::printf("nnz %d tilenum %d reside_nnz %d numblk %d\n", nnz, matrixA->tilenum, matrixA->reside_nnz,
              matrixA->numblk);
  Tile_destroy(matrixA);
  std::free(matrixA);
  return failed;
}
