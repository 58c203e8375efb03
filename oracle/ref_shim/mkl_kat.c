/* Known-answer check of the MKL entry points libtorch_cpu exports, through the
 * declarations in mkl_spblas.h / mkl.h -- TEST INFRASTRUCTURE ONLY
 * (oracle/build_ref.py runs it before it trusts the reference's CPU module).
 *
 * A = [[1 2 0] [0 0 3] [4 0 5]] in MKL's four-array CSR, B = [[1 2] [3 4]
 * [5 6]] row-major: checks the status codes (the enum values), that 32-bit
 * indices are read as such (LP64), A B, A^T B and cblas_saxpy.
 * Exit status 0: all agree. */
#include <stdio.h>

#include "mkl.h"

static int close_to(const float* got, const float* want, int n) {
  for (int i = 0; i < n; ++i)
    if (got[i] != want[i]) return 0;
  return 1;
}

int main(void) {
  int rb[3] = {0, 2, 3}, re[3] = {2, 3, 5}, ci[5] = {0, 1, 2, 0, 2};
  float va[5] = {1, 2, 3, 4, 5};
  float b[6] = {1, 2, 3, 4, 5, 6};
  float c[6] = {-1, -1, -1, -1, -1, -1};
  sparse_matrix_t a;
  if (mkl_sparse_s_create_csr(&a, SPARSE_INDEX_BASE_ZERO, 3, 3, rb, re, ci, va) != SPARSE_STATUS_SUCCESS) return 2;
  struct matrix_descr d;
  d.type = SPARSE_MATRIX_TYPE_GENERAL;
  d.mode = SPARSE_FILL_MODE_FULL;
  d.diag = SPARSE_DIAG_NON_UNIT;
  if (mkl_sparse_s_mm(SPARSE_OPERATION_NON_TRANSPOSE, 1.0f, a, d, SPARSE_LAYOUT_ROW_MAJOR, b, 2, 2, 0.0f, c, 2) !=
      SPARSE_STATUS_SUCCESS)
    return 3;
  const float ab[6] = {7, 10, 15, 18, 29, 38};
  if (!close_to(c, ab, 6)) return 4;
  if (mkl_sparse_s_mm(SPARSE_OPERATION_TRANSPOSE, 1.0f, a, d, SPARSE_LAYOUT_ROW_MAJOR, b, 2, 2, 0.0f, c, 2) !=
      SPARSE_STATUS_SUCCESS)
    return 5;
  const float atb[6] = {21, 26, 2, 4, 34, 42};
  if (!close_to(c, atb, 6)) return 6;
  if (mkl_sparse_destroy(a) != SPARSE_STATUS_SUCCESS) return 7;
  float y[3] = {1, 1, 1};
  const float x[3] = {1, 2, 3};
  cblas_saxpy(3, 2.0f, x, 1, y, 1);
  const float axpy[3] = {3, 5, 7};
  if (!close_to(y, axpy, 3)) return 8;
  printf("mkl kat ok (max threads %d)\n", mkl_get_max_threads());
  return 0;
}
