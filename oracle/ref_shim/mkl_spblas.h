/* Declarations of the Intel MKL sparse BLAS names that the reference's
 * cbm/cbm_extensions.cpp uses -- TEST INFRASTRUCTURE ONLY (oracle/build_ref.py).
 *
 * Project-written from MKL's published C API (LP64: MKL_INT is a 32-bit int,
 * the `_i4` interface libtorch_cpu links).  Names, enum values and signatures
 * only; no MKL code.  libtorch_cpu.so exports mkl_sparse_s_create_csr,
 * mkl_sparse_s_mm, mkl_sparse_destroy and mkl_sparse_s_export_csr, which the
 * eight product operators need; the constructor's mkl_sparse_s_create_coo,
 * mkl_sparse_convert_csr and mkl_sparse_syrk are not exported anywhere here,
 * so cbm_init_ stays unresolved (its module is loaded with lazy binding and
 * init is never called). */
#ifndef CBM_REF_SHIM_MKL_SPBLAS_H
#define CBM_REF_SHIM_MKL_SPBLAS_H

#ifndef MKL_INT
#define MKL_INT int
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  SPARSE_STATUS_SUCCESS = 0,
  SPARSE_STATUS_NOT_INITIALIZED = 1,
  SPARSE_STATUS_ALLOC_FAILED = 2,
  SPARSE_STATUS_INVALID_VALUE = 3,
  SPARSE_STATUS_EXECUTION_FAILED = 4,
  SPARSE_STATUS_INTERNAL_ERROR = 5,
  SPARSE_STATUS_NOT_SUPPORTED = 6
} sparse_status_t;

typedef enum {
  SPARSE_OPERATION_NON_TRANSPOSE = 10,
  SPARSE_OPERATION_TRANSPOSE = 11,
  SPARSE_OPERATION_CONJUGATE_TRANSPOSE = 12
} sparse_operation_t;

typedef enum {
  SPARSE_MATRIX_TYPE_GENERAL = 20,
  SPARSE_MATRIX_TYPE_SYMMETRIC = 21,
  SPARSE_MATRIX_TYPE_HERMITIAN = 22,
  SPARSE_MATRIX_TYPE_TRIANGULAR = 23,
  SPARSE_MATRIX_TYPE_DIAGONAL = 24,
  SPARSE_MATRIX_TYPE_BLOCK_TRIANGULAR = 25,
  SPARSE_MATRIX_TYPE_BLOCK_DIAGONAL = 26
} sparse_matrix_type_t;

typedef enum { SPARSE_INDEX_BASE_ZERO = 0, SPARSE_INDEX_BASE_ONE = 1 } sparse_index_base_t;

typedef enum { SPARSE_FILL_MODE_LOWER = 40, SPARSE_FILL_MODE_UPPER = 41, SPARSE_FILL_MODE_FULL = 42 } sparse_fill_mode_t;

typedef enum { SPARSE_DIAG_NON_UNIT = 50, SPARSE_DIAG_UNIT = 51 } sparse_diag_type_t;

typedef enum { SPARSE_LAYOUT_ROW_MAJOR = 101, SPARSE_LAYOUT_COLUMN_MAJOR = 102 } sparse_layout_t;

struct matrix_descr {
  sparse_matrix_type_t type;
  sparse_fill_mode_t mode;
  sparse_diag_type_t diag;
};

struct sparse_matrix;
typedef struct sparse_matrix* sparse_matrix_t;

sparse_status_t mkl_sparse_s_create_csr(sparse_matrix_t* A, sparse_index_base_t indexing, MKL_INT rows, MKL_INT cols,
                                        MKL_INT* rows_start, MKL_INT* rows_end, MKL_INT* col_indx, float* values);
sparse_status_t mkl_sparse_s_create_coo(sparse_matrix_t* A, sparse_index_base_t indexing, MKL_INT rows, MKL_INT cols,
                                        MKL_INT nnz, MKL_INT* row_indx, MKL_INT* col_indx, float* values);
sparse_status_t mkl_sparse_convert_csr(const sparse_matrix_t source, sparse_operation_t operation,
                                       sparse_matrix_t* dest);
sparse_status_t mkl_sparse_s_export_csr(const sparse_matrix_t source, sparse_index_base_t* indexing, MKL_INT* rows,
                                        MKL_INT* cols, MKL_INT** rows_start, MKL_INT** rows_end, MKL_INT** col_indx,
                                        float** values);
sparse_status_t mkl_sparse_syrk(const sparse_operation_t operation, const sparse_matrix_t A, sparse_matrix_t* C);
sparse_status_t mkl_sparse_s_mm(const sparse_operation_t operation, const float alpha, const sparse_matrix_t A,
                                const struct matrix_descr descr, const sparse_layout_t layout, const float* B,
                                const MKL_INT columns, const MKL_INT ldb, const float beta, float* C,
                                const MKL_INT ldc);
sparse_status_t mkl_sparse_destroy(sparse_matrix_t A);

#ifdef __cplusplus
}
#endif
#endif
