// dense_lu.cuh -- blocked dense LU with partial pivoting and explicit inverse (device).
#pragma once

#include "engine.cuh"

namespace hamlss {

// Factor the row-major n x n matrix M in place (P A = L U, unit lower L below the
// diagonal, U on and above it; piv[j] = the row swapped with row j at step j) and write
// A^-1 (row-major) to Minv.  Throws HAMLSS_ERR_ZERO_PIVOT for a singular matrix.
// Synchronises the context stream.
void dense_lu_inverse(Ctx& ctx, int n, double* M, double* Minv, int* piv);

// Release a context's cuBLAS handle (Ctx::blas).
void blas_destroy(void* handle);
// The context's cuBLAS handle (a cublasHandle_t, created on first use), bound to the
// context's stream.
void* blas_stream_handle(Ctx& ctx);

}  // namespace hamlss
