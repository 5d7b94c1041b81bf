// dense_lu.cuh -- blocked dense LU with partial pivoting and explicit inverse (device).
#pragma once

#include "engine.cuh"

namespace hamlss {

// Factor the row-major n x n matrix M in place (P A = L U, unit lower L below the
// diagonal, U on and above it; piv[j] = the row swapped with row j at step j) and write
// A^-1 (row-major) to Minv.  Throws HAMLSS_ERR_ZERO_PIVOT for a singular matrix.
// Synchronises the context stream.
void dense_lu_inverse(Ctx& ctx, int n, double* M, double* Minv, int* piv);

// Gram matrix G = Y^T Y ((c x c, row-major, device) of the c columns of Y (column j at
// Y + j * ld, n entries each), c <= 33: for n <= 32768 one thread per entry summing in
// row order (the reference's sequential dot product, bit for bit); above, block partial
// sums over row tiles in shared memory, then one ordered reduction over the blocks
// (deterministic).  `part` holds
// sm_count * 4 * c * (c + 1) / 2 doubles.
void gram_matrix(Ctx& ctx, int n, int c, const double* Y, long long ld, double* G, double* part);
int gram_partials(Ctx& ctx, int c);

}  // namespace hamlss
