// ilu_row.cuh -- the ILU(0) row elimination shared by the single-matrix and the batched
// factorisations.
#pragma once

#include "common.cuh"

namespace hamlss {

// IKJ elimination of the rows of one lower level (ilu.cpp:52-83), thread per row.
// status[0] receives the smallest row whose pivot is tiny (ZERO_PIVOT).
__device__ __forceinline__ void ilu_row(int i, const int* __restrict__ rp, const int* __restrict__ ci,
                                        const int* __restrict__ dpos, double* lu, int* status) {
    const int s = rp[i], e = rp[i + 1];
    for (int p = s; p < e; ++p) {
        const int k = ci[p];
        if (k >= i) break;
        const int dk = dpos[k];
        const double ukk = dk >= 0 ? lu[dk] : 0.0;
        if (fabs(ukk) < 2.220446049250313e-16) { atomicMin(status, k); return; }
        const double lik = lu[p] / ukk;
        lu[p] = lik;
        int pi = p + 1;                          // merge pointer into row i (sorted)
        for (int q = rp[k]; q < rp[k + 1]; ++q) {
            const int j = ci[q];
            if (j <= k) continue;
            while (pi < e && ci[pi] < j) ++pi;
            if (pi == e) break;
            if (ci[pi] == j) lu[pi] = __dsub_rn(lu[pi], __dmul_rn(lik, lu[q]));
        }
    }
}

}  // namespace hamlss
