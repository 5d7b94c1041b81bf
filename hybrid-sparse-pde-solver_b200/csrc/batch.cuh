// batch.cuh -- many small, independent, uneven systems solved in one persistent launch.
//
// The reference solves one system per SolverBase::solve call (solver_base.hpp:32-35); a
// batch is the engine's answer to "thousands of small systems": every system keeps the
// reference's algorithm (PCG + Jacobi, cg_solver.cpp:37-191; FGMRES(m) + ILU(0),
// fgmres_solver.cpp:165-241 and ilu.cpp:41-89) but all of them run inside ONE kernel.
//
// Layout (all device resident):
//   the batch is one block-diagonal CSR: system k owns rows [row_off[k], row_off[k+1]) and
//   its entries' columns lie in the same range (checked); int32 indices, FP64 values and an
//   FP32 copy.  Per-row: the diagonal position, w/a_ii in FP32, and for ILU systems the
//   FP32 factor values in A's pattern plus the rows of every system grouped by level.
//   Per-system FP32 work vectors are laid end to end (CG 5n, FGMRES (2m+5)n floats).
// Arithmetic: FP32 values, vectors and SpMV inside an FP64 iterative-refinement loop per
// system (FP64 residual b - A x with FP64 values, x += ||r|| d in FP64); dot products
// accumulate in FP64 and the CG alpha/beta and the Hessenberg / Givens data are FP64.
// Scheduling: a CTA of kBatchThreads threads is split into teams of W threads (one warp up
// to the whole CTA); a team claims one system at a time from an atomic ticket and solves
// it to the end, synchronising on a named barrier of its own.  Systems are grouped in
// size classes, each with its own team width (the "row-scheduling shape"), processed
// largest class first and, inside a class, longest system first.  The widths come from a
// measured autotuner (hamlss_batch_autotune) with an on-disk cache, or defaults.
#pragma once

#include "krylov.cuh"

namespace hamlss {

constexpr int kBatchThreads = 512;
constexpr int kBatchMaxM = 32;          // restart length cap of the batched FGMRES
constexpr int kBatchClasses = 4;        // n <= 1024, <= 4096, <= 16384, larger
constexpr int kBatchWidths[5] = {32, 64, 128, 256, 512};

// method of one system
enum : int { BM_CG_JAC = 0, BM_CG_NONE = 1, BM_GM_ILU = 2, BM_GM_JAC = 3, BM_GM_NONE = 4 };

struct BProb {
    int row0, n, method, klass;
    int levL, nlevL, levU, nlevU;    // level lists of an ILU system (lptr* slots)
    long long w0;                    // first float of its work vectors
};

struct Batch {
    hamlss_ctx* ctx = nullptr;
    int count = 0, N = 0, nnz = 0, m = 20;
    hamlss_params params{};
    std::vector<int> row_off;
    std::vector<BProb> hprob;
    int width[kBatchClasses] = {32, 64, 128, 256};
    DBuf<int> rp, ci, dpos, lptrL, lordL, lptrU, lordU, pstatus, order, tickets;
    DBuf<double> v64, r64, xb, bb, xt;
    DBuf<float> v32, dinv, lu, work;
    DBuf<BProb> prob;
    DBuf<hamlss_batch_result> out;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    double last_ms = 0.0;
    ~Batch();
};

std::unique_ptr<Batch> batch_create(Ctx& ctx, hamlss_ctx* h, int count, const int* row_off,
                                    const int* rp, const int* ci, const double* v,
                                    const int* solver, const int* precond, int where,
                                    const hamlss_params& p);
// Solve every system: b, x (FP64, batch layout) on the device.  class_mask selects the
// size classes to run (all: 0xF).  Returns the kernel time in ms (CUDA events).
double batch_run(Ctx& ctx, Batch& B, const double* b, double* x, unsigned class_mask);
void batch_autotune(Ctx& ctx, Batch& B, const double* b_dev, const char* cache_path,
                    int* widths_out);

}  // namespace hamlss

struct hamlss_batch {
    hamlss_ctx* ctx = nullptr;
    std::unique_ptr<hamlss::Batch> b;
};
