// precond.cuh -- device preconditioners behind one interface (PreconditionerBase,
// include/preconditioners/preconditioner_base.hpp:16-48 in the reference).
#pragma once

#include "engine.cuh"

namespace hamlss {

struct Prec {
    int kind = HAMLSS_PREC_NONE;
    int n = 0;
    virtual ~Prec() = default;
    // z = M^-1 r on device vectors, enqueued on the lane; no-op while *gate != 0.
    virtual void apply(Ctx& ctx, const Lane& L, const double* r, double* z, const int* gate) = 0;
    // FP32 variant used inside mixed-precision solves (values / vectors in float).
    virtual void apply32(Ctx& ctx, const Lane& L, const float* r, float* z, const int* gate) {
        (void)ctx; (void)L; (void)r; (void)z; (void)gate;
        fail(HAMLSS_ERR_INVALID, "this preconditioner has no FP32 path");
    }
    virtual bool has32() const { return false; }
    virtual void prepare32(Ctx& ctx) { (void)ctx; }
};

// JacobiPreconditioner (jacobi.cpp:13-51): inv_diag = omega / a_ii, z = inv_diag .* r.
struct JacobiPrec : Prec {
    DBuf<double> inv;
    DBuf<float> inv32;
    bool inv32_valid = false;
    void apply(Ctx& ctx, const Lane& L, const double* r, double* z, const int* gate) override;
    void apply32(Ctx& ctx, const Lane& L, const float* r, float* z, const int* gate) override;
    bool has32() const override { return true; }
    void prepare32(Ctx& ctx) override;
};

std::unique_ptr<Prec> make_jacobi(Ctx& ctx, hamlss_mat* A, double omega);
std::unique_ptr<Prec> make_ilu0(Ctx& ctx, hamlss_mat* A);
// ILUT(drop_tol, fill_p) (ilu.cpp:94-220) on the device
std::unique_ptr<Prec> make_ilut(Ctx& ctx, hamlss_mat* A, double drop_tol, int fill_p);
// ILUPreconditioner::setup's dispatch (ilu.cpp:31-36): ILUT when drop_tol > 0 or
// fill_per_row > 0, else ILU(0)
std::unique_ptr<Prec> make_ilu(Ctx& ctx, hamlss_mat* A, const hamlss_params& p);
std::unique_ptr<Prec> make_amg(Ctx& ctx, hamlss_mat* A, const hamlss_params& p);

int ilu_copy_factors(const Prec* M, double* out, cudaStream_t s);
// the L\U factor as CSR: *nnz, then rp / ci / v when non-null (host arrays)
int ilu_factor_csr(const Prec* M, int* nnz, int* rp, int* ci, double* v, cudaStream_t s);
int amg_num_levels(const Prec* P, int* levels);
int amg_level_matrix(const Prec* P, int level, int which, int* rows, int* cols, int* nnz, int* rp,
                     int* ci, double* v, cudaStream_t s);
int amg_aggregate_matrix(Ctx& ctx, hamlss_mat* A, double theta, int* agg_host, int* n_agg);
int ilu_copy_levels(const Prec* M, int which, int* level, int* nlev, cudaStream_t s);
void pattern_levels(Ctx& ctx, int n, int nnz, const int* rp, const int* ci, DBuf<int>& dpos,
                    DBuf<int>& levelL, DBuf<int>& levelU, int* nlevL, int* nlevU);

// Extract a_ii into A->diag (once per value version).
void ensure_diag(Ctx& ctx, hamlss_mat* A);

}  // namespace hamlss

struct hamlss_prec {
    hamlss_ctx* ctx = nullptr;
    hamlss_mat* A = nullptr;
    std::unique_ptr<hamlss::Prec> p;
};
