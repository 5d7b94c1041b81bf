// shim_test.cpp -- the drop-in shim used the way the project's own code uses its solvers.
//
// Built against the project's headers and linked with the project's library (built from
// its sources into oracle/_ref/) plus libhamlss_b200.so; run by tests/test_gpu_shim.py.
// Each check runs the project's CPU class and the device class on the same inputs.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <stdexcept>

#include "hsps_device.hpp"
#include "preconditioners/amg.hpp"
#include "preconditioners/ilu.hpp"
#include "preconditioners/jacobi.hpp"
#include "solvers/cg_solver.hpp"
#include "solvers/fgmres_solver.hpp"
#include "solvers/pipelined_fgmres_solver.hpp"

using namespace hsps;

static int failures = 0;
#define CHECK(cond, msg)                                                   \
    do {                                                                   \
        if (!(cond)) { std::printf("FAIL: %s\n", msg); ++failures; }       \
        else std::printf("ok: %s\n", msg);                                 \
    } while (0)

static double rel_res(const SparseMatrix& A, const Vector& b, const Vector& x) {
    Vector r = A * x;
    for (Index i = 0; i < b.size(); ++i) r[i] = b[i] - r[i];
    return r.norm2() / b.norm2();
}

int main() {
    SolverParams p;
    p.tol = 1e-9;
    p.max_iter = 3000;
    p.restart_size = 40;
    p.drop_tol = 0.0;

    for (const char* kind : {"poisson", "convdiff"}) {
        bool pois = kind[0] == 'p';
        SparseMatrix A = pois ? SparseMatrix::poisson_2d(32)
                              : SparseMatrix::convection_diffusion_2d(32, 1.0, 200.0, 100.0);
        Vector b(A.rows(), 1.0);
        struct Pair { SolverType s; PrecondType m; };
        Pair pairs[] = {{SolverType::CG, PrecondType::JACOBI}, {SolverType::FGMRES, PrecondType::ILU},
                        {SolverType::FGMRES, PrecondType::AMG}};
        for (auto pr : pairs) {
            if (!pois && pr.s == SolverType::CG) continue;
            auto cpu = SolverFactory::make(pr.s, pr.m, A, p);
            auto dev = hsps_b200::DeviceSolverFactory::make(pr.s, pr.m, A, p);
            Vector xc(A.rows(), 0.0), xd;        // xd resized to zeros by the device solver
            SolverStats sc, sd;
            bool oc = cpu.first->solve(A, b, xc, sc);
            bool od = dev.first->solve(A, b, xd, sd);
            char msg[256];
            std::snprintf(msg, sizeof msg, "%s %s+%s: converged %d/%d iters %d/%d rel %.2e", kind,
                          to_string(pr.s), to_string(pr.m), (int)oc, (int)od, sc.iterations,
                          sd.iterations, rel_res(A, b, xd));
            CHECK(oc == od && std::abs(sc.iterations - sd.iterations) <= 1 &&
                  (!od || rel_res(A, b, xd) < 1e-8), msg);
        }
    }

    {   // adaptive selector, reference rule
        auto A = SparseMatrix::convection_diffusion_2d(24, 1.0, 3000.0, 1500.0);
        Vector b(A.rows(), 1.0);
        SolverParams q = p;
        q.max_iter = 150;
        AdaptiveSelector cpu(q);
        hsps_b200::DeviceAdaptiveSelector dev(q);
        Vector xc(A.rows(), 0.0), xd(A.rows(), 0.0);
        SolverStats sc, sd;
        bool oc = cpu.solve(A, b, xc, sc);
        bool od = dev.solve(A, b, xd, sd);
        char msg[256];
        std::snprintf(msg, sizeof msg, "adaptive: converged %d/%d escalations %zu/%zu final %s/%s",
                      (int)oc, (int)od, cpu.escalation_log().size(), dev.escalation_log().size(),
                      to_string(cpu.current_state()), to_string(dev.current_state()));
        CHECK(oc == od && cpu.escalation_log().size() == dev.escalation_log().size() &&
              cpu.current_state() == dev.current_state(), msg);
    }

    {   // ILUT: the factory's ILU under the default drop_tol, and the class with fill
        SolverParams q = p;
        q.drop_tol = 1e-4;
        auto A = SparseMatrix::convection_diffusion_2d(32, 1.0, 200.0, 100.0);
        Vector b(A.rows(), 1.0);
        auto cpu = SolverFactory::make(SolverType::FGMRES, PrecondType::ILU, A, q);
        auto dev = hsps_b200::DeviceSolverFactory::make(SolverType::FGMRES, PrecondType::ILU, A, q);
        Vector xc(A.rows(), 0.0), xd;
        SolverStats sc, sd;
        bool oc = cpu.first->solve(A, b, xc, sc);
        bool od = dev.first->solve(A, b, xd, sd);
        char msg[256];
        std::snprintf(msg, sizeof msg, "FGMRES+ILUT(1e-4): converged %d/%d iters %d/%d", (int)oc,
                      (int)od, sc.iterations, sd.iterations);
        CHECK(oc == od && std::abs(sc.iterations - sd.iterations) <= 1, msg);
        ILUPreconditioner ic;
        hsps_b200::DeviceILU id;
        ic.set_drop_tol(1e-3); ic.set_fill_per_row(5); ic.setup(A);
        id.set_drop_tol(1e-3); id.set_fill_per_row(5); id.setup(A);
        Vector r(A.rows()), zc(A.rows()), zd(A.rows());
        for (Index i = 0; i < A.rows(); ++i) r[i] = std::sin(0.37 * i);
        ic.apply(r, zc);
        id.apply(r, zd);
        double diff = 0.0;
        for (Index i = 0; i < A.rows(); ++i) diff = std::max(diff, std::abs(zc[i] - zd[i]));
        std::snprintf(msg, sizeof msg, "ILUT(1e-3, 5) apply: max |cpu - device| = %.3e", diff);
        CHECK(diff == 0.0, msg);
    }

    {   // pipelined FGMRES and s-step CG, side by side with the project's classes
        auto A = SparseMatrix::convection_diffusion_2d(24, 1.0, 40.0, 20.0);
        Vector b(A.rows(), 1.0);
        SolverParams q = p;
        q.restart_size = 20;
        auto Mc = SolverFactory::make_precond(PrecondType::ILU, A, q);
        auto Md = hsps_b200::DeviceSolverFactory::make_precond(PrecondType::ILU, A, q);
        PipelinedFGMRESSolver pc;
        hsps_b200::DevicePipelinedFGMRESSolver pd;
        pc.set_params(q); pc.set_preconditioner(Mc);
        pd.set_params(q); pd.set_preconditioner(Md);
        Vector xc(A.rows(), 0.0), xd;
        SolverStats sc, sd;
        bool oc = pc.solve(A, b, xc, sc), od = pd.solve(A, b, xd, sd);
        char msg[256];
        std::snprintf(msg, sizeof msg, "pipelined FGMRES+ILU: converged %d/%d iters %d/%d", (int)oc,
                      (int)od, sc.iterations, sd.iterations);
        CHECK(oc == od && std::abs(sc.iterations - sd.iterations) <= 1 &&
              sd.solver_used == SolverType::FGMRES, msg);
        // the s-step update converges on a unit-diagonal operator: D^-1/2 A D^-1/2
        auto H = SparseMatrix::poisson_2d(16);
        std::vector<Index> r, c;
        std::vector<Real> v;
        for (Index i = 0; i < H.rows(); ++i)
            for (Index k = H.row_ptr()[i]; k < H.row_ptr()[i + 1]; ++k) {
                r.push_back(i);
                c.push_back(H.col_idx()[k]);
                v.push_back(H.values()[k] / 8.0 + (H.col_idx()[k] == i ? 0.5 : 0.0));
            }
        auto S = SparseMatrix::from_coo(H.rows(), H.cols(), r, c, v);
        Vector bs(S.rows(), 1.0);
        q.sstep_k = 4;
        q.max_iter = 400;
        auto cpu = SolverFactory::make(SolverType::SSTEP_CG, PrecondType::JACOBI, S, q);
        auto dev = hsps_b200::DeviceSolverFactory::make(SolverType::SSTEP_CG, PrecondType::JACOBI, S, q);
        Vector yc(S.rows(), 0.0), yd;
        SolverStats tc, td;
        bool ac = cpu.first->solve(S, bs, yc, tc), ad = dev.first->solve(S, bs, yd, td);
        std::snprintf(msg, sizeof msg, "s-step CG (k = 4): converged %d/%d iters %d/%d sstep_k %d/%d",
                      (int)ac, (int)ad, tc.iterations, td.iterations, tc.sstep_k, td.sstep_k);
        CHECK(ac == ad && std::abs(tc.iterations - td.iterations) <= 4 && tc.sstep_k == td.sstep_k &&
              td.solver_used == SolverType::SSTEP_CG, msg);
    }

    {   // error behaviour
        bool threw = false;
        try { hsps_b200::DeviceSolverFactory::make("CG", "SOR", SparseMatrix::poisson_2d(4), p); }
        catch (const std::invalid_argument&) { threw = true; }
        CHECK(threw, "unknown preconditioner name -> std::invalid_argument");
        threw = false;
        std::vector<Index> r = {0, 1}, c = {0, 1};
        std::vector<Real> v = {1.0, 0.0};
        auto Z = SparseMatrix::from_coo(2, 2, r, c, v);
        try { hsps_b200::DeviceJacobi J; J.setup(Z); }
        catch (const std::runtime_error&) { threw = true; }
        CHECK(threw, "zero diagonal -> std::runtime_error");
    }
    std::printf("%s (%d failures)\n", failures ? "FAILED" : "PASSED", failures);
    return failures ? 1 : 0;
}
