// Test infrastructure only: a C-ABI driver over the reference's own CPU core.
//
// This file is compiled together with the reference's unmodified C++ sources
// (src/fe_absorption.cpp, src/hdfe_regressor_v11.cpp, src/ols.cpp, src/iv.cpp,
// src/schwarz_demean.cpp, src/akm_kss.cpp) by oracle/Makefile into
// oracle/_ref/libxhdfe_ref.so.  It is the checker that pins the oracle and the
// timed CPU baseline; nothing in the product links or loads it.
//
// Entry points mirror the reference's public calls:
//   xref_absorb       -> hdfe::detail::absorb_fixed_effects_v6  (src/fe_absorption.cpp:8750)
//   xref_absorb_slopes-> the same, with HeterogeneousSlopeTerm slopes (include/fe_absorption.hpp:49-53)
//   xref_absorb_gi    -> hdfe::detail::absorb_fixed_effects_group_individual (include/fe_absorption.hpp:103-109)
//   xref_partial_out  -> hdfe::v11::HdfeRegressorV11::partial_out (src/hdfe_regressor_v11.cpp:10275)
//   xref_fit          -> hdfe::v11::HdfeRegressorV11::fit         (src/hdfe_regressor_v11.cpp:7522)
//   xref_akm_kss      -> hdfe::akm::akm_kss_decompose              (include/hdfe/akm_kss.hpp:227-233)
//   xref_recover_fe   -> hdfe::detail::recover_fixed_effects        (include/fe_absorption.hpp:127-130)
//   xref_run_ols      -> hdfe::detail::run_ols                      (include/ols.hpp:40-51)
//   xref_components   -> hdfe::v11::compute_first_pair_component_stats (include/hdfe/hdfe_regressor_v11.hpp:75-78)
// Every entry point catches all exceptions and returns a nonzero status with
// the message copied into err (the reference's own fail-closed contract).

#include <Eigen/Dense>

#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <vector>

#include "fe_absorption.hpp"
#include "fe_absorption_cuda.hpp"
#include "hdfe/hdfe_regressor.hpp"
#include "schwarz_demean.hpp"
#include "hdfe/akm_kss.hpp"
#include "ols.hpp"
#include "hdfe/hdfe_regressor_v11.hpp"

namespace {

using Eigen::Map;
using Eigen::MatrixXd;
using Eigen::VectorXd;
using Eigen::VectorXi;

struct XrefOptions {
    double tol;
    int tolerance_mode;   // 0 xhdfe-fast, 1 reghdfe-comparable, 2 strict-residual
    int absorption_method;  // hdfe::AbsorptionMethod integer value
    int num_threads;
    int max_iter;
    int drop_singletons;
    int se_type;          // 0 homoskedastic, 1 robust, 2 cluster
    int fit_intercept;
    int gpu_backend;      // 0 library default, 1 force CPU, 2 force CUDA
    int use_krylov;       // 1: HdfeOptions::use_krylov (the coefficient-space Jacobi-PCG
                          //    absorber, src/fe_absorption.cpp:10110), CPU backend
};

// Thread-local backend selection through the reference's own override
// (include/fe_absorption_cuda.hpp:108-122).
std::unique_ptr<hdfe::detail::ScopedGpuBackendOverride> backend_guard(const XrefOptions* o) {
    if (o->gpu_backend == 1)
        return std::make_unique<hdfe::detail::ScopedGpuBackendOverride>(hdfe::detail::GpuBackend::Cpu);
    if (o->gpu_backend == 2)
        return std::make_unique<hdfe::detail::ScopedGpuBackendOverride>(hdfe::detail::GpuBackend::Cuda);
    return nullptr;
}

hdfe::HdfeOptions to_options(const XrefOptions* o) {
    hdfe::HdfeOptions opts;
    opts.tol = o->tol;
    opts.tolerance_mode = static_cast<hdfe::ToleranceMode>(o->tolerance_mode);
    opts.absorption_method = static_cast<hdfe::AbsorptionMethod>(o->absorption_method);
    opts.num_threads = o->num_threads;
    opts.num_threads_explicit = o->num_threads > 0;
    if (o->max_iter > 0) {
        opts.max_iter = o->max_iter;
    }
    opts.drop_singletons = o->drop_singletons != 0;
    opts.se_type = static_cast<hdfe::StandardErrorType>(o->se_type);
    opts.fit_intercept = o->fit_intercept != 0;
    opts.use_krylov = o->use_krylov != 0;
    return opts;
}

std::vector<VectorXi> to_fes(const int32_t* fe_flat, int64_t n, int dims) {
    std::vector<VectorXi> fes;
    fes.reserve(static_cast<std::size_t>(dims));
    for (int d = 0; d < dims; ++d) {
        VectorXi v(n);
        std::memcpy(v.data(), fe_flat + static_cast<std::size_t>(d) * n,
                    sizeof(int32_t) * static_cast<std::size_t>(n));
        fes.push_back(std::move(v));
    }
    return fes;
}

void set_err(char* err, int err_len, const char* msg) {
    if (err && err_len > 0) {
        std::strncpy(err, msg, static_cast<std::size_t>(err_len) - 1);
        err[err_len - 1] = '\0';
    }
}

}  // namespace

extern "C" {

// Demean y (n) and X (n x k, column-major) on all FE dims, no singleton drop.
// info[0]=iterations info[1]=converged info[2]=precision_certified
// info[3]=gpu_status_code dinfo[0]=abs_residual dinfo[1]=abs_residual_rel
int xref_absorb(const double* y, const double* X, int64_t n, int k,
                const int32_t* fe_flat, int dims, const double* w,
                const XrefOptions* o, double* y_out, double* X_out,
                int* info, double* dinfo, char* err, int err_len) {
    try {
        Map<const VectorXd> ym(y, n);
        Map<const MatrixXd> Xm(X, n, k);
        std::vector<VectorXi> fes = to_fes(fe_flat, n, dims);
        VectorXd wv;
        if (w) {
            wv = Map<const VectorXd>(w, n);
        }
        hdfe::HdfeOptions opts = to_options(o);
        auto guard = backend_guard(o);
        hdfe::detail::AbsorptionResult r = hdfe::detail::absorb_fixed_effects_v6(
            ym, Xm, fes, w ? &wv : nullptr, opts, opts.absorption_method);
        std::memcpy(y_out, r.y_tilde.data(), sizeof(double) * static_cast<std::size_t>(n));
        if (k > 0) {
            std::memcpy(X_out, r.X_tilde.data(),
                        sizeof(double) * static_cast<std::size_t>(n) * k);
        }
        info[0] = r.iterations;
        info[1] = r.converged ? 1 : 0;
        info[2] = r.precision_certified ? 1 : 0;
        info[3] = r.gpu_status_code;
        dinfo[0] = r.abs_residual;
        dinfo[1] = r.abs_residual_rel;
        return 0;
    } catch (const std::exception& e) {
        set_err(err, err_len, e.what());
        return 1;
    } catch (...) {
        set_err(err, err_len, "unknown exception");
        return 1;
    }
}

// absorb_fixed_effects_v6 with heterogeneous slopes: slope_kind[d] is 0 for a
// plain FE, 1 for a slope without intercept, 2 for intercept and slope; the
// slope values of dim d are slope_flat[d * n .. d * n + n).  Same outputs as
// xref_absorb.
int xref_absorb_slopes(const double* y, const double* X, int64_t n, int k,
                       const int32_t* fe_flat, int dims, const double* w,
                       const double* slope_flat, const int* slope_kind,
                       const XrefOptions* o, double* y_out, double* X_out,
                       int* info, double* dinfo, char* err, int err_len) {
    try {
        Map<const VectorXd> ym(y, n);
        Map<const MatrixXd> Xm(X, n, k);
        std::vector<VectorXi> fes = to_fes(fe_flat, n, dims);
        VectorXd wv;
        if (w) {
            wv = Map<const VectorXd>(w, n);
        }
        std::vector<hdfe::detail::HeterogeneousSlopeTerm> slopes;
        for (int d = 0; d < dims; ++d) {
            if (slope_kind[d] == 0) continue;
            hdfe::detail::HeterogeneousSlopeTerm t;
            t.fe_index = d;
            t.values = Map<const VectorXd>(slope_flat + static_cast<std::size_t>(d) * n, n);
            t.include_intercept = slope_kind[d] == 2;
            slopes.push_back(std::move(t));
        }
        hdfe::HdfeOptions opts = to_options(o);
        auto guard = backend_guard(o);
        hdfe::detail::AbsorptionResult r = hdfe::detail::absorb_fixed_effects_v6(
            ym, Xm, fes, w ? &wv : nullptr, opts, opts.absorption_method, slopes);
        std::memcpy(y_out, r.y_tilde.data(), sizeof(double) * static_cast<std::size_t>(n));
        if (k > 0) {
            std::memcpy(X_out, r.X_tilde.data(),
                        sizeof(double) * static_cast<std::size_t>(n) * k);
        }
        info[0] = r.iterations;
        info[1] = r.converged ? 1 : 0;
        info[2] = r.precision_certified ? 1 : 0;
        info[3] = r.gpu_status_code;
        dinfo[0] = r.abs_residual;
        dinfo[1] = r.abs_residual_rel;
        return 0;
    } catch (const std::exception& e) {
        set_err(err, err_len, e.what());
        return 1;
    } catch (...) {
        set_err(err, err_len, "unknown exception");
        return 1;
    }
}

// absorb_fixed_effects_group_individual: rows are groups; the structure's
// CSR arrays as in GroupIndividualStructure (include/fe_absorption.hpp:13-21).
// Same outputs as xref_absorb.
int xref_absorb_gi(const double* y, const double* X, int64_t n, int k, const int32_t* fe_flat,
                   int dims, const double* w, const int32_t* group_ptr,
                   const int32_t* group_individual, const int32_t* individual_ptr,
                   const int32_t* individual_group, const double* group_scale,
                   int num_individuals, int64_t num_edges, const XrefOptions* o, double* y_out,
                   double* X_out, int* info, double* dinfo, char* err, int err_len) {
    try {
        const VectorXd yv = Map<const VectorXd>(y, n);
        const MatrixXd Xm = Map<const MatrixXd>(X, n, k);
        std::vector<VectorXi> fes = to_fes(fe_flat, n, dims);
        VectorXd wv;
        if (w) {
            wv = Map<const VectorXd>(w, n);
        }
        hdfe::detail::GroupIndividualStructure gi;
        gi.num_groups = static_cast<int>(n);
        gi.num_individuals = num_individuals;
        gi.group_ptr.assign(group_ptr, group_ptr + n + 1);
        gi.group_individual.assign(group_individual, group_individual + num_edges);
        gi.individual_ptr.assign(individual_ptr, individual_ptr + num_individuals + 1);
        gi.individual_group.assign(individual_group, individual_group + num_edges);
        gi.group_scale.assign(group_scale, group_scale + n);
        hdfe::HdfeOptions opts = to_options(o);
        auto guard = backend_guard(o);
        hdfe::detail::AbsorptionResult r = hdfe::detail::absorb_fixed_effects_group_individual(
            yv, Xm, fes, gi, w ? &wv : nullptr, opts, opts.absorption_method);
        std::memcpy(y_out, r.y_tilde.data(), sizeof(double) * static_cast<std::size_t>(n));
        if (k > 0) {
            std::memcpy(X_out, r.X_tilde.data(),
                        sizeof(double) * static_cast<std::size_t>(n) * k);
        }
        info[0] = r.iterations;
        info[1] = r.converged ? 1 : 0;
        info[2] = r.precision_certified ? 1 : 0;
        info[3] = r.gpu_status_code;
        dinfo[0] = r.abs_residual;
        dinfo[1] = r.abs_residual_rel;
        return 0;
    } catch (const std::exception& e) {
        set_err(err, err_len, e.what());
        return 1;
    } catch (...) {
        set_err(err, err_len, "unknown exception");
        return 1;
    }
}

// HdfeRegressorV11::partial_out with singleton drop.  Outputs are sized n;
// only the first info[3] rows are written.  sample_index receives the kept
// 0-based row indices.
int xref_partial_out(const double* y, const double* X, int64_t n, int k,
                     const int32_t* fe_flat, int dims, const double* w,
                     const XrefOptions* o, double* y_out, double* X_out,
                     int32_t* sample_index, int* info, double* dinfo,
                     char* err, int err_len) {
    try {
        Map<const VectorXd> ym(y, n);
        Map<const MatrixXd> Xm(X, n, k);
        std::vector<VectorXi> fes = to_fes(fe_flat, n, dims);
        VectorXd wv;
        if (w) {
            wv = Map<const VectorXd>(w, n);
        }
        hdfe::HdfeOptions opts = to_options(o);
        auto guard = backend_guard(o);
        hdfe::v11::HdfeRegressorV11 reg(opts);
        hdfe::detail::AbsorptionResult r =
            reg.partial_out(ym, Xm, fes, w ? &wv : nullptr, nullptr, nullptr);
        const hdfe::HdfeResults& res = reg.results();
        const int64_t kept = r.y_tilde.size();
        std::memcpy(y_out, r.y_tilde.data(), sizeof(double) * static_cast<std::size_t>(kept));
        if (k > 0) {
            std::memcpy(X_out, r.X_tilde.data(),
                        sizeof(double) * static_cast<std::size_t>(kept) * k);
        }
        for (int64_t i = 0; i < kept && i < res.sample_index.size(); ++i) {
            sample_index[i] = res.sample_index[i];
        }
        info[0] = r.iterations;
        info[1] = r.converged ? 1 : 0;
        info[2] = r.precision_certified ? 1 : 0;
        info[3] = static_cast<int>(kept);
        info[4] = reg.gpu_status_code();
        dinfo[0] = r.abs_residual;
        dinfo[1] = r.abs_residual_rel;
        return 0;
    } catch (const std::exception& e) {
        set_err(err, err_len, e.what());
        return 1;
    } catch (...) {
        set_err(err, err_len, "unknown exception");
        return 1;
    }
}

// HdfeRegressorV11::fit.  coef/se have room for k+1 entries (intercept last
// when fit_intercept).  cluster may be null (then se_type must not be 2).
// info[0]=iterations info[1]=converged info[2]=precision_certified
// info[3]=nobs info[4]=num_singletons info[5]=number of coefficients
// dinfo[0]=abs_residual_rel dinfo[1]=rss dinfo[2]=r2_within dinfo[3]=df_a
int xref_fit(const double* y, const double* X, int64_t n, int k,
             const int32_t* fe_flat, int dims, const double* w,
             const int32_t* cluster, const XrefOptions* o, double* coef,
             double* se, int* info, double* dinfo, char* err, int err_len) {
    try {
        Map<const VectorXd> ym(y, n);
        Map<const MatrixXd> Xm(X, n, k);
        std::vector<VectorXi> fes = to_fes(fe_flat, n, dims);
        VectorXd wv;
        if (w) {
            wv = Map<const VectorXd>(w, n);
        }
        std::vector<VectorXi> clusters;
        if (cluster) {
            clusters = to_fes(cluster, n, 1);
        }
        hdfe::HdfeOptions opts = to_options(o);
        auto guard = backend_guard(o);
        hdfe::v11::HdfeRegressorV11 reg(opts);
        reg.fit(ym, Xm, fes, w ? &wv : nullptr, cluster ? &clusters : nullptr);
        const hdfe::HdfeResults& res = reg.results();
        const int p = static_cast<int>(res.coefficients.size());
        for (int j = 0; j < p; ++j) {
            coef[j] = res.coefficients[j];
            se[j] = res.std_errors[j];
        }
        info[0] = res.num_iterations;
        info[1] = res.converged ? 1 : 0;
        info[2] = res.precision_certified ? 1 : 0;
        info[3] = res.nobs;
        info[4] = res.num_singletons;
        info[5] = p;
        info[6] = reg.gpu_status_code();
        dinfo[0] = res.abs_residual_rel;
        dinfo[1] = res.rss;
        dinfo[2] = res.r2_within;
        dinfo[3] = res.df_a;
        return 0;
    } catch (const std::exception& e) {
        set_err(err, err_len, e.what());
        return 1;
    } catch (...) {
        set_err(err, err_len, "unknown exception");
        return 1;
    }
}

// The same decomposition, returning its working rows: *n_rows rows (at most
// cap) with their leverage pii, original worker and firm ids and person-year
// weight, in the library's row order (hdfe::akm::AkmKssResult::pii,
// row_worker, row_firm, row_weight; include/hdfe/akm_kss.hpp:120-124).
int xref_akm_kss_rows(const double* y, const int32_t* worker, const int32_t* firm, int64_t n,
                      const int* opts, uint64_t seed, double cg_tol, int64_t cap, double* pii,
                      int32_t* row_worker, int32_t* row_firm, double* row_weight, int64_t* n_rows,
                      char* err, int err_len) {
    try {
        const VectorXd yv = Map<const VectorXd>(y, n);
        VectorXi wv(n), fv(n);
        for (int64_t i = 0; i < n; ++i) {
            wv[i] = worker[i];
            fv[i] = firm[i];
        }
        hdfe::akm::AkmOptions o;
        o.leverage_method = opts[0] == 1   ? hdfe::akm::LeverageMethod::Exact
                            : opts[0] == 2 ? hdfe::akm::LeverageMethod::Jla
                                           : hdfe::akm::LeverageMethod::Auto;
        if (opts[1] > 0) o.jla_draws = opts[1];
        if (opts[2] >= 0) o.direct_max_firms = opts[2];
        o.use_gpu = opts[3] != 0;
        o.num_threads = opts[4];
        o.cg_max_iter = opts[5];
        o.seed = seed;
        if (cg_tol > 0.0) o.cg_tol = cg_tol;
        const hdfe::akm::AkmKssResult r = hdfe::akm::akm_kss_decompose(yv, wv, fv, nullptr, o);
        const int64_t R = static_cast<int64_t>(r.pii.size());
        *n_rows = R;
        if (R > cap) {
            set_err(err, err_len, "row buffers too small");
            return 1;
        }
        for (int64_t k = 0; k < R; ++k) {
            pii[k] = r.pii[k];
            row_worker[k] = r.row_worker[k];
            row_firm[k] = r.row_firm[k];
            row_weight[k] = r.row_weight[k];
        }
        return 0;
    } catch (const std::exception& e) {
        set_err(err, err_len, e.what());
        return 1;
    } catch (...) {
        set_err(err, err_len, "unknown exception");
        return 1;
    }
}

// AKM + leave-out decomposition.  opts (ints): [0] leverage method (0 auto,
// 1 exact, 2 jla), [1] jla_draws, [2] direct_max_firms (-1: library default),
// [3] use_gpu, [4] num_threads, [5] cg_max_iter; seed and cg_tol as given.
// out (doubles, 16): plugin var_alpha, var_psi, cov; agsu (3); kss (3); var_y;
// sigma2_ho; mean_pii; max_pii; n_obs of the leave-out sample.
// info (ints, 8): [0] workers, [1] firms, [2] matches, [3] gpu_used,
// [4] gpu_status_code, [5] solver_direct, [6] converged, [7] jla_draws_used.
// iters_out: total PCG iterations.
int xref_akm_kss(const double* y, const int32_t* worker, const int32_t* firm, int64_t n,
                 const int* opts, uint64_t seed, double cg_tol, double* out, int* info,
                 long long* iters_out, char* err, int err_len) {
    try {
        const VectorXd yv = Map<const VectorXd>(y, n);
        VectorXi wv(n), fv(n);
        for (int64_t i = 0; i < n; ++i) {
            wv[i] = worker[i];
            fv[i] = firm[i];
        }
        hdfe::akm::AkmOptions o;
        o.leverage_method = opts[0] == 1   ? hdfe::akm::LeverageMethod::Exact
                            : opts[0] == 2 ? hdfe::akm::LeverageMethod::Jla
                                           : hdfe::akm::LeverageMethod::Auto;
        if (opts[1] > 0) o.jla_draws = opts[1];
        if (opts[2] >= 0) o.direct_max_firms = opts[2];
        o.use_gpu = opts[3] != 0;
        o.num_threads = opts[4];
        o.cg_max_iter = opts[5];
        o.seed = seed;
        if (cg_tol > 0.0) o.cg_tol = cg_tol;
        const hdfe::akm::AkmKssResult r = hdfe::akm::akm_kss_decompose(yv, wv, fv, nullptr, o);
        const double vals[16] = {r.plugin.var_alpha, r.plugin.var_psi, r.plugin.cov_alpha_psi,
                                 r.agsu.var_alpha,   r.agsu.var_psi,   r.agsu.cov_alpha_psi,
                                 r.kss.var_alpha,    r.kss.var_psi,    r.kss.cov_alpha_psi,
                                 r.var_y,            r.sigma2_ho,      r.mean_pii,
                                 r.max_pii,          static_cast<double>(r.sample.n_obs), 0.0, 0.0};
        std::memcpy(out, vals, sizeof(vals));
        info[0] = r.sample.n_workers;
        info[1] = r.sample.n_firms;
        info[2] = static_cast<int>(r.sample.n_matches);
        info[3] = r.gpu_used ? 1 : 0;
        info[4] = r.gpu_status_code;
        info[5] = r.solver_direct ? 1 : 0;
        info[6] = r.converged ? 1 : 0;
        info[7] = r.jla_draws_used;
        *iters_out = r.solver_iterations;
        return 0;
    } catch (const std::exception& e) {
        set_err(err, err_len, e.what());
        return 1;
    } catch (...) {
        set_err(err, err_len, "unknown exception");
        return 1;
    }
}

// Saved-FE recovery of a partial residual: contrib (n x dims, column-major)
// receives the per-dim FE contributions; info: [0] iterations, [1] converged;
// dinfo: [0] max_delta.
int xref_recover_fe(const double* partial, int64_t n, const int32_t* fe_flat, int dims,
                    const double* w, const XrefOptions* o, double fe_tolerance, double* contrib,
                    int* info, double* dinfo, char* err, int err_len) {
    try {
        const VectorXd pv = Map<const VectorXd>(partial, n);
        std::vector<VectorXi> fes = to_fes(fe_flat, n, dims);
        VectorXd wv;
        if (w) wv = Map<const VectorXd>(w, n);
        hdfe::HdfeOptions opts = to_options(o);
        opts.fe_tolerance = fe_tolerance;
        auto guard = backend_guard(o);
        const hdfe::detail::FeRecoveryResult r =
            hdfe::detail::recover_fixed_effects(pv, fes, w ? &wv : nullptr, opts);
        for (int d = 0; d < dims; ++d) {
            if (static_cast<int64_t>(r.contributions.size()) <= d ||
                r.contributions[d].size() != n) {
                set_err(err, err_len, "recover_fixed_effects returned no contribution");
                return 1;
            }
            std::memcpy(contrib + static_cast<int64_t>(d) * n, r.contributions[d].data(),
                        sizeof(double) * n);
        }
        info[0] = r.iterations;
        info[1] = r.converged ? 1 : 0;
        dinfo[0] = r.max_delta;
        return 0;
    } catch (const std::exception& e) {
        set_err(err, err_len, e.what());
        return 1;
    } catch (...) {
        set_err(err, err_len, "unknown exception");
        return 1;
    }
}

// OLS on within-transformed data.  X: n x p column-major; clusters: n dense
// ids or null.  out_vec (4p): coef, se, then covariance (p x p column-major)
// follows in out_cov; scalars (8): rss, sigma2, df_resid, cov_scale,
// cluster_u2, r2, r2_within, num_clusters.
int xref_run_ols(const double* y, const double* X, int64_t n, int p, const double* w,
                 const int32_t* clusters, int se_type, double tss, double within_tss,
                 double n_effective, int weights_are_frequencies, double* coef, double* se,
                 double* cov, double* scalars, char* err, int err_len) {
    try {
        const VectorXd yv = Map<const VectorXd>(y, n);
        const MatrixXd Xm = Map<const MatrixXd>(X, n, p);
        VectorXd wv;
        if (w) wv = Map<const VectorXd>(w, n);
        VectorXi cv;
        if (clusters) {
            cv.resize(n);
            for (int64_t i = 0; i < n; ++i) cv[i] = clusters[i];
        }
        const hdfe::detail::OlsResult r = hdfe::detail::run_ols(
            yv, Xm, w ? &wv : nullptr, clusters ? &cv : nullptr,
            static_cast<hdfe::StandardErrorType>(se_type), tss, within_tss, n_effective,
            weights_are_frequencies != 0);
        for (int j = 0; j < p; ++j) {
            coef[j] = r.coefficients[j];
            se[j] = r.std_errors[j];
        }
        std::memcpy(cov, r.covariance.data(), sizeof(double) * p * p);
        scalars[0] = r.rss;
        scalars[1] = r.sigma2;
        scalars[2] = r.df_resid;
        scalars[3] = r.cov_scale;
        scalars[4] = r.cluster_u2;
        scalars[5] = r.r2;
        scalars[6] = r.r2_within;
        scalars[7] = r.num_clusters;
        return 0;
    } catch (const std::exception& e) {
        set_err(err, err_len, e.what());
        return 1;
    } catch (...) {
        set_err(err, err_len, "unknown exception");
        return 1;
    }
}

// Mobility groups of the first FE pair: out_i[0] num_components; out_l[0]
// largest_component_n_obs; out_d[0..1] obs and weight shares.
int xref_components(const int32_t* fe1, const int32_t* fe2, int64_t n, const double* w, int* out_i,
                    long long* out_l, double* out_d, char* err, int err_len) {
    try {
        VectorXi a(n), b(n);
        for (int64_t i = 0; i < n; ++i) {
            a[i] = fe1[i];
            b[i] = fe2[i];
        }
        VectorXd wv;
        if (w) wv = Map<const VectorXd>(w, n);
        const hdfe::v11::FeComponentStats st =
            hdfe::v11::compute_first_pair_component_stats(a, b, w ? &wv : nullptr);
        out_i[0] = st.num_components;
        out_l[0] = st.largest_component_n_obs;
        out_d[0] = st.largest_component_obs_share;
        out_d[1] = st.largest_component_weight_share;
        return 0;
    } catch (const std::exception& e) {
        set_err(err, err_len, e.what());
        return 1;
    } catch (...) {
        set_err(err, err_len, "unknown exception");
        return 1;
    }
}

// xhdfe::schwarz_demean_raw (include/schwarz_demean.hpp:30-34) on Y (n) and X
// (n x k, column-major) in place; fe_flat holds dims id arrays of length n.
// Returns 1 when the call returned true, 0 when false.
int xref_schwarz_demean_raw(double* Y, double* X, int64_t n, int k, const int32_t* fe_flat, int dims,
                            const int32_t* nlev, int threads, double tol, int max_iter, int* iters_out) {
    std::vector<const int32_t*> fe;
    std::vector<int> lv;
    for (int d = 0; d < dims; ++d) {
        fe.push_back(fe_flat + static_cast<std::size_t>(d) * n);
        lv.push_back(nlev[d]);
    }
    try {
        return xhdfe::schwarz_demean_raw(Y, X, n, k, fe, lv, threads, tol, max_iter, iters_out, -1) ? 1 : 0;
    } catch (...) {
        return 0;
    }
}

}  // extern "C"
