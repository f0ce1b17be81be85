// Reference-side binding: the C++ symbols that reisportela/xhdfe-xfe's core
// calls when it is built with -DHDFE_USE_CUDA, implemented over the C ABI of
// libb200fe.so (include/b200fe.h).  Compile this file with the reference's
// headers in place of src/fe_absorption_cuda.cu and src/akm_kss_cuda.cu and
// link libb200fe.so; src/fe_absorption.cpp, the pybind11 module, the R package
// and the Stata plugin then reach the B200 absorber unchanged.
//
// Symbols (signatures from include/fe_absorption_cuda.hpp and
// include/hdfe/akm_kss_cuda.hpp of the reference):
//   cuda_backend_available                     (fe_absorption_cuda.hpp:125)
//   absorb_fixed_effects_cuda                  (fe_absorption_cuda.hpp:127-134)
//   absorb_fixed_effects_group_individual_cuda (fe_absorption_cuda.hpp:136-145)
//   fe_recovery_max_delta_cuda(_cached)        (fe_absorption_cuda.hpp:152-162)
//   cuda_cert_shadow_begin/finish/abort        (fe_absorption_cuda.hpp:74-99)
//   akm_cuda_*                                 (akm_kss_cuda.hpp:17-74)
//   xhdfe::schwarz_demean_raw                  (schwarz_demean.hpp:30-34; this file
//                                               then replaces src/schwarz_demean.cpp)
// The host certificate certify_cuda_absorption_result stays the reference's
// own src/fe_absorption_cuda_certificate.cpp.
//
// Contract kept from the reference (src/fe_absorption_cuda.cu:2294-4738):
// return false on any failure (the caller reports status 4 and fails closed
// when the GPU backend was requested, src/fe_absorption.cpp:9227-9237);
// return true with converged=false on non-convergence; never throw.  Features
// this library does not provide yet return false, so the reference fails
// closed rather than silently using another path: saved fixed effects together
// with heterogeneous slopes, and saved fixed effects in the reference's
// per-sweep means mode.  Heterogeneous slopes (GpuFeInput with is_slope) run on
// b200fe_absorb_slopes, group/individual FEs on b200fe_absorb_group_individual.  Saved FEs in the coefficient mode
// (fe_alpha_y / fe_alpha_X, what recover_fixed_effects consumes) come from
// b200fe_absorb_fe.  The
// AKM/KSS solver (akm_cuda_*) runs on the library's batched PCG
// (b200fe_kss_*).

#include <Eigen/Dense>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <vector>

#include "b200fe.h"
#include "fe_absorption_cuda.hpp"
#include "hdfe/akm_kss_cuda.hpp"
#include "schwarz_demean.hpp"

namespace {

// One context per host thread, like the reference's thread_local workspace
// (src/fe_absorption_cuda.cu:1536).
b200fe_context* thread_ctx() {
    thread_local b200fe_context* ctx = nullptr;
    thread_local bool tried = false;
    if (!tried) {
        tried = true;
        if (b200fe_context_create(0, &ctx) != B200FE_OK) ctx = nullptr;
    }
    return ctx;
}

}  // namespace

namespace hdfe {
namespace detail {

bool cuda_backend_available() { return b200fe_device_available() != 0; }

bool absorb_fixed_effects_cuda(const Eigen::Ref<const Eigen::VectorXd>& y,
                               const Eigen::Ref<const Eigen::MatrixXd>& X,
                               const std::vector<GpuFeInput>& fe_inputs,
                               const Eigen::VectorXd* weights,
                               const std::vector<std::size_t>& sweep_order,
                               const HdfeOptions& options, AbsorptionMethod /*method*/,
                               AbsorptionResult& result) {
    try {
        const int64_t n = y.size();
        const int k = static_cast<int>(X.cols());
        if (X.rows() != n) return false;  // the reference requires ld == n
        if (fe_inputs.empty()) {
            result.y_tilde = y;
            result.X_tilde = X;
            result.iterations = 0;
            result.converged = true;
            return true;
        }
        if (fe_inputs.size() > B200FE_MAX_DIMS) return false;
        // saved FEs: the coefficient path of the reference (store_alphas,
        // src/fe_absorption_cuda.cu:2345-2349); its other retain mode returns
        // per-sweep means this solver does not form, so it fails closed
        const bool save_fe = options.retain_fixed_effects;
        if (save_fe && (options.fe_recovery_method != FeRecoveryMethod::Hybrid ||
                        k > options.savefe_fastpath_max_cols))
            return false;
        std::vector<const int32_t*> gids;
        std::vector<int32_t> levels;
        std::vector<const double*> zvals;
        std::vector<unsigned char> icpt;
        bool any_slope = false;
        for (const GpuFeInput& fe : fe_inputs) {
            if (!fe.group_ids) return false;
            if (fe.is_slope && !fe.slope_values) return false;
            any_slope = any_slope || fe.is_slope;
            gids.push_back(fe.group_ids);
            levels.push_back(fe.num_groups);
            zvals.push_back(fe.is_slope ? fe.slope_values : nullptr);
            icpt.push_back(fe.is_slope ? (fe.slope_has_intercept ? 1 : 0) : 1);
        }
        // saved FEs with slopes: not provided, fail closed
        if (any_slope && save_fe) return false;
        b200fe_context* ctx = thread_ctx();
        if (!ctx) return false;
        b200fe_options o;
        b200fe_default_options(&o);
        o.tol = options.tol > 0.0 ? options.tol : 1e-8;
        o.tolerance_mode = static_cast<int>(options.tolerance_mode);
        if (options.max_iter > 0) o.max_iter = options.max_iter;
        if (save_fe) {
            // recover_fixed_effects accepts the coefficients only if the
            // residual's group means stay below fe_tolerance (an absolute
            // check): solve two orders tighter than that
            const double fe_tol = options.fe_tolerance > 0.0 ? options.fe_tolerance : o.tol;
            o.tol = std::max(std::min(o.tol, fe_tol) * 1e-2, 1e-14);
            o.fe_linf_tol = 0.5 * fe_tol;  // every group mean within half the check's bound
        }
        // contiguous copies: Eigen::Ref may have an inner stride
        const Eigen::VectorXd yc = y;
        const Eigen::MatrixXd Xc = X;
        result.y_tilde.resize(n);
        result.X_tilde.resize(n, k);
        const std::size_t D = fe_inputs.size();
        std::vector<Eigen::MatrixXd> fe(save_fe ? D : 0);
        std::vector<double*> fe_ptr(D, nullptr);
        for (std::size_t d = 0; d < fe.size(); ++d) {
            fe[d].resize(levels[d], k + 1);  // column-major, column 0 for y
            fe_ptr[d] = fe[d].data();
        }
        b200fe_result r;
        const int rc =
            any_slope
                ? b200fe_absorb_slopes(ctx, yc.data(), k ? Xc.data() : nullptr, n, k,
                                       static_cast<int>(gids.size()), gids.data(), levels.data(),
                                       zvals.data(), icpt.data(),
                                       weights ? weights->data() : nullptr, &o,
                                       result.y_tilde.data(), k ? result.X_tilde.data() : nullptr,
                                       &r)
                : b200fe_absorb_fe(ctx, yc.data(), k ? Xc.data() : nullptr, n, k,
                                   static_cast<int>(gids.size()), gids.data(), levels.data(),
                                   weights ? weights->data() : nullptr, &o,
                                   result.y_tilde.data(), k ? result.X_tilde.data() : nullptr,
                                   save_fe ? fe_ptr.data() : nullptr, &r);
        if (rc != B200FE_OK && rc != B200FE_NOT_CONVERGED) return false;
        if (save_fe) {  // the fields the reference fills (src/fe_absorption_cuda.cu:4663-4690)
            result.fe_group_ids.assign(D, {});
            result.fe_weight_sums.assign(D, Eigen::VectorXd());
            result.fe_alpha_y.assign(D, Eigen::VectorXd());
            result.fe_alpha_X.assign(D, Eigen::MatrixXd());
            result.fe_means.clear();
            for (std::size_t d = 0; d < D; ++d) {
                const int G = levels[d];
                result.fe_group_ids[d].assign(fe_inputs[d].group_ids, fe_inputs[d].group_ids + n);
                result.fe_weight_sums[d].resize(G);
                if (fe_inputs[d].weight_sums) {
                    for (int g = 0; g < G; ++g) result.fe_weight_sums[d][g] = fe_inputs[d].weight_sums[g];
                } else {
                    result.fe_weight_sums[d].setZero();
                    for (int64_t i = 0; i < n; ++i)
                        result.fe_weight_sums[d][fe_inputs[d].group_ids[i]] +=
                            weights ? (*weights)[i] : 1.0;
                }
                result.fe_alpha_y[d] = fe[d].col(0);
                result.fe_alpha_X[d] = fe[d].rightCols(k);
            }
        }
        result.iterations = r.iterations;
        result.converged = rc == B200FE_OK;
        result.fe_levels.clear();
        for (std::size_t d = 0; d < fe_inputs.size(); ++d)
            result.fe_levels.push_back(fe_inputs[d].num_levels_present > 0
                                           ? fe_inputs[d].num_levels_present
                                           : fe_inputs[d].num_groups);
        result.sweep_order_used.assign(sweep_order.begin(), sweep_order.end());
        return true;
    } catch (...) {
        return false;
    }
}

bool absorb_fixed_effects_group_individual_cuda(
    const Eigen::Ref<const Eigen::VectorXd>& y, const Eigen::Ref<const Eigen::MatrixXd>& X,
    const std::vector<GpuFeInput>& standard_fe_inputs, const GroupIndividualStructure& gi,
    const Eigen::VectorXd* weights, const std::vector<std::size_t>& sweep_order,
    const HdfeOptions& options, AbsorptionMethod /*method*/, AbsorptionResult& result) {
    try {
        const int64_t n = y.size();
        const int k = static_cast<int>(X.cols());
        // the reference's own preconditions (src/fe_absorption_cuda.cu:4750-4770)
        if (X.rows() != n || gi.num_groups != n || gi.num_individuals <= 0 ||
            static_cast<int64_t>(gi.group_ptr.size()) != n + 1 ||
            static_cast<int64_t>(gi.group_scale.size()) != n ||
            static_cast<int64_t>(gi.individual_ptr.size()) != int64_t(gi.num_individuals) + 1 ||
            gi.group_individual.size() != gi.individual_group.size() ||
            static_cast<std::size_t>(gi.group_ptr.back()) != gi.group_individual.size())
            return false;
        if (standard_fe_inputs.size() > B200FE_MAX_DIMS) return false;
        std::vector<const int32_t*> gids;
        std::vector<int32_t> levels;
        for (const GpuFeInput& fe : standard_fe_inputs) {
            if (fe.is_slope || !fe.group_ids) return false;
            gids.push_back(fe.group_ids);
            levels.push_back(fe.num_groups);
        }
        b200fe_context* ctx = thread_ctx();
        if (!ctx) return false;
        b200fe_options o;
        b200fe_default_options(&o);
        o.tol = options.tol > 0.0 ? options.tol : 1e-8;
        o.tolerance_mode = static_cast<int>(options.tolerance_mode);
        if (options.max_iter > 0) o.max_iter = options.max_iter;
        b200fe_group_individual g;
        g.num_individuals = gi.num_individuals;
        g.num_edges = static_cast<int64_t>(gi.group_individual.size());
        g.group_ptr = gi.group_ptr.data();
        g.group_individual = gi.group_individual.data();
        g.individual_ptr = gi.individual_ptr.data();
        g.individual_group = gi.individual_group.data();
        g.group_scale = gi.group_scale.data();
        const Eigen::VectorXd yc = y;
        const Eigen::MatrixXd Xc = X;
        result.y_tilde.resize(n);
        result.X_tilde.resize(n, k);
        b200fe_result r;
        const int rc = b200fe_absorb_group_individual(
            ctx, yc.data(), k ? Xc.data() : nullptr, n, k, static_cast<int>(gids.size()),
            gids.data(), levels.data(), &g, weights ? weights->data() : nullptr, &o,
            result.y_tilde.data(), k ? result.X_tilde.data() : nullptr, &r);
        if (rc != B200FE_OK && rc != B200FE_NOT_CONVERGED) return false;
        result.iterations = r.iterations;
        result.converged = rc == B200FE_OK;
        result.sweep_order_used.assign(sweep_order.begin(), sweep_order.end());
        return true;
    } catch (...) {
        return false;
    }
}

static bool recovery_max_delta(const Eigen::Ref<const Eigen::VectorXd>& residual,
                               const std::vector<GpuFeInput>& fe_inputs,
                               const Eigen::VectorXd* weights,
                               const std::vector<std::size_t>& sweep_order, double& out) {
    try {
        b200fe_context* ctx = thread_ctx();
        if (!ctx || fe_inputs.size() > B200FE_MAX_DIMS) return false;
        std::vector<const int32_t*> gids;
        std::vector<int32_t> levels;
        for (const GpuFeInput& fe : fe_inputs) {
            if (fe.is_slope || !fe.group_ids) return false;
            gids.push_back(fe.group_ids);
            levels.push_back(fe.num_groups);
        }
        std::vector<int32_t> order(sweep_order.begin(), sweep_order.end());
        const Eigen::VectorXd rc = residual;
        return b200fe_fe_recovery_max_delta(ctx, rc.data(), rc.size(),
                                            static_cast<int>(gids.size()), gids.data(),
                                            levels.data(), weights ? weights->data() : nullptr,
                                            order.empty() ? nullptr : order.data(),
                                            &out) == B200FE_OK;
    } catch (...) {
        return false;
    }
}

bool fe_recovery_max_delta_cuda(const Eigen::Ref<const Eigen::VectorXd>& residual,
                                const std::vector<GpuFeInput>& fe_inputs,
                                const Eigen::VectorXd* weights,
                                const std::vector<std::size_t>& sweep_order,
                                double& out_max_delta) {
    return recovery_max_delta(residual, fe_inputs, weights, sweep_order, out_max_delta);
}

bool fe_recovery_max_delta_cuda_cached(const Eigen::Ref<const Eigen::VectorXd>& residual,
                                       const std::vector<GpuFeInput>& fe_inputs,
                                       const Eigen::VectorXd* weights,
                                       const std::vector<std::size_t>& sweep_order,
                                       double& out_max_delta) {
    return recovery_max_delta(residual, fe_inputs, weights, sweep_order, out_max_delta);
}

// The device shadow certificate is an optional cross-check the reference runs
// only when XHDFE_GPU_CERT_SHADOW=1; here it reports ERROR and the host
// certificate stays authoritative, as in the reference.
CudaCertShadowHandle* cuda_cert_shadow_begin(const double*, const double*, int, int, int,
                                             const double*, const int* const*,
                                             const double* const*, const int*, int,
                                             const double* const*, const unsigned char*) {
    return nullptr;
}

bool cuda_cert_shadow_finish(CudaCertShadowHandle*, const double*, const double*, double,
                             CudaCertShadowResult* out) {
    if (out) out->verdict = 3;
    return false;
}

void cuda_cert_shadow_abort(CudaCertShadowHandle*) {}

}  // namespace detail

namespace akm {

// The AKM/KSS firm-system solver (akm_kss_cuda.hpp:17-74) over the B200
// batched Jacobi-PCG (b200fe_kss_*): the same grounded system, stopping rule,
// per-lane iteration counts and failure reporting.
struct AkmCudaContext {
    b200fe_kss* kss = nullptr;
};

bool akm_cuda_available() { return b200fe_device_available() != 0; }

bool akm_cuda_stable_sort_u64(const std::uint64_t* keys, std::int64_t* order_out, std::size_t n) {
    if (n > static_cast<std::size_t>(INT32_MAX)) return false;
    return b200fe_stable_sort_u64(keys, order_out, static_cast<int64_t>(n)) == B200FE_OK;
}

AkmCudaContext* akm_cuda_create(int n_workers, int n_firms, const int* m_w, const int* m_f,
                                const double* m_c, std::size_t n_matches,
                                const std::int64_t* w_ptr, const std::int64_t* f_ptr,
                                const std::int64_t* f_matches, const double* Dw,
                                const double* Df, const double* inv_diagS) {
    try {
        b200fe_kss* k = nullptr;
        if (b200fe_kss_create(n_workers, n_firms, m_w, m_f, m_c, static_cast<int64_t>(n_matches),
                              w_ptr, f_ptr, f_matches, Dw, Df, inv_diagS, &k) != B200FE_OK)
            return nullptr;
        AkmCudaContext* c = new AkmCudaContext;
        c->kss = k;
        return c;
    } catch (...) {
        return nullptr;
    }
}

void akm_cuda_destroy(AkmCudaContext* ctx) {
    if (!ctx) return;
    b200fe_kss_destroy(ctx->kss);
    delete ctx;
}

int akm_cuda_solve_S(AkmCudaContext* ctx, const double* rhs, double* z, double tol, int max_iter) {
    if (!ctx) return -1;
    int it = -1;
    return b200fe_kss_solve(ctx->kss, rhs, z, tol, max_iter, &it) == B200FE_OK ? it : -1;
}

int akm_cuda_solve_S_multi(AkmCudaContext* ctx, const double* rhs_pack, double* z_pack, int nb,
                           double tol, int max_iter, int* iters_out) {
    if (!ctx) return -1;
    return b200fe_kss_solve_multi(ctx->kss, rhs_pack, z_pack, nb, tol, max_iter, iters_out) ==
                   B200FE_OK
               ? 0
               : -1;
}

int akm_cuda_max_lanes() { return b200fe_kss_max_lanes(); }

double* akm_cuda_pack_buffer(AkmCudaContext* ctx, int nb) {
    return ctx ? b200fe_kss_pack_buffer(ctx->kss, nb) : nullptr;
}

}  // namespace akm
}  // namespace hdfe

namespace xhdfe {

// The reference's raw in-place within-demean (include/schwarz_demean.hpp:30-34,
// src/schwarz_demean.cpp:419-438), called by its CPU absorber's Schwarz gate
// (src/fe_absorption.cpp:5199), on the B200 absorber (b200fe_demean_raw).  Same
// contract: Y (n) and X (n x k, column-major) overwritten with the unweighted
// within residuals on success, iters_out set; false with Y and X untouched when
// unsupported (fewer than two FE dims, n <= 0, k < 0, more than 16 columns,
// mismatched level list) or when the device solve fails or does not converge.
// threads and collapse select the reference's CPU factorisation and have no
// meaning here.
bool schwarz_demean_raw(double* Y, double* X, int64_t n, int k, const std::vector<const int32_t*>& fe,
                        const std::vector<int>& nlev, int threads, double tol, int max_iter,
                        int* iters_out, int collapse) {
    (void)threads;
    (void)collapse;
    if (fe.size() < 2 || nlev.size() != fe.size() || n <= 0 || k < 0 || k + 1 > 16 ||
        fe.size() > B200FE_MAX_DIMS || !Y || (k > 0 && !X))
        return false;
    try {
        std::vector<int32_t> G(nlev.begin(), nlev.end());
        std::vector<double> y(Y, Y + n);
        std::vector<double> x(X ? X : Y, X ? X + static_cast<std::size_t>(n) * k : Y);
        int its = 0;
        const int rc = b200fe_demean_raw(y.data(), k > 0 ? x.data() : nullptr, n, k,
                                         static_cast<int>(fe.size()), fe.data(), G.data(), tol,
                                         max_iter, &its);
        if (iters_out) *iters_out = its;
        if (rc != B200FE_OK) return false;
        std::copy(y.begin(), y.end(), Y);
        if (k > 0) std::copy(x.begin(), x.end(), X);
        return true;
    } catch (...) {
        return false;
    }
}

}  // namespace xhdfe
