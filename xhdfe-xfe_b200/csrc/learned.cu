// The learned warm start: the network's C-ABI entry points (forward pass,
// loss gradient, Adam step, installing trained parameters in a context) and
// the inference call the solver makes before its refinement loop.  Kernels in
// mlp_kernels.cuh; the features and the use of the prediction are in b200fe.cu
// (solve_block).  No counterpart in the reference.

#include "context.cuh"
#include "mlp_kernels.cuh"

using namespace b200fe;
using namespace b200fe_host;

namespace b200fe_host {

int mlp_forward_device(b200fe_context* ctx, const void* packed, const float* d_x, int64_t n, float* d_y) {
    if (n <= 0) return B200FE_OK;
    const int64_t tiles = (n + 15) / 16;
    const int grid = static_cast<int>(std::max<int64_t>(
        1, std::min<int64_t>((tiles + 7) / 8, static_cast<int64_t>(ctx->num_sms) * 8)));
    mlp_forward_kernel<<<grid, 256, 0, ctx->stream>>>(static_cast<const MlpPacked*>(packed), d_x, n, d_y);
    B_LAUNCHED();
    return B200FE_OK;
}

int mlp_pack_device(b200fe_context* ctx, const float* d_params, const char* name, void** packed) {
    MlpPacked* pk;
    B_CHECK(get_buf(ctx, name, 1, &pk));
    mlp_pack_kernel<<<(kMlpHid * kLdH + 255) / 256, 256, 0, ctx->stream>>>(d_params, pk);
    B_LAUNCHED();
    *packed = pk;
    return B200FE_OK;
}

}  // namespace b200fe_host

extern "C" {

int b200fe_mlp_num_params(void) { return kMlpParams; }

int b200fe_mlp_forward(b200fe_context* ctx, const float* d_params, const float* d_x, int64_t n,
                       float* d_y) {
    if (!ctx || !d_params || (n > 0 && (!d_x || !d_y)) || n < 0) return B200FE_INVALID_ARG;
    cudaGetLastError();
    cudaSetDevice(ctx->device);
    void* pk = nullptr;
    B_CHECK(mlp_pack_device(ctx, d_params, "mlp_packed_call", &pk));
    B_CHECK(mlp_forward_device(ctx, pk, d_x, n, d_y));
    B_TRY(cudaStreamSynchronize(ctx->stream));
    return B200FE_OK;
}

int b200fe_mlp_grad(b200fe_context* ctx, const float* d_params, const float* d_x, const float* d_targets,
                    int64_t n, double* d_grad_loss) {
    if (!ctx || !d_params || !d_x || !d_targets || !d_grad_loss || n <= 0) return B200FE_INVALID_ARG;
    cudaGetLastError();
    cudaSetDevice(ctx->device);
    const size_t smem = sizeof(MlpGradSmem);
    B_TRY(raise_smem_limit(reinterpret_cast<const void*>(&mlp_grad_kernel), static_cast<int>(smem)));
    const int64_t blocks = (n + kMlpBlock - 1) / kMlpBlock;
    const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(blocks, ctx->num_sms)));
    float* partial;
    B_CHECK(get_buf(ctx, "mlp_partial", static_cast<size_t>(grid) * (kMlpParams + 1), &partial));
    mlp_grad_kernel<<<grid, kMlpGradThreads, smem, ctx->stream>>>(d_params, d_x, d_targets, n,
                                                                  1.0f / static_cast<float>(n), partial);
    B_LAUNCHED();
    mlp_reduce_kernel<<<(kMlpParams + 256) / 256, 256, 0, ctx->stream>>>(partial, grid, d_grad_loss);
    B_LAUNCHED();
    B_TRY(cudaStreamSynchronize(ctx->stream));
    return B200FE_OK;
}

int b200fe_mlp_adam(b200fe_context* ctx, float* d_params, float* d_m, float* d_v, const double* d_grad,
                    int step, double lr) {
    if (!ctx || !d_params || !d_m || !d_v || !d_grad || step < 1 || !(lr > 0.0)) return B200FE_INVALID_ARG;
    cudaGetLastError();
    cudaSetDevice(ctx->device);
    mlp_adam_kernel<<<(kMlpParams + 255) / 256, 256, 0, ctx->stream>>>(d_params, d_m, d_v, d_grad, step, lr,
                                                                     0.9, 0.999, 1e-8);
    B_LAUNCHED();
    B_TRY(cudaStreamSynchronize(ctx->stream));
    return B200FE_OK;
}

int b200fe_warmstart_set(b200fe_context* ctx, const float* params, int mode) {
    if (!ctx || mode < 0 || mode > 3) return B200FE_INVALID_ARG;
    cudaGetLastError();
    cudaSetDevice(ctx->device);
    if (!params || mode == 0) {
        ctx->ws_mode = 0;
        ctx->ws_packed = nullptr;
        return B200FE_OK;
    }
    for (int i = 0; i < kMlpParams; ++i) {
        if (!std::isfinite(params[i])) {
            ctx->err = "warm-start parameters must be finite";
            return B200FE_INVALID_ARG;
        }
    }
    float* d_params;
    B_CHECK(get_buf(ctx, "ws_params", kMlpParams, &d_params));
    B_TRY(cudaMemcpyAsync(d_params, params, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice, ctx->stream));
    void* pk = nullptr;
    B_CHECK(mlp_pack_device(ctx, d_params, "mlp_packed_ws", &pk));
    B_TRY(cudaStreamSynchronize(ctx->stream));
    ctx->ws_packed = pk;
    ctx->ws_mode = mode;
    return B200FE_OK;
}

}  // extern "C"
