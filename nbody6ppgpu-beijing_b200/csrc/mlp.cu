// mlp.cu -- training and inference of the learned neighbour-radius model
// (the network and its features are defined in mlp.cuh).
//
// Training is supervised regression on samples logged from plain
// Ahmad-Cohen runs: features of a particle at one regular step and the
// target dlog = log(RS*/RS), where RS* is the radius that would have given
// NNBOPT neighbours at its next regular step (estimated from the count that
// step found, nnb ~ RS^3).  Loss: mean squared error in standardised units.
//
//   mlp_grad_kernel   one warp per sample: bf16-weight forward pass, FP32
//                     backward pass; per-warp gradient buffers in shared
//                     memory, summed per CTA in a fixed order;
//   mlp_reduce        CTA partials summed in block order (deterministic);
//   mlp_adam          Adam step on the FP32 master copy, then the bf16 copy
//                     that every forward pass reads.
//
// The model is small (4,609 parameters, ~4.5 kFLOP per sample), so the
// passes run on the FP32 pipes: a batch of 1024 samples is ~10 MFLOP, far
// below what tensor-core tiling would pay for.
#include "nb6_common.cuh"
#include "mlp.cuh"

#include <algorithm>
#include <random>
#include <vector>

namespace {

constexpr int GW = 4;  // warps per CTA, gradient kernel
constexpr int MLP_SMEM_W2T = MLP_H * MLP_H * 2;  // transposed W2 (bf16) for the backward pass
constexpr size_t GRAD_SMEM = (size_t)MLP_SMEM_BYTES + MLP_SMEM_W2T + (size_t)GW * MLP_NPARAM * sizeof(float) +
                             GW * sizeof(float);

struct MlpState {
    bool have = false;      // parameters set or trained
    int enabled = 0;        // proposals in regular-force calls
    std::vector<float> host;  // FP32 parameters + moments
    DevBuf<float> w32, m1, m2, grad, part, norm, dx, dy, loss;
    DevBuf<__nv_bfloat16> w16;
    DevBuf<int> perm;
    long long adam_t = 0;
};
MlpState M;

__global__ void mlp_to_bf16(const float *__restrict__ w32, __nv_bfloat16 *__restrict__ w16) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < MLP_SMEM_BYTES / 2; k += gridDim.x * blockDim.x)
        w16[k] = __float2bfloat16_rn(k < MLP_NPARAM ? w32[k] : 0.0f);
}

// Gradient of sum_s (out_s - y_s)^2 / n over the samples [off, off + cnt)
// of the (optionally permuted) set; per-CTA partials into part[block][.],
// squared-error partials into part_loss[block].
__global__ void __launch_bounds__(GW * 32)
    mlp_grad_kernel(int cnt, int off, float inv_n, const float *__restrict__ x, const float *__restrict__ y,
                    const int *__restrict__ perm, const __nv_bfloat16 *__restrict__ w16,
                    const float *__restrict__ norm, float *__restrict__ part, float *__restrict__ part_loss) {
    extern __shared__ __align__(16) unsigned char smem[];
    __nv_bfloat16 *sw = reinterpret_cast<__nv_bfloat16 *>(smem);
    __nv_bfloat16 *w2t = reinterpret_cast<__nv_bfloat16 *>(smem + MLP_SMEM_BYTES);
    float *gbuf = reinterpret_cast<float *>(smem + MLP_SMEM_BYTES + MLP_SMEM_W2T);
    float *lbuf = gbuf + (size_t)GW * MLP_NPARAM;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    mlp_load(sw, w16);
    for (int k = threadIdx.x; k < MLP_H * MLP_H; k += blockDim.x) {
        const int kin = k / MLP_H, r = k % MLP_H;  // W2[kin][r] -> w2t[r][kin]
        w2t[r * MLP_H + kin] = w16[MLP_OFF_W2 + k];
    }
    float *g = gbuf + (size_t)warp * MLP_NPARAM;
    for (int k = lane; k < MLP_NPARAM; k += 32) g[k] = 0.0f;
    __syncthreads();
    float lsum = 0.0f;
    const float ymean = norm[2 * MLP_IN], yinv = 1.0f / norm[2 * MLP_IN + 1];
    for (int q = blockIdx.x * GW + warp; q < cnt; q += gridDim.x * GW) {
        const int s = perm ? perm[off + q] : off + q;
        float f[MLP_IN];
#pragma unroll
        for (int k = 0; k < MLP_IN; ++k) f[k] = x[(size_t)s * MLP_IN + k];
        MlpAct a;
        const float out = mlp_forward_warp(sw, norm, f, lane, a);
        const float err = out - (y[s] - ymean) * yinv;
        lsum += err * err;
        const float d = 2.0f * err * inv_n;
        if (lane == 0) g[MLP_OFF_B3] += d;
        float dz2[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int r = lane + 32 * u;
            g[MLP_OFF_W3 + r] += d * a.h2[u];
            dz2[u] = d * bf(sw, MLP_OFF_W3 + r) * mlp_dsilu(a.z2[u]);
            g[MLP_OFF_B2 + r] += dz2[u];
        }
        float dh1[2] = {0.0f, 0.0f};
#pragma unroll 8
        for (int k = 0; k < MLP_H; ++k) {
            const float hk = __shfl_sync(0xffffffffu, a.h1[k >> 5], k & 31);
            const float dk = __shfl_sync(0xffffffffu, dz2[k >> 5], k & 31);
            // dW2[k][r] for the lane's r; dh1 for the lane's k' via W2[k'][k] = w2t[k][k']
            g[MLP_OFF_W2 + k * MLP_H + lane] += dz2[0] * hk;
            g[MLP_OFF_W2 + k * MLP_H + lane + 32] += dz2[1] * hk;
            dh1[0] = fmaf(__bfloat162float(w2t[k * MLP_H + lane]), dk, dh1[0]);
            dh1[1] = fmaf(__bfloat162float(w2t[k * MLP_H + lane + 32]), dk, dh1[1]);
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int r = lane + 32 * u;
            const float dz1 = dh1[u] * mlp_dsilu(a.z1[u]);
            g[MLP_OFF_B1 + r] += dz1;
#pragma unroll
            for (int k = 0; k < MLP_IN; ++k) g[MLP_OFF_W1 + k * MLP_H + r] += dz1 * a.xn[k];
        }
    }
    if (lane == 0) lbuf[warp] = lsum;
    __syncthreads();
    float *p = part + (size_t)blockIdx.x * MLP_NPARAM;
    for (int k = threadIdx.x; k < MLP_NPARAM; k += blockDim.x) {
        float acc = 0.0f;
#pragma unroll
        for (int w = 0; w < GW; ++w) acc += gbuf[(size_t)w * MLP_NPARAM + k];
        p[k] = acc;
    }
    if (threadIdx.x == 0) {
        float l = 0.0f;
        for (int w = 0; w < GW; ++w) l += lbuf[w];
        part_loss[blockIdx.x] = l;
    }
}

// grad[k] = sum over blocks in block order; loss[0] += sum of squared errors.
__global__ void mlp_reduce(int nb, const float *__restrict__ part, const float *__restrict__ part_loss,
                           float *__restrict__ grad, float *__restrict__ loss) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < MLP_NPARAM) {
        float acc = 0.0f;
        for (int b = 0; b < nb; ++b) acc += part[(size_t)b * MLP_NPARAM + k];
        grad[k] = acc;
    }
    if (k == 0) {
        float l = 0.0f;
        for (int b = 0; b < nb; ++b) l += part_loss[b];
        loss[0] += l;
    }
}

__global__ void mlp_adam(float *__restrict__ w, float *__restrict__ m1, float *__restrict__ m2,
                         const float *__restrict__ g, float lr, float b1, float b2, float eps, float bc1,
                         float bc2) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= MLP_NPARAM) return;
    const float gk = g[k];
    const float a = b1 * m1[k] + (1.0f - b1) * gk;
    const float b = b2 * m2[k] + (1.0f - b2) * gk * gk;
    m1[k] = a;
    m2[k] = b;
    w[k] -= lr * (a / bc1) / (sqrtf(b / bc2) + eps);
}

__global__ void __launch_bounds__(128)
    mlp_predict_kernel(int n, const float *__restrict__ x, float *__restrict__ y,
                       const __nv_bfloat16 *__restrict__ w16, const float *__restrict__ norm) {
    __shared__ __align__(16) __nv_bfloat16 sw[MLP_SMEM_BYTES / 2];
    mlp_load(sw, w16);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int s = blockIdx.x * 4 + warp; s < n; s += gridDim.x * 4) {
        float f[MLP_IN];
#pragma unroll
        for (int k = 0; k < MLP_IN; ++k) f[k] = x[(size_t)s * MLP_IN + k];
        MlpAct a;
        const float out = mlp_forward_warp(sw, norm, f, lane, a);
        if (lane == 0) y[s] = out * norm[2 * MLP_IN + 1] + norm[2 * MLP_IN];
    }
}

void mlp_alloc() {
    if (M.w32.ptr) return;
    nb6_devinit_once(0);
    M.w32.reserve(MLP_NPARAM);
    M.m1.reserve(MLP_NPARAM);
    M.m2.reserve(MLP_NPARAM);
    M.grad.reserve(MLP_NPARAM);
    M.norm.reserve(MLP_NNORM);
    M.loss.reserve(1);
    M.w16.reserve(MLP_SMEM_BYTES / 2);
    M.host.assign(MLP_NPARAM + MLP_NNORM, 0.0f);
    NB6_CUDA_CHECK(cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)GRAD_SMEM));
}

// Host copy -> device FP32 master, moments and the bf16 copy; resets Adam.
void mlp_upload() {
    cudaStream_t st = nb6_stream();
    NB6_CUDA_CHECK(cudaMemcpyAsync(M.w32.ptr, M.host.data(), sizeof(float) * MLP_NPARAM,
                                   cudaMemcpyHostToDevice, st));
    NB6_CUDA_CHECK(cudaMemcpyAsync(M.norm.ptr, M.host.data() + MLP_NPARAM, sizeof(float) * MLP_NNORM,
                                   cudaMemcpyHostToDevice, st));
    NB6_CUDA_CHECK(cudaMemsetAsync(M.m1.ptr, 0, sizeof(float) * MLP_NPARAM, st));
    NB6_CUDA_CHECK(cudaMemsetAsync(M.m2.ptr, 0, sizeof(float) * MLP_NPARAM, st));
    mlp_to_bf16<<<(MLP_SMEM_BYTES / 2 + 255) / 256, 256, 0, st>>>(M.w32.ptr, M.w16.ptr);
    NB6_CUDA_CHECK(cudaGetLastError());
    NB6_CUDA_CHECK(cudaStreamSynchronize(st));
    M.adam_t = 0;
    M.have = true;
}

void mlp_download() {
    NB6_CUDA_CHECK(cudaStreamSynchronize(nb6_stream()));
    NB6_CUDA_CHECK(cudaMemcpy(M.host.data(), M.w32.ptr, sizeof(float) * MLP_NPARAM, cudaMemcpyDeviceToHost));
}

void mlp_upload_samples(int n, const float *x, const float *y) {
    M.dx.reserve((size_t)n * MLP_IN);
    NB6_CUDA_CHECK(cudaMemcpy(M.dx.ptr, x, sizeof(float) * MLP_IN * (size_t)n, cudaMemcpyHostToDevice));
    if (y) {
        M.dy.reserve(n);
        NB6_CUDA_CHECK(cudaMemcpy(M.dy.ptr, y, sizeof(float) * (size_t)n, cudaMemcpyHostToDevice));
    }
}

int grad_blocks(int cnt) { return std::max(1, std::min((cnt + GW * 8 - 1) / (GW * 8), nb6_num_sms() * 2)); }

// One gradient over samples [off, off+cnt) of the uploaded set into M.grad.
void mlp_grad_launch(int cnt, int off, const int *perm, cudaStream_t st) {
    const int nb = grad_blocks(cnt);
    M.part.reserve((size_t)nb * (MLP_NPARAM + 1));
    float *part_loss = M.part.ptr + (size_t)nb * MLP_NPARAM;
    mlp_grad_kernel<<<nb, GW * 32, GRAD_SMEM, st>>>(cnt, off, 1.0f / (float)cnt, M.dx.ptr, M.dy.ptr, perm,
                                                    M.w16.ptr, M.norm.ptr, M.part.ptr, part_loss);
    NB6_CUDA_CHECK(cudaGetLastError());
    mlp_reduce<<<(MLP_NPARAM + 255) / 256, 256, 0, st>>>(nb, M.part.ptr, part_loss, M.grad.ptr, M.loss.ptr);
    NB6_CUDA_CHECK(cudaGetLastError());
}

bool check_n(int n) {
    if (n <= 0) {
        nb6_fatal(NB6_ERR_BAD_ARG);
        return false;
    }
    return true;
}

}  // namespace

// Epilogue arguments for the regular-force call: proposals on when enabled
// and a model is loaded.
MlpArgs nb6_mlp_args(const double *h2, const double *dtr) {
    MlpArgs a;
    a.h2 = h2;
    a.dtr = dtr;
    a.w = M.w16.ptr;
    a.norm = M.norm.ptr;
    a.on = (M.enabled && M.have) ? 1 : 0;
    return a;
}

extern "C" {

// Number of floats of a model: parameters (see mlp.cuh for the layout)
// followed by the moments in_mean[5], in_scale[5], out_mean, out_std.
int nb6_mlp_size_(void) { return MLP_NPARAM + MLP_NNORM; }

// Random initial parameters (He-scaled normal, zero biases), identity moments.
void nb6_mlp_init_(int *seed) {
    mlp_alloc();
    std::mt19937 gen((unsigned)*seed);
    auto fill = [&](int off, int fan_in, int count) {
        std::normal_distribution<float> d(0.0f, std::sqrt(2.0f / (float)fan_in));
        for (int k = 0; k < count; ++k) M.host[off + k] = d(gen);
    };
    std::fill(M.host.begin(), M.host.end(), 0.0f);
    fill(MLP_OFF_W1, MLP_IN, MLP_IN * MLP_H);
    fill(MLP_OFF_W2, MLP_H, MLP_H * MLP_H);
    fill(MLP_OFF_W3, MLP_H, MLP_H);
    float *nm = M.host.data() + MLP_NPARAM;
    for (int k = 0; k < MLP_IN; ++k) nm[MLP_IN + k] = 1.0f;
    nm[2 * MLP_IN + 1] = 1.0f;
    mlp_upload();
}

void nb6_mlp_set_(const float *model) {
    mlp_alloc();
    std::copy(model, model + MLP_NPARAM + MLP_NNORM, M.host.begin());
    mlp_upload();
}

void nb6_mlp_get_(float *model) {
    if (!M.have) {
        nb6_fatal(NB6_ERR_NOT_OPEN);
        return;
    }
    mlp_download();
    std::copy(M.host.begin(), M.host.end(), model);
}

// Gradient of the mean squared error (standardised units) over n samples
// x[n][5], y[n] at the current parameters, and the loss.  Deterministic.
void nb6_mlp_grad_(int *n, const float *x, const float *y, float *grad, float *loss) {
    if (!M.have) {
        nb6_fatal(NB6_ERR_NOT_OPEN);
        return;
    }
    if (!check_n(*n)) return;
    mlp_upload_samples(*n, x, y);
    cudaStream_t st = nb6_stream();
    NB6_CUDA_CHECK(cudaMemsetAsync(M.loss.ptr, 0, sizeof(float), st));
    mlp_grad_launch(*n, 0, nullptr, st);
    NB6_CUDA_CHECK(cudaStreamSynchronize(st));
    NB6_CUDA_CHECK(cudaMemcpy(grad, M.grad.ptr, sizeof(float) * MLP_NPARAM, cudaMemcpyDeviceToHost));
    float l = 0.0f;
    NB6_CUDA_CHECK(cudaMemcpy(&l, M.loss.ptr, sizeof(float), cudaMemcpyDeviceToHost));
    *loss = l / (float)*n;
}

// Train on n samples: moments from the data, then `epochs` passes of Adam
// over shuffled mini-batches of `batch`.  loss_hist[e] = mean squared error
// (standardised) over epoch e.  Starts from the current parameters (call
// nb6_mlp_init_ first for a fresh model).
void nb6_mlp_train_(int *n_, const float *x, const float *y, int *epochs, int *batch, float *lr, int *seed,
                    float *loss_hist) {
    const int n = *n_, B = std::max(1, std::min(*batch, n));
    if (!check_n(n) || *epochs < 0) return;
    mlp_alloc();
    if (!M.have) {
        int s = *seed;
        nb6_mlp_init_(&s);
    }
    // moments of the inputs and the target
    float *nm = M.host.data() + MLP_NPARAM;
    for (int k = 0; k <= MLP_IN; ++k) {
        double s1 = 0.0, s2 = 0.0;
        for (int q = 0; q < n; ++q) {
            const double v = k < MLP_IN ? x[(size_t)q * MLP_IN + k] : y[q];
            s1 += v;
            s2 += v * v;
        }
        const double mean = s1 / n, var = std::max(s2 / n - mean * mean, 1e-12);
        if (k < MLP_IN) {
            nm[k] = (float)mean;
            nm[MLP_IN + k] = (float)(1.0 / std::sqrt(var));
        } else {
            nm[2 * MLP_IN] = (float)mean;
            nm[2 * MLP_IN + 1] = (float)std::sqrt(var);
        }
    }
    mlp_download();  // keep the device parameters, refresh the moments
    mlp_upload();
    mlp_upload_samples(n, x, y);
    M.perm.reserve(n);
    std::vector<int> perm(n);
    for (int q = 0; q < n; ++q) perm[q] = q;
    std::mt19937 gen((unsigned)*seed);
    cudaStream_t st = nb6_stream();
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int e = 0; e < *epochs; ++e) {
        std::shuffle(perm.begin(), perm.end(), gen);
        NB6_CUDA_CHECK(cudaMemcpyAsync(M.perm.ptr, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
        NB6_CUDA_CHECK(cudaMemsetAsync(M.loss.ptr, 0, sizeof(float), st));
        for (int off = 0; off + B <= n; off += B) {
            mlp_grad_launch(B, off, M.perm.ptr, st);
            M.adam_t++;
            const float bc1 = 1.0f - std::pow(b1, (float)M.adam_t);
            const float bc2 = 1.0f - std::pow(b2, (float)M.adam_t);
            mlp_adam<<<(MLP_NPARAM + 255) / 256, 256, 0, st>>>(M.w32.ptr, M.m1.ptr, M.m2.ptr, M.grad.ptr, *lr,
                                                               b1, b2, eps, bc1, bc2);
            NB6_CUDA_CHECK(cudaGetLastError());
            mlp_to_bf16<<<(MLP_SMEM_BYTES / 2 + 255) / 256, 256, 0, st>>>(M.w32.ptr, M.w16.ptr);
            NB6_CUDA_CHECK(cudaGetLastError());
        }
        float l = 0.0f;
        NB6_CUDA_CHECK(cudaStreamSynchronize(st));
        NB6_CUDA_CHECK(cudaMemcpy(&l, M.loss.ptr, sizeof(float), cudaMemcpyDeviceToHost));
        if (loss_hist) loss_hist[e] = l / (float)((n / B) * B);
    }
    mlp_download();
}

// y[n] = model output (dlog RS) for x[n][5], bf16 parameters, FP32 sums.
void nb6_mlp_predict_(int *n, const float *x, float *y) {
    if (!M.have) {
        nb6_fatal(NB6_ERR_NOT_OPEN);
        return;
    }
    if (!check_n(*n)) return;
    mlp_upload_samples(*n, x, nullptr);
    DevBuf<float> out;
    out.reserve(*n);
    cudaStream_t st = nb6_stream();
    const int blocks = std::max(1, std::min((*n + 3) / 4, nb6_num_sms() * 8));
    mlp_predict_kernel<<<blocks, 128, 0, st>>>(*n, M.dx.ptr, out.ptr, M.w16.ptr, M.norm.ptr);
    NB6_CUDA_CHECK(cudaGetLastError());
    NB6_CUDA_CHECK(cudaStreamSynchronize(st));
    NB6_CUDA_CHECK(cudaMemcpy(y, out.ptr, sizeof(float) * (size_t)*n, cudaMemcpyDeviceToHost));
    out.release();
}

// Radius proposals in regular-force calls on (1) or off (0).
void nb6_mlp_enable_(int *flag) {
    if (*flag && !M.have) {
        nb6_fatal(NB6_ERR_NOT_OPEN);
        return;
    }
    M.enabled = *flag ? 1 : 0;
}

}  // extern "C"
