// mlp.cuh -- the learned neighbour-radius model shared by the training
// kernels (mlp.cu) and the regular-force epilogue (regular.cu).
//
// A 5 -> 64 -> 64 -> 1 perceptron with SiLU hidden units.  Parameters are
// kept in FP32 (master copy, optimiser) and used in bf16 by every forward
// pass; all sums accumulate in FP32.  One warp evaluates one sample: lane l
// owns hidden units l and l + 32 of both layers.
//
// Inputs (features of one particle at a regular step, all from quantities
// the regular-force call already has):
//   f0 = log(1 + nnb)            nnb = neighbour count (self included)
//   f1 = log(RS) = log(h2) / 2
//   f2 = log(1 + nnb) - 1.5 log(h2)   local density, ~ nnb / RS^3
//   f3 = log |a_reg|
//   f4 = -log2(dtr)              timestep level of the regular step
// Output: dlog = log(RS_next / RS), the change of the neighbour radius that
// should bring the next neighbour count to NNBOPT.  Inputs are standardised
// and the output de-standardised with the model's stored moments.
#pragma once

#include <cuda_bf16.h>
#include <math.h>

constexpr int MLP_IN = 5;
constexpr int MLP_H = 64;
// Flat parameter vector.  W1[k][r]: input k -> hidden-1 unit r;
// W2[k][r]: hidden-1 unit k -> hidden-2 unit r; W3[r]: hidden-2 unit r ->
// output.  (Input-major, so a warp reading one input row is conflict free.)
constexpr int MLP_OFF_W1 = 0;
constexpr int MLP_OFF_B1 = MLP_OFF_W1 + MLP_IN * MLP_H;   // 320
constexpr int MLP_OFF_W2 = MLP_OFF_B1 + MLP_H;            // 384
constexpr int MLP_OFF_B2 = MLP_OFF_W2 + MLP_H * MLP_H;    // 4480
constexpr int MLP_OFF_W3 = MLP_OFF_B2 + MLP_H;            // 4544
constexpr int MLP_OFF_B3 = MLP_OFF_W3 + MLP_H;            // 4608
constexpr int MLP_NPARAM = MLP_OFF_B3 + 1;                // 4609
// Moments: in_mean[5], in_scale[5] (1 / std), out_mean, out_std.
constexpr int MLP_NNORM = 2 * MLP_IN + 2;
// bf16 parameters in shared memory, padded to 16 bytes.
constexpr int MLP_SMEM_BYTES = ((MLP_NPARAM * 2 + 15) / 16) * 16;

// What the regular-force epilogue needs to propose radii: the call's h2 and
// dtr (device), the bf16 parameters and the moments.  on = 0: no proposal.
struct MlpArgs {
    const double *h2;
    const double *dtr;
    const __nv_bfloat16 *w;
    const float *norm;
    int on;
};

__device__ __forceinline__ float mlp_silu(float z) { return z / (1.0f + expf(-z)); }

// d silu / dz = s (1 + z (1 - s)), s = sigmoid(z)
__device__ __forceinline__ float mlp_dsilu(float z) {
    const float s = 1.0f / (1.0f + expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

// Features of one particle (see the header comment); nnb < 0 is read as |nnb|.
__host__ __device__ inline void mlp_features(double nnb, double h2, double a2, double dtr, float *f) {
    const double n = nnb < 0 ? -nnb : nnb;
    const double ln = log(1.0 + n);
    const double lh = log(h2 > 1e-300 ? h2 : 1e-300);
    f[0] = (float)ln;
    f[1] = (float)(0.5 * lh);
    f[2] = (float)(ln - 1.5 * lh);
    f[3] = (float)(0.5 * log(a2 > 1e-300 ? a2 : 1e-300));
    f[4] = (float)(-log2(dtr > 1e-300 ? dtr : 1e-300));
}

// Copy the bf16 parameters into shared memory (all threads of the CTA).
__device__ __forceinline__ void mlp_load(__nv_bfloat16 *sw, const __nv_bfloat16 *w) {
    const int4 *src = reinterpret_cast<const int4 *>(w);
    int4 *dst = reinterpret_cast<int4 *>(sw);
    for (int k = threadIdx.x; k < MLP_SMEM_BYTES / 16; k += blockDim.x) dst[k] = src[k];
}

// Activations one lane keeps for the backward pass.
struct MlpAct {
    float z1[2], h1[2], z2[2], h2[2];
    float xn[MLP_IN];
    float out;  // standardised output (same in every lane)
};

__device__ __forceinline__ float bf(const __nv_bfloat16 *p, int k) { return __bfloat162float(p[k]); }

// Warp forward pass on raw features f (every lane passes the same f).
// Returns the standardised output in every lane.
__device__ __forceinline__ float mlp_forward_warp(const __nv_bfloat16 *sw, const float *norm, const float *f,
                                                  int lane, MlpAct &a) {
#pragma unroll
    for (int k = 0; k < MLP_IN; ++k) a.xn[k] = (f[k] - norm[k]) * norm[MLP_IN + k];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
        const int r = lane + 32 * u;
        float z = bf(sw, MLP_OFF_B1 + r);
#pragma unroll
        for (int k = 0; k < MLP_IN; ++k) z = fmaf(bf(sw, MLP_OFF_W1 + k * MLP_H + r), a.xn[k], z);
        a.z1[u] = z;
        a.h1[u] = mlp_silu(z);
    }
    float z2a = bf(sw, MLP_OFF_B2 + lane), z2b = bf(sw, MLP_OFF_B2 + lane + 32);
#pragma unroll 8
    for (int k = 0; k < MLP_H; ++k) {
        const float hk = __shfl_sync(0xffffffffu, a.h1[k >> 5], k & 31);
        z2a = fmaf(bf(sw, MLP_OFF_W2 + k * MLP_H + lane), hk, z2a);
        z2b = fmaf(bf(sw, MLP_OFF_W2 + k * MLP_H + lane + 32), hk, z2b);
    }
    a.z2[0] = z2a;
    a.z2[1] = z2b;
    a.h2[0] = mlp_silu(z2a);
    a.h2[1] = mlp_silu(z2b);
    float o = bf(sw, MLP_OFF_W3 + lane) * a.h2[0] + bf(sw, MLP_OFF_W3 + lane + 32) * a.h2[1];
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) o += __shfl_xor_sync(0xffffffffu, o, s);
    a.out = o + bf(sw, MLP_OFF_B3);
    return a.out;
}
