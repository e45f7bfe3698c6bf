// potential.cu -- N^2 potential behind the reference's gpupot_ C ABI
// (gpupot.gpu.cu:116-127): pot[k] = sum_{j: r2 > 0} m_j / r_ij for
// i = istart-1+k, k in [0, ni).
//
// The j set (m, x) is copied once per call into device buffers that persist
// across calls (the reference allocates and frees per call,
// gpupot.gpu.cu:72-79,107-108), split into hi/lo SoA float4 tiles, and
// streamed through a 4-stage bulk-copy ring exactly like the regular kernel.
// Each thread holds NI i-particles; pair math is FP32 on hi/lo differences
// with rsqrt + one Newton step, FP32 partial sums fold into double-single
// accumulators per 128-j tile, slices are summed in FP64 in a fixed order.
#include "nb6_common.cuh"

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <string.h>

namespace {

constexpr int JT = 128;
constexpr int NSTAGE = 4;
constexpr int NT = 128;
constexpr unsigned long long WAIT_NS = 2000000000ull;

struct PotArgs {
    const float4 *__restrict__ posH;  // (xH, yH, zH, m)
    const float4 *__restrict__ posL;  // (xL, yL, zL, 0)
    int ntile, nslices;
    int i0, ni;                       // absolute first i (0-based), count
    float2 *__restrict__ part;        // [nslices][ni] (hi, lo)
    int *status;
};

template <int NI>
__global__ void __launch_bounds__(NT) pot_kernel(const PotArgs a) {
    __shared__ __align__(128) float4 sj[NSTAGE][2][JT];
    __shared__ __align__(8) uint64_t bar[NSTAGE];
    const int tid = threadIdx.x;
    const int slice = blockIdx.y;
    const int t_begin = (int)(((long long)slice * a.ntile) / a.nslices);
    const int t_end = (int)(((long long)(slice + 1) * a.ntile) / a.nslices);
    const int nt = t_end - t_begin;

    float xh[NI], yh[NI], zh[NI], xl[NI], yl[NI], zl[NI];
    float ph[NI], pl[NI], ps[NI];
    int ii[NI];
#pragma unroll
    for (int k = 0; k < NI; ++k) {
        const int i = blockIdx.x * (NT * NI) + k * NT + tid;
        ii[k] = i;
        ph[k] = pl[k] = ps[k] = 0.f;
        if (i < a.ni) {
            const float4 h = a.posH[a.i0 + i];
            const float4 l = a.posL[a.i0 + i];
            xh[k] = h.x; yh[k] = h.y; zh[k] = h.z;
            xl[k] = l.x; yl[k] = l.y; zl[k] = l.z;
        } else {
            xh[k] = yh[k] = zh[k] = xl[k] = yl[k] = zl[k] = 0.f;
        }
    }
    if (tid == 0) {
#pragma unroll
        for (int st = 0; st < NSTAGE; ++st) mbar_init(&bar[st], 1);
        fence_mbar_init();
    }
    __syncthreads();
    auto issue = [&](int st, int tile) {
        const size_t off = (size_t)tile * JT;
        mbar_arrive_expect_tx(&bar[st], 2u * JT * sizeof(float4));
        bulk_g2s(sj[st][0], a.posH + off, JT * sizeof(float4), &bar[st]);
        bulk_g2s(sj[st][1], a.posL + off, JT * sizeof(float4), &bar[st]);
    };
    if (tid == 0)
        for (int st = 0; st < NSTAGE && st < nt; ++st) issue(st, t_begin + st);

    for (int t = 0; t < nt; ++t) {
        const int st = t % NSTAGE;
        const bool ok = mbar_wait_timed(&bar[st], (uint32_t)((t / NSTAGE) & 1), WAIT_NS);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                set_status(a.status, NB6_ERR_WAIT_TIMEOUT);
                const int issued = min(nt, NSTAGE + max(t - 1, 0));
                for (int u = t; u < issued; ++u)
                    mbar_wait_timed(&bar[u % NSTAGE], (uint32_t)((u / NSTAGE) & 1), WAIT_NS / 8);
            }
            return;
        }
        if (tid == 0 && t >= 1 && t - 1 + NSTAGE < nt) issue((t - 1) % NSTAGE, t_begin + t - 1 + NSTAGE);
        const float4 *A = sj[st][0];
        const float4 *B = sj[st][1];
#pragma unroll 8
        for (int q = 0; q < JT; ++q) {
            const float4 h = A[q];
            const float4 l = B[q];
#pragma unroll
            for (int k = 0; k < NI; ++k) {
                const float dx = (h.x - xh[k]) + (l.x - xl[k]);
                const float dy = (h.y - yh[k]) + (l.y - yl[k]);
                const float dz = (h.z - zh[k]) + (l.z - zl[k]);
                const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                float y = rsqrt2_nr(r2);          // 2/r
                y = (r2 > 0.f) ? y : 0.f;         // gpupot.gpu.cu:52 skips r2 == 0
                ps[k] = fmaf(h.w, y, ps[k]);
            }
        }
#pragma unroll
        for (int k = 0; k < NI; ++k) {
            ds_fold(ph[k], pl[k], ps[k]);
            ps[k] = 0.f;
        }
    }
#pragma unroll
    for (int k = 0; k < NI; ++k)
        if (ii[k] < a.ni) a.part[(size_t)slice * a.ni + ii[k]] = make_float2(ph[k], pl[k]);
}

__global__ void pot_finalize(const float2 *__restrict__ part, int nslices, int ni,
                             double *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ni) return;
    double s = 0.0;
    for (int sl = 0; sl < nslices; ++sl) {
        const float2 p = part[(size_t)sl * ni + i];
        s += (double)p.x + (double)p.y;
    }
    out[i] = 0.5 * s;  // undo the 2/r scaling of rsqrt2_nr
}

__global__ void pot_pack(int n, int npad, const double *__restrict__ m,
                         const double *__restrict__ x, float4 *__restrict__ posH,
                         float4 *__restrict__ posL, int *status) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < npad; j += gridDim.x * blockDim.x) {
        if (j < n) {
            const double x0 = x[3 * j], x1 = x[3 * j + 1], x2 = x[3 * j + 2], mj = m[j];
            if (x0 != x0 || x1 != x1 || x2 != x2 || mj != mj) set_status(status, NB6_ERR_NAN_INPUT);
            float4 h, l;
            split_hl(x0, h.x, l.x);
            split_hl(x1, h.y, l.y);
            split_hl(x2, h.z, l.z);
            h.w = (float)mj;
            l.w = 0.f;
            posH[j] = h;
            posL[j] = l;
        } else {
            posH[j] = make_float4(1.0e15f, 1.0e15f, 1.0e15f, 0.f);
            posL[j] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
    }
}

// ----------------------------------------------------------------------------
// Ordered path (the whole set, n >= POT_ORDER_MIN): the bodies in Morton
// order with one bounding box per 128-body tile, as the regular force orders
// its j set.  A (warp, tile) whose box is at least one half extent away
// from every lane's i takes the packed far loop: differences from
// tile-relative coordinates fl32(x_j - c) (stored) and fl32(x_i - c)
// (formed in FP64 per tile), one FP32 add each instead of three, within 4
// FP32 ulps of the FP64-formed difference (|x_j - c| <= h <= r), and two j
// per f32x2 instruction.  Other tiles take the hi/lo loop above.  Results
// are written back in the caller's order.
// ----------------------------------------------------------------------------
constexpr int POT_ORDER_MIN = 32768;

NB6_DEV float2 pair2(float v) { return make_float2(v, v); }

__global__ void pot_extent(int n, const double *__restrict__ x, unsigned *__restrict__ ext) {
    unsigned mn[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, mx[3] = {0u, 0u, 0u};
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const unsigned o = f2ord((float)x[3 * (size_t)j + k]);
            mn[k] = min(mn[k], o);
            mx[k] = max(mx[k], o);
        }
#pragma unroll
    for (int k = 0; k < 3; ++k)
        for (int o = 16; o > 0; o >>= 1) {
            mn[k] = min(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
            mx[k] = max(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
        }
    if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            atomicMin(&ext[k], mn[k]);
            atomicMax(&ext[3 + k], mx[k]);
        }
}

__global__ void pot_keys(int n, const double *__restrict__ x, const unsigned *__restrict__ ext,
                         unsigned *__restrict__ keys, int *__restrict__ vals) {
    float lo[3], sc[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        lo[k] = ord2f(ext[k]);
        const float w = ord2f(ext[3 + k]) - lo[k];
        sc[k] = w > 0.f ? 1023.99f / w : 0.f;
    }
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        unsigned key = 0;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float f = ((float)x[3 * (size_t)j + k] - lo[k]) * sc[k];
            key |= spread10((unsigned)fminf(fmaxf(f, 0.f), 1023.f)) << k;
        }
        keys[j] = key;
        vals[j] = j;
    }
}

// Ordered hi/lo layout (+ mass) and FP64 positions; padding slots massless
// and far away.
__global__ void pot_permute(int n, int npad, const int *__restrict__ perm, const double *__restrict__ m,
                            const double *__restrict__ x, float4 *__restrict__ posH, float4 *__restrict__ posL,
                            double *__restrict__ xs) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < npad; s += gridDim.x * blockDim.x) {
        if (s < n) {
            const int j = perm[s];
            const double x0 = x[3 * (size_t)j], x1 = x[3 * (size_t)j + 1], x2 = x[3 * (size_t)j + 2];
            float4 h, l;
            split_hl(x0, h.x, l.x);
            split_hl(x1, h.y, l.y);
            split_hl(x2, h.z, l.z);
            h.w = (float)m[j];
            l.w = 0.f;
            posH[s] = h;
            posL[s] = l;
            xs[3 * (size_t)s] = x0;
            xs[3 * (size_t)s + 1] = x1;
            xs[3 * (size_t)s + 2] = x2;
        } else {
            posH[s] = make_float4(1.0e15f, 1.0e15f, 1.0e15f, 0.f);
            posL[s] = make_float4(0.f, 0.f, 0.f, 0.f);
            xs[3 * (size_t)s] = xs[3 * (size_t)s + 1] = xs[3 * (size_t)s + 2] = 1.0e15;
        }
    }
}

// One warp per tile: box of the hi positions of its real bodies (centre
// rounded to nearest, half extents rounded up).
__global__ void pot_boxes(int n, int ntile, const float4 *__restrict__ posH, float4 *__restrict__ tbox) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= ntile) return;
    double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
    for (int q = lane; q < JT; q += 32) {
        const int k = warp * JT + q;
        if (k >= n) break;
        const float4 p = posH[k];
        const double c[3] = {p.x, p.y, p.z};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            mn[d] = fmin(mn[d], c[d]);
            mx[d] = fmax(mx[d], c[d]);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            mn[d] = fmin(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
            mx[d] = fmax(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o));
        }
    if (lane == 0) {
        tbox[2 * warp] = make_float4(__double2float_rn(0.5 * (mn[0] + mx[0])), __double2float_rn(0.5 * (mn[1] + mx[1])),
                                     __double2float_rn(0.5 * (mn[2] + mx[2])), 0.f);
        tbox[2 * warp + 1] = make_float4(__double2float_ru(0.5 * (mx[0] - mn[0])), __double2float_ru(0.5 * (mx[1] - mn[1])),
                                         __double2float_ru(0.5 * (mx[2] - mn[2])), 0.f);
    }
}

// Tile-relative positions and masses, component-major rows (xr, yr, zr, m)
// of npad floats each.
__global__ void pot_rel(int npad, const double *__restrict__ xs, const float4 *__restrict__ posH,
                        const float4 *__restrict__ tbox, float *__restrict__ rel) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < npad; s += gridDim.x * blockDim.x) {
        const float4 c = tbox[2 * (s / JT)];
        rel[s] = __double2float_rn(xs[3 * (size_t)s] - (double)c.x);
        rel[(size_t)npad + s] = __double2float_rn(xs[3 * (size_t)s + 1] - (double)c.y);
        rel[2 * (size_t)npad + s] = __double2float_rn(xs[3 * (size_t)s + 2] - (double)c.z);
        rel[3 * (size_t)npad + s] = posH[s].w;
    }
}

struct PotOrdArgs {
    const float4 *__restrict__ posH;  // ordered (xH, yH, zH, m)
    const float4 *__restrict__ posL;  // ordered (xL, yL, zL, 0)
    const float *__restrict__ rel;    // ordered rows xr, yr, zr, m (4 x npad)
    const double *__restrict__ xs;    // ordered FP64 positions
    const float4 *__restrict__ tbox;  // per tile: (centre, 0), (half extents, 0)
    size_t npad;
    int n, ntile, nslices;
    float2 *__restrict__ part;        // [nslices][n] over ordered slots
    int *status;
};

__global__ void __launch_bounds__(NT) pot_kernel_ord(const PotOrdArgs a) {
    __shared__ __align__(128) float4 sh[NSTAGE][2][JT];
    __shared__ __align__(128) float sr[NSTAGE][4][JT];
    __shared__ __align__(8) uint64_t bar[NSTAGE];
    const int tid = threadIdx.x, lane = tid & 31;
    const int slice = blockIdx.y;
    // tiles of this slice: every nslices-th (the near tiles of a compact
    // group of i are dealt out among the slices)
    const int nt = slice < a.ntile ? (a.ntile - slice + a.nslices - 1) / a.nslices : 0;
    const int s = blockIdx.x * NT + tid;
    const bool on = s < a.n;
    float xh = 0.f, yh = 0.f, zh = 0.f, xl = 0.f, yl = 0.f, zl = 0.f;
    double xd = 0.0, yd = 0.0, zd = 0.0;
    if (on) {
        const float4 h = a.posH[s], l = a.posL[s];
        xh = h.x; yh = h.y; zh = h.z;
        xl = l.x; yl = l.y; zl = l.z;
        xd = a.xs[3 * (size_t)s];
        yd = a.xs[3 * (size_t)s + 1];
        zd = a.xs[3 * (size_t)s + 2];
    }
    float ph = 0.f, pl = 0.f;
    if (tid == 0) {
#pragma unroll
        for (int st = 0; st < NSTAGE; ++st) mbar_init(&bar[st], 1);
        fence_mbar_init();
    }
    __syncthreads();
    auto issue = [&](int st, int tile) {
        const size_t off = (size_t)tile * JT;
        mbar_arrive_expect_tx(&bar[st], 2u * JT * sizeof(float4) + 4u * JT * sizeof(float));
        bulk_g2s(sh[st][0], a.posH + off, JT * sizeof(float4), &bar[st]);
        bulk_g2s(sh[st][1], a.posL + off, JT * sizeof(float4), &bar[st]);
#pragma unroll
        for (int c = 0; c < 4; ++c) bulk_g2s(sr[st][c], a.rel + (size_t)c * a.npad + off, JT * sizeof(float), &bar[st]);
    };
    if (tid == 0)
        for (int st = 0; st < NSTAGE && st < nt; ++st) issue(st, slice + st * a.nslices);

    for (int t = 0; t < nt; ++t) {
        const int st = t % NSTAGE;
        const bool ok = mbar_wait_timed(&bar[st], (uint32_t)((t / NSTAGE) & 1), WAIT_NS);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                set_status(a.status, NB6_ERR_WAIT_TIMEOUT);
                const int issued = min(nt, NSTAGE + max(t - 1, 0));
                for (int u = t; u < issued; ++u)
                    mbar_wait_timed(&bar[u % NSTAGE], (uint32_t)((u / NSTAGE) & 1), WAIT_NS / 8);
            }
            return;
        }
        if (tid == 0 && t >= 1 && t - 1 + NSTAGE < nt) issue((t - 1) % NSTAGE, slice + (t - 1 + NSTAGE) * a.nslices);
        const int tile = slice + t * a.nslices;
        const float4 bc = __ldg(&a.tbox[2 * tile]), bh = __ldg(&a.tbox[2 * tile + 1]);
        // far: the box at least one half extent from this lane's i (with a
        // margin for the FP32 test); padding lanes are far
        const float ex = fmaxf(fabsf(xh - bc.x) - bh.x, 0.f);
        const float ey = fmaxf(fabsf(yh - bc.y) - bh.y, 0.f);
        const float ez = fmaxf(fabsf(zh - bc.z) - bh.z, 0.f);
        const float hm = fmaxf(fmaxf(bh.x, bh.y), bh.z);
        const bool far = __all_sync(0xffffffffu, !on || ex * ex + ey * ey + ez * ez > 1.01f * hm * hm);
        float p;
        if (far) {
            const float2 nxr = pair2(-__double2float_rn(xd - (double)bc.x));
            const float2 nyr = pair2(-__double2float_rn(yd - (double)bc.y));
            const float2 nzr = pair2(-__double2float_rn(zd - (double)bc.z));
            float2 acc = make_float2(0.f, 0.f);  // sum m / r, lane = j parity
#pragma unroll 4
            for (int q = 0; q < JT; q += 4) {
                const float4 X = *reinterpret_cast<const float4 *>(&sr[st][0][q]);
                const float4 Y = *reinterpret_cast<const float4 *>(&sr[st][1][q]);
                const float4 Z = *reinterpret_cast<const float4 *>(&sr[st][2][q]);
                const float4 M = *reinterpret_cast<const float4 *>(&sr[st][3][q]);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const float2 xr = h ? make_float2(X.z, X.w) : make_float2(X.x, X.y);
                    const float2 yr = h ? make_float2(Y.z, Y.w) : make_float2(Y.x, Y.y);
                    const float2 zr = h ? make_float2(Z.z, Z.w) : make_float2(Z.x, Z.y);
                    const float2 mm = h ? make_float2(M.z, M.w) : make_float2(M.x, M.y);
                    const float2 dx = __fadd2_rn(xr, nxr);
                    const float2 dy = __fadd2_rn(yr, nyr);
                    const float2 dz = __fadd2_rn(zr, nzr);
                    const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
                    // 1/r straight from rsqrt.approx: every term of the
                    // sum is positive, so its relative error bound carries
                    // over to the sum unamplified (no Newton step needed,
                    // unlike the cancelling force sums)
                    float2 y0;
                    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y0.x) : "f"(r2.x));
                    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y0.y) : "f"(r2.y));
                    acc = __ffma2_rn(mm, y0, acc);
                }
            }
            p = 2.0f * (acc.x + acc.y);  // the 2/r units of the hi/lo loop
        } else {
            const float4 *A = sh[st][0];
            const float4 *B = sh[st][1];
            float ps = 0.f;
#pragma unroll 8
            for (int q = 0; q < JT; ++q) {
                const float4 h = A[q];
                const float4 l = B[q];
                const float dx = (h.x - xh) + (l.x - xl);
                const float dy = (h.y - yh) + (l.y - yl);
                const float dz = (h.z - zh) + (l.z - zl);
                const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                float y = rsqrt2_nr(r2);          // 2/r
                y = (r2 > 0.f) ? y : 0.f;         // gpupot.gpu.cu:52 skips r2 == 0
                ps = fmaf(h.w, y, ps);
            }
            p = ps;
        }
        ds_fold(ph, pl, p);
        (void)lane;
    }
    if (on) a.part[(size_t)slice * a.n + s] = make_float2(ph, pl);
}

// Sum of the slices of ordered slot s, written to the caller's index perm[s].
__global__ void pot_finalize_ord(const float2 *__restrict__ part, int nslices, int n, const int *__restrict__ perm,
                                 double *__restrict__ out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    double v = 0.0;
    for (int sl = 0; sl < nslices; ++sl) {
        const float2 p = part[(size_t)sl * n + s];
        v += (double)p.x + (double)p.y;
    }
    out[perm[s]] = 0.5 * v;
}

struct PotState {
    DevBuf<double> m, x, out;
    DevBuf<float4> posH, posL;
    DevBuf<float2> part;
    HostBuf<double> hout;
    int n = 0, ntile = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float last_ms = 0.f;
    // ordered set (whole-set calls with n >= POT_ORDER_MIN)
    const double *dm = nullptr, *dx = nullptr;  // the uploaded m, x of the call
    DevBuf<float4> posH_s, posL_s, tbox;
    DevBuf<float> rel;
    DevBuf<double> xs;
    DevBuf<unsigned> keys_in, keys_out, ext;
    DevBuf<int> vals_in, perm;
    DevBuf<char> sort_tmp;
};
PotState P;

// Build the ordered set of the uploaded bodies (P.dm, P.dx, P.n).
void pot_order(cudaStream_t st) {
    const int n = P.n;
    const size_t npad = (size_t)P.ntile * JT;
    P.keys_in.reserve(n);
    P.keys_out.reserve(n);
    P.vals_in.reserve(n);
    P.perm.reserve(n);
    P.ext.reserve(6);
    P.posH_s.reserve(npad);
    P.posL_s.reserve(npad);
    P.xs.reserve(3 * npad);
    P.rel.reserve(4 * npad);
    P.tbox.reserve(2 * (size_t)P.ntile);
    const unsigned init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    NB6_CUDA_CHECK(cudaMemcpyAsync(P.ext.ptr, init, sizeof(init), cudaMemcpyHostToDevice, st));
    const int blocks = std::max(1, std::min((n + 255) / 256, nb6_num_sms() * 8));
    pot_extent<<<blocks, 256, 0, st>>>(n, P.dx, P.ext.ptr);
    pot_keys<<<blocks, 256, 0, st>>>(n, P.dx, P.ext.ptr, P.keys_in.ptr, P.vals_in.ptr);
    NB6_CUDA_CHECK(cudaGetLastError());
    size_t tmp = 0;
    NB6_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, tmp, P.keys_in.ptr, P.keys_out.ptr, P.vals_in.ptr,
                                                   P.perm.ptr, n, 0, 30, st));
    P.sort_tmp.reserve(tmp + 16);
    NB6_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(P.sort_tmp.ptr, tmp, P.keys_in.ptr, P.keys_out.ptr,
                                                   P.vals_in.ptr, P.perm.ptr, n, 0, 30, st));
    const int pblocks = (int)std::min<size_t>((npad + 255) / 256, (size_t)nb6_num_sms() * 8);
    pot_permute<<<pblocks, 256, 0, st>>>(n, (int)npad, P.perm.ptr, P.dm, P.dx, P.posH_s.ptr, P.posL_s.ptr, P.xs.ptr);
    pot_boxes<<<(P.ntile * 32 + 255) / 256, 256, 0, st>>>(n, P.ntile, P.posH_s.ptr, P.tbox.ptr);
    pot_rel<<<pblocks, 256, 0, st>>>((int)npad, P.xs.ptr, P.posH_s.ptr, P.tbox.ptr, P.rel.ptr);
    NB6_CUDA_CHECK(cudaGetLastError());
}

int pot_ord_occ() {
    static int occ = -1;
    if (occ < 0) {
        NB6_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, pot_kernel_ord, NT, 0));
        if (occ < 1) occ = 1;
    }
    return occ;
}

// Potential of every body, ordered path; result in P.out (caller's order).
void pot_device_ord(cudaStream_t st) {
    const int n = P.n;
    const int nitile = (n + NT - 1) / NT;
    int nslices = std::max(1, nb6_num_sms() * pot_ord_occ() / nitile);
    nslices = std::min(nslices, P.ntile);
    P.part.reserve((size_t)nslices * n);
    P.out.reserve(n);
    PotOrdArgs a;
    a.posH = P.posH_s.ptr;
    a.posL = P.posL_s.ptr;
    a.rel = P.rel.ptr;
    a.xs = P.xs.ptr;
    a.tbox = P.tbox.ptr;
    a.npad = (size_t)P.ntile * JT;
    a.n = n;
    a.ntile = P.ntile;
    a.nslices = nslices;
    a.part = P.part.ptr;
    a.status = nb6_dev_status();
    pot_kernel_ord<<<dim3(nitile, nslices), NT, 0, st>>>(a);
    NB6_CUDA_CHECK(cudaGetLastError());
    pot_finalize_ord<<<(n + 255) / 256, 256, 0, st>>>(P.part.ptr, nslices, n, P.perm.ptr, P.out.ptr);
    NB6_CUDA_CHECK(cudaGetLastError());
}

template <int NI> int pot_occ() {
    static int occ = -1;
    if (occ < 0) {
        NB6_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, pot_kernel<NI>, NT, 0));
        if (occ < 1) occ = 1;
    }
    return occ;
}

// The whole set of a large call takes the ordered path (NB6_POT_ORDER=0:
// never).
bool pot_ordered(int i0, int ni) {
    static const int ordered = [] {
        const char *e = getenv("NB6_POT_ORDER");
        return (e && atoi(e) == 0) ? 0 : 1;
    }();
    return ordered && i0 == 0 && ni == P.n && P.n >= POT_ORDER_MIN;
}

// Potential of i in [i0, i0+ni) against the packed j set; result in P.out.
// The whole set of a large call takes the ordered path (built by
// pot_prepare).
void pot_device(int i0, int ni, cudaStream_t st) {
    if (pot_ordered(i0, ni)) {
        pot_device_ord(st);
        return;
    }
    int NI = 1;
    for (int c : {4, 2, 1}) {
        const int tile = NT * c;
        const int nit = (ni + tile - 1) / tile;
        if ((double)ni / ((double)nit * tile) >= 0.9 || c == 1) {
            NI = c;
            break;
        }
    }
    const int tile = NT * NI;
    const int nitile = (ni + tile - 1) / tile;
    const int occ = NI == 4 ? pot_occ<4>() : NI == 2 ? pot_occ<2>() : pot_occ<1>();
    int nslices = std::max(1, nb6_num_sms() * occ / nitile);
    nslices = std::min(nslices, P.ntile);
    P.part.reserve((size_t)nslices * ni);
    P.out.reserve(ni);
    PotArgs a;
    a.posH = P.posH.ptr;
    a.posL = P.posL.ptr;
    a.ntile = P.ntile;
    a.nslices = nslices;
    a.i0 = i0;
    a.ni = ni;
    a.part = P.part.ptr;
    a.status = nb6_dev_status();
    dim3 grid(nitile, nslices);
    if (NI == 4) pot_kernel<4><<<grid, NT, 0, st>>>(a);
    else if (NI == 2) pot_kernel<2><<<grid, NT, 0, st>>>(a);
    else pot_kernel<1><<<grid, NT, 0, st>>>(a);
    NB6_CUDA_CHECK(cudaGetLastError());
    pot_finalize<<<(ni + 255) / 256, 256, 0, st>>>(P.part.ptr, nslices, ni, P.out.ptr);
    NB6_CUDA_CHECK(cudaGetLastError());
}

// The bodies of a call on the device (copied from the host when they are
// there); pot_prepare then packs (and orders) them.
void pot_upload(int n, const double *m, const double *x, cudaStream_t st, bool from_host) {
    P.n = n;
    P.ntile = std::max(1, (n + JT - 1) / JT);
    const size_t npad = (size_t)P.ntile * JT;
    const double *dm = m, *dx = x;
    if (from_host) {
        P.m.reserve(npad);
        P.x.reserve(3 * npad);
        if (n > 0) {
            NB6_CUDA_CHECK(cudaMemcpyAsync(P.m.ptr, m, sizeof(double) * n, cudaMemcpyHostToDevice, st));
            NB6_CUDA_CHECK(cudaMemcpyAsync(P.x.ptr, x, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, st));
        }
        dm = P.m.ptr;
        dx = P.x.ptr;
    }
    P.dm = dm;
    P.dx = dx;
}

void pot_prepare(int i0, int ni, cudaStream_t st) {
    const int n = P.n;
    const size_t npad = (size_t)P.ntile * JT;
    const double *dm = P.dm, *dx = P.dx;
    P.posH.reserve(npad);
    P.posL.reserve(npad);
    const int blocks = (int)std::min<size_t>((npad + 255) / 256, (size_t)nb6_num_sms() * 8);
    pot_pack<<<blocks, 256, 0, st>>>(n, (int)npad, dm, dx, P.posH.ptr, P.posL.ptr, nb6_dev_status());
    NB6_CUDA_CHECK(cudaGetLastError());
    if (pot_ordered(i0, ni)) pot_order(st);
}

}  // namespace

extern "C" {

void gpupot_(int *irank, int *istart, int *ni_, int *n_, double *m, double (*x)[3], double *pot) {
    nb6_devinit_once(irank ? *irank : 0);
    const int n = *n_, ni = *ni_, i0 = *istart - 1;
    if (n <= 0 || ni <= 0 || i0 < 0 || i0 + ni > n) {
        fprintf(stderr, "gpupot: bad range istart=%d ni=%d n=%d\n", *istart, ni, n);
        nb6_fatal(NB6_ERR_BAD_ARG);
        return;
    }
    const double t0 = nb6_wtime();
    cudaStream_t st = nb6_stream();
    if (!P.ev0) {
        NB6_CUDA_CHECK(cudaEventCreate(&P.ev0));
        NB6_CUDA_CHECK(cudaEventCreate(&P.ev1));
    }
    pot_upload(n, m, &x[0][0], st, true);
    NB6_CUDA_CHECK(cudaEventRecord(P.ev0, st));
    pot_prepare(i0, ni, st);
    pot_device(i0, ni, st);
    NB6_CUDA_CHECK(cudaEventRecord(P.ev1, st));
    P.hout.reserve(ni);
    NB6_CUDA_CHECK(cudaMemcpyAsync(P.hout.ptr, P.out.ptr, sizeof(double) * ni, cudaMemcpyDeviceToHost, st));
    NB6_CUDA_CHECK(cudaStreamSynchronize(st));
    NB6_CUDA_CHECK(cudaEventElapsedTime(&P.last_ms, P.ev0, P.ev1));
    if (nb6_check_dev_status() != 0) return;
    memcpy(pot, P.hout.ptr, sizeof(double) * ni);
    if (getenv("NB6_VERBOSE"))
        fprintf(stderr, "[R.%d GPU Pot.A] Ni %d  NTOT %d  pot(s) %f\n", irank ? *irank : 0, ni, n,
                nb6_wtime() - t0);
}

// Extension (no reference counterpart): potential on DEVICE arrays m[n],
// x[n][3]; the result stays on the device, its pointer is returned in *d_out.
// Enqueued on the library stream without a sync.
void nb6_pot_device_(int *istart, int *ni, int *n, const double *d_m, const double *d_x,
                     double **d_out) {
    nb6_devinit_once(0);
    cudaStream_t st = nb6_stream();
    if (!P.ev0) {
        NB6_CUDA_CHECK(cudaEventCreate(&P.ev0));
        NB6_CUDA_CHECK(cudaEventCreate(&P.ev1));
    }
    pot_upload(*n, d_m, d_x, st, false);
    NB6_CUDA_CHECK(cudaEventRecord(P.ev0, st));
    pot_prepare(*istart - 1, *ni, st);
    pot_device(*istart - 1, *ni, st);
    NB6_CUDA_CHECK(cudaEventRecord(P.ev1, st));
    *d_out = P.out.ptr;
}

// Device time (ms) of the last potential call after its upload: packing,
// spatial order, kernel and sums (after a sync).
float nb6_pot_last_kernel_ms_() {
    NB6_CUDA_CHECK(cudaEventSynchronize(P.ev1));
    NB6_CUDA_CHECK(cudaEventElapsedTime(&P.last_ms, P.ev0, P.ev1));
    return P.last_ms;
}

}  // extern "C"
