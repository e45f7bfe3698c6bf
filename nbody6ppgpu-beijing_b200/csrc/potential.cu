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

struct PotState {
    DevBuf<double> m, x, out;
    DevBuf<float4> posH, posL;
    DevBuf<float2> part;
    HostBuf<double> hout;
    int n = 0, ntile = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float last_ms = 0.f;
};
PotState P;

template <int NI> int pot_occ() {
    static int occ = -1;
    if (occ < 0) {
        NB6_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, pot_kernel<NI>, NT, 0));
        if (occ < 1) occ = 1;
    }
    return occ;
}

// Potential of i in [i0, i0+ni) against the packed j set; result in P.out.
void pot_device(int i0, int ni, cudaStream_t st) {
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

void pot_upload(int n, const double *m, const double *x, cudaStream_t st, bool from_host) {
    P.n = n;
    P.ntile = std::max(1, (n + JT - 1) / JT);
    const size_t npad = (size_t)P.ntile * JT;
    P.posH.reserve(npad);
    P.posL.reserve(npad);
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
    const int blocks = (int)std::min<size_t>((npad + 255) / 256, (size_t)nb6_num_sms() * 8);
    pot_pack<<<blocks, 256, 0, st>>>(n, (int)npad, dm, dx, P.posH.ptr, P.posL.ptr, nb6_dev_status());
    NB6_CUDA_CHECK(cudaGetLastError());
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
    pot_device(*istart - 1, *ni, st);
    NB6_CUDA_CHECK(cudaEventRecord(P.ev1, st));
    *d_out = P.out.ptr;
}

// Device time (ms) of the last potential kernel pair (after a sync).
float nb6_pot_last_kernel_ms_() {
    NB6_CUDA_CHECK(cudaEventSynchronize(P.ev1));
    NB6_CUDA_CHECK(cudaEventElapsedTime(&P.last_ms, P.ev0, P.ev1));
    return P.last_ms;
}

}  // extern "C"
