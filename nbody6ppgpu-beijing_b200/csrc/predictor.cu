// predictor.cu -- device-resident Hermite state and the j-particle predictor.
//
// The reference predicts every j on the host in FP64 before each regular
// block (xbpredall.F:48-62, jpred_int.f:16-25):
//     s = TIME - T0;  X = ((FDOT*s + F)*s + X0DOT)*s + X0
//     XDOT = (FDOT*1.5s + F)*2s + X0DOT            (F = a/2, FDOT = adot/6)
// and then copies all of them to the GPU (GPUNB_SEND, intgrt.F:882).  Here the
// state (T0, X0, X0DOT, F, FDOT, BODY) stays in HBM in FP64:
//
//   nb6_state_open_/set_/update_/close_   own and refresh the state (update_
//                                         scatters the particles a corrector
//                                         step changed);
//   nb6_predict_                          XBPREDALL on the GPU, results to the
//                                         caller's X/XDOT (drop-in for the
//                                         host loop);
//   nb6_predict_device_                   same, results left in HBM;
//   nb6_predict_send_                     predict + pack straight into the
//                                         regular-force j buffers: replaces
//                                         XBPREDALL + GPUNB_SEND with no host
//                                         traffic.
//
// The predictor is an HBM-streaming kernel: 104 bytes read (T0 + 4 x 3 FP64)
// and 48 written per body; the fused variant also writes the FP32 tiles.
// None of these entry points has a reference counterpart.
#include "nb6_common.cuh"

#include <algorithm>

bool regular_bind_j(int n, double **jm, double **jx, double **jv, JSetOut *out);

namespace {

struct State {
    bool open = false;
    int nmax = 0, n = 0;
    DevBuf<double> t0, x0, x0dot, f, fdot, body;
    DevBuf<double> xp, vp;            // predicted output (device)
    DevBuf<double> stage;             // update staging (device)
    DevBuf<int> sidx;
    HostBuf<double> hstage;
    HostBuf<int> hidx;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};
State S;

NB6_DEV void pred3(double s, const double *__restrict__ x0, const double *__restrict__ x0dot,
                   const double *__restrict__ f, const double *__restrict__ fdot, size_t j,
                   double *x, double *v) {
    const double s1 = 1.5 * s, s2 = 2.0 * s;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double fd = fdot[3 * j + k], ff = f[3 * j + k], vd = x0dot[3 * j + k];
        x[k] = ((fd * s + ff) * s + vd) * s + x0[3 * j + k];
        v[k] = (fd * s1 + ff) * s2 + vd;
    }
}

// Two bodies per thread: their six coordinates of each array are three
// 16-byte loads (the arrays are (n, 3) FP64 from cudaMalloc, so body 2p
// starts on a 16-byte boundary) and the results three 16-byte stores; the
// arithmetic is pred3's, operation for operation.
NB6_DEV void load6(const double *__restrict__ a, size_t p, double *o) {
    const double2 *q = reinterpret_cast<const double2 *>(a) + 3 * p;
    const double2 u = __ldg(q), v = __ldg(q + 1), w = __ldg(q + 2);
    o[0] = u.x; o[1] = u.y; o[2] = v.x; o[3] = v.y; o[4] = w.x; o[5] = w.y;
}

NB6_DEV void store6(double *__restrict__ a, size_t p, const double *o) {
    double2 *q = reinterpret_cast<double2 *>(a) + 3 * p;
    q[0] = make_double2(o[0], o[1]);
    q[1] = make_double2(o[2], o[3]);
    q[2] = make_double2(o[4], o[5]);
}

__global__ void predict_kernel(int n, double time, const double *__restrict__ t0,
                               const double *__restrict__ x0, const double *__restrict__ x0dot,
                               const double *__restrict__ f, const double *__restrict__ fdot,
                               double *__restrict__ xp, double *__restrict__ vp) {
    const size_t npair = (size_t)n / 2;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < npair;
         p += (size_t)gridDim.x * blockDim.x) {
        const double2 tt = __ldg(reinterpret_cast<const double2 *>(t0) + p);
        double X0[6], VD[6], FF[6], FD[6], x[6], v[6];
        load6(x0, p, X0);
        load6(x0dot, p, VD);
        load6(f, p, FF);
        load6(fdot, p, FD);
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const double s = time - (b ? tt.y : tt.x), s1 = 1.5 * s, s2 = 2.0 * s;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const int c = 3 * b + k;
                x[c] = ((FD[c] * s + FF[c]) * s + VD[c]) * s + X0[c];
                v[c] = (FD[c] * s1 + FF[c]) * s2 + VD[c];
            }
        }
        store6(xp, p, x);
        store6(vp, p, v);
    }
    if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {   // an odd last body
        const size_t j = (size_t)n - 1;
        double x[3], v[3];
        pred3(time - t0[j], x0, x0dot, f, fdot, j, x, v);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            xp[3 * j + k] = x[k];
            vp[3 * j + k] = v[k];
        }
    }
}

// Predict bodies [j0, j0+n) and write the regular-force j set (FP64 copy and
// the float layouts, padded with far massless bodies).
__global__ void predict_pack_kernel(int j0, int n, double time, const double *__restrict__ t0,
                                    const double *__restrict__ x0, const double *__restrict__ x0dot,
                                    const double *__restrict__ f, const double *__restrict__ fdot,
                                    const double *__restrict__ body, double *__restrict__ jm,
                                    double *__restrict__ jx, double *__restrict__ jv, JSetOut o) {
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < o.npad;
         q += (size_t)gridDim.x * blockDim.x) {
        if (q < (size_t)n) {
            const size_t j = (size_t)j0 + q;
            double x[3], v[3];
            pred3(time - t0[j], x0, x0dot, f, fdot, j, x, v);
            const double m = body[j];
            jm[q] = m;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                jx[3 * q + k] = x[k];
                jv[3 * q + k] = v[k];
            }
            write_j(o, q, true, x[0], x[1], x[2], m, v[0], v[1], v[2]);
        } else {
            write_j(o, q, false, 0, 0, 0, 0, 0, 0, 0);
        }
    }
}

// stage layout per updated body: t0, x0[3], x0dot[3], f[3], fdot[3], body
__global__ void state_scatter(int nu, const int *__restrict__ idx, const double *__restrict__ st,
                              double *t0, double *x0, double *x0dot, double *f, double *fdot,
                              double *body) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= nu) return;
    const size_t j = (size_t)idx[u];
    const double *s = st + (size_t)u * 14;
    t0[j] = s[0];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        x0[3 * j + k] = s[1 + k];
        x0dot[3 * j + k] = s[4 + k];
        f[3 * j + k] = s[7 + k];
        fdot[3 * j + k] = s[10 + k];
    }
    body[j] = s[13];
}

int grid_for(size_t n) {
    return (int)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, (size_t)nb6_num_sms() * 16));
}

bool check_open(int n) {
    if (!S.open) {
        nb6_fatal(NB6_ERR_NOT_OPEN);
        return false;
    }
    if (n < 0 || n > S.nmax) {
        fprintf(stderr, "nb6 state: n=%d outside [0, %d]\n", n, S.nmax);
        nb6_fatal(NB6_ERR_TOO_LARGE);
        return false;
    }
    return true;
}

}  // namespace

extern "C" {

void nb6_state_open_(int *nmax) {
    nb6_devinit_once(0);
    if (S.open) return;
    S.open = true;
    S.nmax = *nmax;
    const size_t n = (size_t)std::max(*nmax, 1);
    S.t0.reserve(n);
    S.x0.reserve(3 * n);
    S.x0dot.reserve(3 * n);
    S.f.reserve(3 * n);
    S.fdot.reserve(3 * n);
    S.body.reserve(n);
    if (!S.ev0) {
        NB6_CUDA_CHECK(cudaEventCreate(&S.ev0));
        NB6_CUDA_CHECK(cudaEventCreate(&S.ev1));
    }
}

void nb6_state_close_() {
    if (!S.open) return;
    S.open = false;
    S.t0.release();
    S.x0.release();
    S.x0dot.release();
    S.f.release();
    S.fdot.release();
    S.body.release();
    S.xp.release();
    S.vp.release();
    S.stage.release();
    S.sidx.release();
    S.hstage.release();
    S.hidx.release();
    S.n = 0;
}

// Upload the whole state of n bodies (Fortran X0(3,N) etc. = C double[n][3]).
void nb6_state_set_(int *n, double *body, double *t0, double (*x0)[3], double (*x0dot)[3],
                    double (*f)[3], double (*fdot)[3]) {
    if (!check_open(*n)) return;
    S.n = *n;
    const size_t k = (size_t)*n;
    cudaStream_t st = nb6_stream();
    if (k == 0) return;
    NB6_CUDA_CHECK(cudaMemcpyAsync(S.t0.ptr, t0, 8 * k, cudaMemcpyHostToDevice, st));
    NB6_CUDA_CHECK(cudaMemcpyAsync(S.x0.ptr, x0, 24 * k, cudaMemcpyHostToDevice, st));
    NB6_CUDA_CHECK(cudaMemcpyAsync(S.x0dot.ptr, x0dot, 24 * k, cudaMemcpyHostToDevice, st));
    NB6_CUDA_CHECK(cudaMemcpyAsync(S.f.ptr, f, 24 * k, cudaMemcpyHostToDevice, st));
    NB6_CUDA_CHECK(cudaMemcpyAsync(S.fdot.ptr, fdot, 24 * k, cudaMemcpyHostToDevice, st));
    NB6_CUDA_CHECK(cudaMemcpyAsync(S.body.ptr, body, 8 * k, cudaMemcpyHostToDevice, st));
    NB6_CUDA_CHECK(cudaStreamSynchronize(st));
}

// Refresh nu bodies with 1-based indices idx[]; the arrays are compact [nu].
void nb6_state_update_(int *nu_, int *idx, double *body, double *t0, double (*x0)[3],
                       double (*x0dot)[3], double (*f)[3], double (*fdot)[3]) {
    const int nu = *nu_;
    if (!check_open(S.n)) return;
    if (nu <= 0) return;
    S.hstage.reserve((size_t)nu * 14);
    S.hidx.reserve(nu);
    for (int u = 0; u < nu; ++u) {
        if (idx[u] < 1 || idx[u] > S.n) {
            fprintf(stderr, "nb6_state_update: index %d outside [1, %d]\n", idx[u], S.n);
            nb6_fatal(NB6_ERR_BAD_ARG);
            return;
        }
        double *s = S.hstage.ptr + (size_t)u * 14;
        s[0] = t0[u];
        for (int k = 0; k < 3; ++k) {
            s[1 + k] = x0[u][k];
            s[4 + k] = x0dot[u][k];
            s[7 + k] = f[u][k];
            s[10 + k] = fdot[u][k];
        }
        s[13] = body[u];
        S.hidx.ptr[u] = idx[u] - 1;
    }
    cudaStream_t st = nb6_stream();
    S.stage.reserve((size_t)nu * 14);
    S.sidx.reserve(nu);
    NB6_CUDA_CHECK(cudaMemcpyAsync(S.stage.ptr, S.hstage.ptr, sizeof(double) * 14 * nu,
                                   cudaMemcpyHostToDevice, st));
    NB6_CUDA_CHECK(cudaMemcpyAsync(S.sidx.ptr, S.hidx.ptr, sizeof(int) * nu, cudaMemcpyHostToDevice, st));
    state_scatter<<<(nu + 255) / 256, 256, 0, st>>>(nu, S.sidx.ptr, S.stage.ptr, S.t0.ptr, S.x0.ptr,
                                                   S.x0dot.ptr, S.f.ptr, S.fdot.ptr, S.body.ptr);
    NB6_CUDA_CHECK(cudaGetLastError());
    NB6_CUDA_CHECK(cudaStreamSynchronize(st));
}

// XBPREDALL on the device; predicted X, XDOT of all n bodies left in HBM.
void nb6_predict_device_(double *time, double **d_x, double **d_xdot) {
    if (!check_open(S.n)) return;
    const size_t n = (size_t)S.n;
    S.xp.reserve(3 * std::max<size_t>(n, 1));
    S.vp.reserve(3 * std::max<size_t>(n, 1));
    cudaStream_t st = nb6_stream();
    NB6_CUDA_CHECK(cudaEventRecord(S.ev0, st));
    if (n > 0)
        predict_kernel<<<grid_for((n + 1) / 2), 256, 0, st>>>((int)n, *time, S.t0.ptr, S.x0.ptr, S.x0dot.ptr,
                                                    S.f.ptr, S.fdot.ptr, S.xp.ptr, S.vp.ptr);
    NB6_CUDA_CHECK(cudaGetLastError());
    NB6_CUDA_CHECK(cudaEventRecord(S.ev1, st));
    *d_x = S.xp.ptr;
    *d_xdot = S.vp.ptr;
}

// XBPREDALL drop-in: predicted X, XDOT of all n bodies into host arrays.
void nb6_predict_(double *time, double (*x)[3], double (*xdot)[3]) {
    double *dx, *dv;
    nb6_predict_device_(time, &dx, &dv);
    if (S.n <= 0) return;
    cudaStream_t st = nb6_stream();
    NB6_CUDA_CHECK(cudaMemcpyAsync(x, dx, 24 * (size_t)S.n, cudaMemcpyDeviceToHost, st));
    NB6_CUDA_CHECK(cudaMemcpyAsync(xdot, dv, 24 * (size_t)S.n, cudaMemcpyDeviceToHost, st));
    NB6_CUDA_CHECK(cudaStreamSynchronize(st));
}

// XBPREDALL + GPUNB_SEND(NN, BODY(IFIRST), X(1,IFIRST), XDOT(1,IFIRST)) with
// no host traffic: bodies [ifirst, ifirst+nn) (1-based) are predicted and
// packed as the regular-force j set.  gpunb_open_ must have been called.
void nb6_predict_send_(double *time, int *ifirst, int *nn) {
    if (!check_open(S.n)) return;
    const int j0 = *ifirst - 1, n = *nn;
    if (j0 < 0 || n < 0 || j0 + n > S.n) {
        fprintf(stderr, "nb6_predict_send: range [%d, %d) outside the state\n", j0 + 1, j0 + n + 1);
        nb6_fatal(NB6_ERR_BAD_ARG);
        return;
    }
    double *jm, *jx, *jv;
    JSetOut o;
    if (!regular_bind_j(n, &jm, &jx, &jv, &o)) return;
    cudaStream_t st = nb6_stream();
    NB6_CUDA_CHECK(cudaEventRecord(S.ev0, st));
    predict_pack_kernel<<<grid_for(o.npad), 256, 0, st>>>(j0, n, *time, S.t0.ptr, S.x0.ptr,
                                                          S.x0dot.ptr, S.f.ptr, S.fdot.ptr,
                                                          S.body.ptr, jm, jx, jv, o);
    NB6_CUDA_CHECK(cudaGetLastError());
    NB6_CUDA_CHECK(cudaEventRecord(S.ev1, st));
}

float nb6_predict_last_kernel_ms_() {
    float ms = 0.f;
    NB6_CUDA_CHECK(cudaEventSynchronize(S.ev1));
    NB6_CUDA_CHECK(cudaEventElapsedTime(&ms, S.ev0, S.ev1));
    return ms;
}

}  // extern "C"
