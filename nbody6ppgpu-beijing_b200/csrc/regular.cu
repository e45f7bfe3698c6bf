// regular.cu -- regular force + jerk + potential + neighbour list on sm_100a,
// behind the reference's gpunb_* C ABI (gpunb.velocity.cu:905-940).
//
// Per call of gpunb_regf_ (ni active particles against the nj particles of the
// last gpunb_send_):
//
//   regf_kernel     grid (i-tiles x j-slices).  Each thread holds NI
//                   i-particles in registers (FP64 position split hi/lo);
//                   the CTA streams its j-slice through a 4-stage shared
//                   memory ring filled by 1-D bulk copies (cp.async.bulk,
//                   mbarrier completion, bounded waits).  Pair math is FP32
//                   with hi/lo coordinate differences and rsqrt + one Newton
//                   step; per-i sums fold into double-single accumulators once
//                   per 128-j tile.  The neighbour test runs with a 1% slack;
//                   every candidate is re-decided exactly in FP64 (the rule of
//                   gpunb.velocity.cu:176-188 / regint.f:49-65) off the hot
//                   loop, so the list equals the FP64 rule's list.
//   regf_finalize   one warp per i: deterministic FP64 sum of the slice
//                   partials, and the neighbour ids sorted ascending (warp
//                   bitonic sort in shared memory), overflow -> -nnb.
//
// Semantics kept from the reference: acc/jrk/pot exclude neighbours, pot is
// positive, jrk is adot, list ids are 0-based j relative to the first particle
// sent, ascending, self included; nnb > nnbmax -> list[0] = -nnb and no ids
// (reg.avx.cpp:320-327).
#include "nb6_common.cuh"

#include <algorithm>
#include <climits>
#include <math.h>
#include <string.h>

namespace {

constexpr int JT = 128;      // j per pipeline stage
constexpr int NSTAGE = 4;    // ring depth
constexpr int NT = 128;      // threads per CTA
constexpr float CAND_SLACK = 1.01f;
constexpr unsigned long long WAIT_NS = 2000000000ull;  // 2 s per wait
constexpr int FIN_WARPS = 4;

// j unroll of the hot loop: large enough for ILP, small enough that the
// loop body stays resident in the instruction cache.
#ifndef UNROLL_J
#define UNROLL_J 8
#endif
constexpr int kUnrollJ = UNROLL_J;
// The rare candidate path is kept out of line by default so that it does not
// inflate the register allocation of the hot loop.
#ifndef FLUSH_INLINE
#define FLUSH_INLINE __noinline__
#endif

struct RegArgs {
    const float4 *__restrict__ posH;  // (xH, yH, zH, m)
    const float4 *__restrict__ posL;  // (xL, yL, zL, 0)
    const float4 *__restrict__ vel;   // (vx, vy, vz, 0)
    const double *__restrict__ jm;    // FP64 copies for the exact recheck
    const double *__restrict__ jx;
    const double *__restrict__ jv;
    int nj, ntile, nslices;
    const double *__restrict__ ih2;
    const double *__restrict__ idtr;
    const double *__restrict__ ix;
    const double *__restrict__ iv;
    int ni, ni_pad;
    float4 *__restrict__ part;   // [nslices][ni_pad][4]
    int *__restrict__ nbcnt;     // [ni]
    int *__restrict__ nbbuf;     // [ni][lcap]
    int lcap;
    int *status;
};

struct IPart {
    float xh, yh, zh, xl, yl, zl, vx, vy, vz, h2c, dt;
};

struct Sums {
    float ax, ay, az, jx, jy, jz, po;
};

NB6_DEV void zero(Sums &s) { s.ax = s.ay = s.az = s.jx = s.jy = s.jz = s.po = 0.f; }

// The FP32 candidate test, shared verbatim by the hot loop and the rare path
// so both always classify a pair the same way (explicit fmaf/__fmul_rn: no
// contraction freedom).  Candidate: min(r2, |dx + dt dv|^2) < 1.01 crit.
struct PairGeom {
    float dx, dy, dz, dvx, dvy, dvz, r2;
    bool cand;
};

template <bool MFLAG>
NB6_DEV PairGeom reg_geom(const IPart &ip, const float4 &a, const float4 &b, const float4 &c) {
    PairGeom g;
    g.dx = (a.x - ip.xh) + (b.x - ip.xl);
    g.dy = (a.y - ip.yh) + (b.y - ip.yl);
    g.dz = (a.z - ip.zh) + (b.z - ip.zl);
    g.dvx = c.x - ip.vx;
    g.dvy = c.y - ip.vy;
    g.dvz = c.z - ip.vz;
    g.r2 = fmaf(g.dz, g.dz, fmaf(g.dy, g.dy, __fmul_rn(g.dx, g.dx)));
    const float px = fmaf(ip.dt, g.dvx, g.dx);
    const float py = fmaf(ip.dt, g.dvy, g.dy);
    const float pz = fmaf(ip.dt, g.dvz, g.dz);
    const float rp2 = fmaf(pz, pz, fmaf(py, py, __fmul_rn(px, px)));
    const float crit = MFLAG ? __fmul_rn(a.w, ip.h2c) : ip.h2c;
    g.cand = fminf(g.r2, rp2) < crit;
    return g;
}

// Pair interaction in FP32; returns whether j is a neighbour candidate.
// Sums are kept scaled: pot x2, acc and jerk x8 (see rsqrt2_nr).
template <bool MFLAG>
NB6_DEV bool reg_pair(const IPart &ip, const float4 &a, const float4 &b, const float4 &c,
                      Sums &s) {
    const PairGeom g = reg_geom<MFLAG>(ip, a, b, c);
    const float dx = g.dx, dy = g.dy, dz = g.dz, dvx = g.dvx, dvy = g.dvy, dvz = g.dvz;
    const float r2 = g.r2;
    const bool cand = g.cand;
    const float rv = fmaf(dz, dvz, fmaf(dy, dvy, dx * dvx));
    float y = rsqrt2_nr(r2);
    y = cand ? 0.0f : y;
    const float y2 = y * y;
    const float my = a.w * y;
    const float my3 = my * y2;
    const float al = (y2 * -0.75f) * rv;
    s.po += my;
    s.ax = fmaf(my3, dx, s.ax);
    s.ay = fmaf(my3, dy, s.ay);
    s.az = fmaf(my3, dz, s.az);
    s.jx = fmaf(my3, fmaf(al, dx, dvx), s.jx);
    s.jy = fmaf(my3, fmaf(al, dy, dvy), s.jy);
    s.jz = fmaf(my3, fmaf(al, dz, dvz), s.jz);
    return cand;
}

// Rare path for one i and one 32-j group that held at least one candidate:
// re-derive the candidates with the same FP32 test, then decide each exactly
// in FP64.  Operation order matches the FP64 rule of regint.f:41-65 with the
// strict "<" of gpunb.velocity.cu:188,236; no FMA contraction.
template <bool MFLAG>
__device__ FLUSH_INLINE Sums reg_flush(const RegArgs &a, const IPart ip, int i, const float4 *A,
                                       const float4 *B, const float4 *Cv, int jbase, Sums s) {
    const double xi0 = a.ix[3 * i], xi1 = a.ix[3 * i + 1], xi2 = a.ix[3 * i + 2];
    const double vi0 = a.iv[3 * i], vi1 = a.iv[3 * i + 1], vi2 = a.iv[3 * i + 2];
    const double h2 = a.ih2[i], dt = a.idtr[i];
    for (int b = 0; b < 32; ++b) {
        if (!reg_geom<MFLAG>(ip, A[b], B[b], Cv[b]).cand) continue;
        const int j = jbase + b;
        if (j >= a.nj) continue;  // padding slots are never neighbours
        const double dx = __dsub_rn(a.jx[3 * j], xi0);
        const double dy = __dsub_rn(a.jx[3 * j + 1], xi1);
        const double dz = __dsub_rn(a.jx[3 * j + 2], xi2);
        const double dvx = __dsub_rn(a.jv[3 * j], vi0);
        const double dvy = __dsub_rn(a.jv[3 * j + 1], vi1);
        const double dvz = __dsub_rn(a.jv[3 * j + 2], vi2);
        const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)),
                                    __dmul_rn(dz, dz));
        const double px = __dadd_rn(dx, __dmul_rn(dt, dvx));
        const double py = __dadd_rn(dy, __dmul_rn(dt, dvy));
        const double pz = __dadd_rn(dz, __dmul_rn(dt, dvz));
        const double r2p = __dadd_rn(__dadd_rn(__dmul_rn(px, px), __dmul_rn(py, py)),
                                     __dmul_rn(pz, pz));
        const double rmin = (r2 < r2p) ? r2 : r2p;
        const double crit = MFLAG ? __dmul_rn(a.jm[j], h2) : h2;
        if (rmin < crit) {
            const int pos = atomicAdd(&a.nbcnt[i], 1);
            if (pos < a.lcap) a.nbbuf[(size_t)i * a.lcap + pos] = j;
        } else {
            // inside the slack band but not a neighbour: add it here
            const double rinv2 = 1.0 / r2;
            const double rinv = sqrt(rinv2);
            const double mr = a.jm[j] * rinv;
            const double mr3 = mr * rinv2;
            const double rv = dx * dvx + dy * dvy + dz * dvz;
            const double al = -3.0 * rv * rinv2;
            s.po += (float)(2.0 * mr);
            s.ax += (float)(8.0 * mr3 * dx);
            s.ay += (float)(8.0 * mr3 * dy);
            s.az += (float)(8.0 * mr3 * dz);
            s.jx += (float)(8.0 * mr3 * (dvx + al * dx));
            s.jy += (float)(8.0 * mr3 * (dvy + al * dy));
            s.jz += (float)(8.0 * mr3 * (dvz + al * dz));
        }
    }
    return s;
}

NB6_DEV void issue_tile(const RegArgs &a, float4 (*stage)[JT], uint64_t *bar, int tile) {
    const size_t off = (size_t)tile * JT;
    mbar_arrive_expect_tx(bar, 3u * JT * sizeof(float4));
    bulk_g2s(stage[0], a.posH + off, JT * sizeof(float4), bar);
    bulk_g2s(stage[1], a.posL + off, JT * sizeof(float4), bar);
    bulk_g2s(stage[2], a.vel + off, JT * sizeof(float4), bar);
}

template <int NI, bool MFLAG>
__global__ void __launch_bounds__(NT) regf_kernel(const RegArgs a) {
    __shared__ __align__(128) float4 sj[NSTAGE][3][JT];
    __shared__ __align__(8) uint64_t bar[NSTAGE];

    const int tid = threadIdx.x;
    const int slice = blockIdx.y;
    const int t_begin = (int)(((long long)slice * a.ntile) / a.nslices);
    const int t_end = (int)(((long long)(slice + 1) * a.ntile) / a.nslices);
    const int nt = t_end - t_begin;

    IPart ip[NI];
    Sums s[NI], H[NI], L[NI];
    int ii[NI];
#pragma unroll
    for (int k = 0; k < NI; ++k) {
        const int i = blockIdx.x * (NT * NI) + k * NT + tid;
        ii[k] = i;
        zero(s[k]);
        zero(H[k]);
        zero(L[k]);
        if (i < a.ni) {
            split_hl(a.ix[3 * i], ip[k].xh, ip[k].xl);
            split_hl(a.ix[3 * i + 1], ip[k].yh, ip[k].yl);
            split_hl(a.ix[3 * i + 2], ip[k].zh, ip[k].zl);
            ip[k].vx = (float)a.iv[3 * i];
            ip[k].vy = (float)a.iv[3 * i + 1];
            ip[k].vz = (float)a.iv[3 * i + 2];
            ip[k].h2c = (float)a.ih2[i] * CAND_SLACK;
            ip[k].dt = (float)a.idtr[i];
        } else {
            ip[k].xh = ip[k].yh = ip[k].zh = ip[k].xl = ip[k].yl = ip[k].zl = 0.f;
            ip[k].vx = ip[k].vy = ip[k].vz = 0.f;
            ip[k].h2c = 0.f;  // padding lanes: never a candidate
            ip[k].dt = 0.f;
        }
    }

    if (tid == 0) {
#pragma unroll
        for (int st = 0; st < NSTAGE; ++st) mbar_init(&bar[st], 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0) {
        for (int st = 0; st < NSTAGE && st < nt; ++st) issue_tile(a, sj[st], &bar[st], t_begin + st);
    }

    for (int t = 0; t < nt; ++t) {
        const int st = t % NSTAGE;
        const bool ok = mbar_wait_timed(&bar[st], (uint32_t)((t / NSTAGE) & 1), WAIT_NS);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                set_status(a.status, NB6_ERR_WAIT_TIMEOUT);
                // drain copies still in flight before the CTA's smem goes away
                const int issued = min(nt, NSTAGE + max(t - 1, 0));
                for (int u = t; u < issued; ++u)
                    mbar_wait_timed(&bar[u % NSTAGE], (uint32_t)((u / NSTAGE) & 1), WAIT_NS / 8);
            }
            return;
        }
        // every thread finished tile t-1: its stage can be refilled
        if (tid == 0 && t >= 1 && t - 1 + NSTAGE < nt)
            issue_tile(a, sj[(t - 1) % NSTAGE], &bar[(t - 1) % NSTAGE], t_begin + t - 1 + NSTAGE);

        const float4 *A = sj[st][0];
        const float4 *B = sj[st][1];
        const float4 *C = sj[st][2];
        const int jt0 = (t_begin + t) * JT;
#pragma unroll 1
        for (int g = 0; g < JT / 32; ++g) {
            bool anyc[NI];
#pragma unroll
            for (int k = 0; k < NI; ++k) anyc[k] = false;
            const float4 *Ag = A + g * 32, *Bg = B + g * 32, *Cg = C + g * 32;
#pragma unroll kUnrollJ
            for (int q = 0; q < 32; ++q) {
                const float4 pa = Ag[q];
                const float4 pb = Bg[q];
                const float4 pc = Cg[q];
#pragma unroll
                for (int k = 0; k < NI; ++k) anyc[k] |= reg_pair<MFLAG>(ip[k], pa, pb, pc, s[k]);
            }
#pragma unroll
            for (int k = 0; k < NI; ++k)
                if (anyc[k]) s[k] = reg_flush<MFLAG>(a, ip[k], ii[k], Ag, Bg, Cg, jt0 + g * 32, s[k]);
        }
#pragma unroll
        for (int k = 0; k < NI; ++k) {
            ds_fold(H[k].ax, L[k].ax, s[k].ax);
            ds_fold(H[k].ay, L[k].ay, s[k].ay);
            ds_fold(H[k].az, L[k].az, s[k].az);
            ds_fold(H[k].jx, L[k].jx, s[k].jx);
            ds_fold(H[k].jy, L[k].jy, s[k].jy);
            ds_fold(H[k].jz, L[k].jz, s[k].jz);
            ds_fold(H[k].po, L[k].po, s[k].po);
            zero(s[k]);
        }
    }

#pragma unroll
    for (int k = 0; k < NI; ++k) {
        const int i = ii[k];
        if (i < a.ni) {
            float4 *p = a.part + ((size_t)slice * a.ni_pad + i) * 4;
            p[0] = make_float4(H[k].ax, L[k].ax, H[k].ay, L[k].ay);
            p[1] = make_float4(H[k].az, L[k].az, H[k].jx, L[k].jx);
            p[2] = make_float4(H[k].jy, L[k].jy, H[k].jz, L[k].jz);
            p[3] = make_float4(H[k].po, L[k].po, 0.f, 0.f);
        }
    }
}

// One warp per i: FP64 sum over slices in a fixed order, then the neighbour
// ids sorted ascending.  outf row = (ax, ay, az, jx, jy, jz, pot, 0).
__global__ void __launch_bounds__(FIN_WARPS * 32)
    regf_finalize(const float4 *__restrict__ part, int nslices, int ni, int ni_pad,
                  const int *__restrict__ nbcnt, const int *__restrict__ nbbuf, int lcap,
                  int cap, int W, int pmax, double *__restrict__ outf,
                  int *__restrict__ outl) {
    extern __shared__ int sbuf[];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * FIN_WARPS + warp;
    if (i >= ni) return;

    double v[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int sl = lane; sl < nslices; sl += 32) {
        const float4 *p = part + ((size_t)sl * ni_pad + i) * 4;
        const float4 q0 = p[0], q1 = p[1], q2 = p[2], q3 = p[3];
        v[0] += (double)q0.x + (double)q0.y;
        v[1] += (double)q0.z + (double)q0.w;
        v[2] += (double)q1.x + (double)q1.y;
        v[3] += (double)q1.z + (double)q1.w;
        v[4] += (double)q2.x + (double)q2.y;
        v[5] += (double)q2.z + (double)q2.w;
        v[6] += (double)q3.x + (double)q3.y;
    }
#pragma unroll
    for (int c = 0; c < 7; ++c) v[c] = warp_sum_d(v[c]);
    if (lane == 0) {
        double *o = outf + (size_t)i * 8;
        o[0] = v[0] * 0.125;
        o[1] = v[1] * 0.125;
        o[2] = v[2] * 0.125;
        o[3] = v[3] * 0.125;
        o[4] = v[4] * 0.125;
        o[5] = v[5] * 0.125;
        o[6] = v[6] * 0.5;
        o[7] = 0.0;
    }

    const int n = nbcnt[i];
    int *row = outl + (size_t)i * W;
    if (n > cap) {
        if (lane == 0) row[0] = -n;
        return;
    }
    int *sb = sbuf + warp * pmax;
    int P = 32;
    while (P < n) P <<= 1;
    const int *src = nbbuf + (size_t)i * lcap;
    for (int k = lane; k < P; k += 32) sb[k] = (k < n) ? src[k] : INT_MAX;
    __syncwarp();
    for (int kk = 2; kk <= P; kk <<= 1) {
        for (int jj = kk >> 1; jj > 0; jj >>= 1) {
            for (int x = lane; x < P; x += 32) {
                const int y = x ^ jj;
                if (y > x) {
                    const int p0 = sb[x], p1 = sb[y];
                    const bool up = (x & kk) == 0;
                    if ((p0 > p1) == up) {
                        sb[x] = p1;
                        sb[y] = p0;
                    }
                }
            }
            __syncwarp();
        }
    }
    if (lane == 0) row[0] = n;
    for (int k = lane; k < n; k += 32) row[1 + k] = sb[k];
}

// FP64 (m, x, v) -> SoA float4 tiles; padding slots are massless and far.
__global__ void regf_pack_j(int nj, int npad, const double *__restrict__ m,
                            const double *__restrict__ x, const double *__restrict__ v,
                            float4 *__restrict__ posH, float4 *__restrict__ posL,
                            float4 *__restrict__ vel, int *status) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < npad; j += gridDim.x * blockDim.x) {
        if (j < nj) {
            const double x0 = x[3 * j], x1 = x[3 * j + 1], x2 = x[3 * j + 2];
            const double v0 = v[3 * j], v1 = v[3 * j + 1], v2 = v[3 * j + 2];
            const double mj = m[j];
            if (x0 != x0 || x1 != x1 || x2 != x2 || v0 != v0 || v1 != v1 || v2 != v2 ||
                mj != mj)
                set_status(status, NB6_ERR_NAN_INPUT);
            float4 h, l;
            split_hl(x0, h.x, l.x);
            split_hl(x1, h.y, l.y);
            split_hl(x2, h.z, l.z);
            h.w = (float)mj;
            l.w = 0.f;
            posH[j] = h;
            posL[j] = l;
            vel[j] = make_float4((float)v0, (float)v1, (float)v2, 0.f);
        } else {
            posH[j] = make_float4(1.0e15f, 1.0e15f, 1.0e15f, 0.f);
            posL[j] = make_float4(0.f, 0.f, 0.f, 0.f);
            vel[j] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
    }
}

// ----------------------------------------------------------------------------
// host state
// ----------------------------------------------------------------------------
struct RegState {
    bool open = false;
    int nbodymax = 0;
    int nj = 0;
    int ntile = 0;
    DevBuf<float4> posH, posL, vel;
    DevBuf<double> jm, jx, jv;
    DevBuf<double> iin;
    DevBuf<float4> part;
    DevBuf<int> nbcnt, nbbuf;
    DevBuf<double> outf;
    DevBuf<int> outl;
    HostBuf<double> hin, houtf;
    HostBuf<int> houtl;
    // reference-style profile counters (gpunb.velocity.cu:558,883-903)
    double time_send = 0, time_grav = 0, time_reduce = 0, time_out = 0;
    long long numInter = 0;
    int icall = 0, ini = 0, isend = 0;
    // kernel-only device time of the last regf launch pair (ms)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float last_kernel_ms = 0.f;
    int forced_ni_per_thread = 0;   // 0 = autotune
    int forced_slices = 0;
    int last_geometry[3] = {0, 0, 0};  // NI, i-tiles, j-slices of the last launch
};
RegState R;

template <int NI, bool MF> int occupancy() {
    static int occ = -1;
    if (occ < 0) {
        NB6_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, regf_kernel<NI, MF>, NT, 0));
        if (occ < 1) occ = 1;
    }
    return occ;
}

template <int NI, bool MF>
void launch_regf(RegArgs a, int nitile, cudaStream_t st) {
    dim3 grid(nitile, a.nslices);
    regf_kernel<NI, MF><<<grid, NT, 0, st>>>(a);
}

int occ_for(int NI, bool mf) {
    if (mf) {
        if (NI == 1) return occupancy<1, true>();
        if (NI == 2) return occupancy<2, true>();
        return occupancy<4, true>();
    }
    if (NI == 1) return occupancy<1, false>();
    if (NI == 2) return occupancy<2, false>();
    return occupancy<4, false>();
}

// Launch geometry: i-per-thread and j-slice count.  Picks the largest NI whose
// i-tiles stay >= 90% full, then enough slices to fill every SM once.
void pick_geometry(int ni, int ntile, bool mf, int &NI, int &nitile, int &nslices) {
    NI = 1;
    if (R.forced_ni_per_thread == 1 || R.forced_ni_per_thread == 2 || R.forced_ni_per_thread == 4) {
        NI = R.forced_ni_per_thread;
    } else {
        const int cands[3] = {4, 2, 1};
        for (int c : cands) {
            const int tile = NT * c;
            const int nit = (ni + tile - 1) / tile;
            if ((double)ni / ((double)nit * tile) >= 0.9 || c == 1) {
                NI = c;
                break;
            }
        }
    }
    const int tile = NT * NI;
    nitile = (ni + tile - 1) / tile;
    const int target = nb6_num_sms() * occ_for(NI, mf);
    nslices = std::max(1, target / nitile);
    if (R.forced_slices > 0) nslices = R.forced_slices;
    nslices = std::min(nslices, ntile);
    nslices = std::max(nslices, 1);
}

bool any_nan(const double *p, size_t n) {
    for (size_t k = 0; k < n; ++k)
        if (p[k] != p[k]) return true;
    return false;
}

}  // namespace

// ----------------------------------------------------------------------------
// device-side regular force on resident i data (used by the ABI and by the
// benchmark's kernel-only timing)
// ----------------------------------------------------------------------------
static void regf_device(int ni, const double *d_h2, const double *d_dtr, const double *d_x,
                        const double *d_v, int lmax, int nnbmax, int mflag, cudaStream_t st,
                        int &W) {
    const int cap = std::max(0, std::min(nnbmax, lmax - 1));
    W = cap + 1;
    const int ni_pad = ni;
    int NI, nitile, nslices;
    pick_geometry(ni, R.ntile, mflag != 0, NI, nitile, nslices);
    R.part.reserve((size_t)nslices * ni_pad * 4);
    R.nbcnt.reserve(ni);
    R.nbbuf.reserve((size_t)ni * std::max(cap, 1));
    R.outf.reserve((size_t)ni * 8);
    R.outl.reserve((size_t)ni * W);
    NB6_CUDA_CHECK(cudaMemsetAsync(R.nbcnt.ptr, 0, sizeof(int) * ni, st));

    RegArgs a;
    a.posH = R.posH.ptr;
    a.posL = R.posL.ptr;
    a.vel = R.vel.ptr;
    a.jm = R.jm.ptr;
    a.jx = R.jx.ptr;
    a.jv = R.jv.ptr;
    a.nj = R.nj;
    a.ntile = R.ntile;
    a.nslices = nslices;
    a.ih2 = d_h2;
    a.idtr = d_dtr;
    a.ix = d_x;
    a.iv = d_v;
    a.ni = ni;
    a.ni_pad = ni_pad;
    a.part = R.part.ptr;
    a.nbcnt = R.nbcnt.ptr;
    a.nbbuf = R.nbbuf.ptr;
    a.lcap = std::max(cap, 1);
    a.status = nb6_dev_status();

    if (!R.ev0) {
        NB6_CUDA_CHECK(cudaEventCreate(&R.ev0));
        NB6_CUDA_CHECK(cudaEventCreate(&R.ev1));
    }
    // kernel-only timing of the main force kernel (read by
    // nb6_regf_last_kernel_ms_ after the stream has drained)
    NB6_CUDA_CHECK(cudaEventRecord(R.ev0, st));
    if (mflag) {
        if (NI == 1) launch_regf<1, true>(a, nitile, st);
        else if (NI == 2) launch_regf<2, true>(a, nitile, st);
        else launch_regf<4, true>(a, nitile, st);
    } else {
        if (NI == 1) launch_regf<1, false>(a, nitile, st);
        else if (NI == 2) launch_regf<2, false>(a, nitile, st);
        else launch_regf<4, false>(a, nitile, st);
    }
    NB6_CUDA_CHECK(cudaGetLastError());
    NB6_CUDA_CHECK(cudaEventRecord(R.ev1, st));
    R.last_geometry[0] = NI;
    R.last_geometry[1] = nitile;
    R.last_geometry[2] = nslices;

    int pmax = 32;
    while (pmax < cap) pmax <<= 1;
    const int fblocks = (ni + FIN_WARPS - 1) / FIN_WARPS;
    const size_t smem = (size_t)FIN_WARPS * pmax * sizeof(int);
    if (smem > 48 * 1024)
        NB6_CUDA_CHECK(cudaFuncSetAttribute(regf_finalize, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)smem));
    regf_finalize<<<fblocks, FIN_WARPS * 32, smem, st>>>(R.part.ptr, nslices, ni, ni_pad,
                                                        R.nbcnt.ptr, R.nbbuf.ptr, a.lcap, cap, W,
                                                        pmax, R.outf.ptr, R.outl.ptr);
    NB6_CUDA_CHECK(cudaGetLastError());
}

// ----------------------------------------------------------------------------
// reference ABI
// ----------------------------------------------------------------------------
extern "C" {

void gpunb_devinit_(int *irank) { nb6_devinit_once(irank ? *irank : 0); }

void gpunb_open_(int *nbmax, int *irank) {
    R.time_send = R.time_grav = R.time_reduce = R.time_out = 0.0;
    R.numInter = 0;
    R.icall = R.ini = R.isend = 0;
    nb6_devinit_once(*irank);
    if (R.open) {
        fprintf(stderr, "gpunb: it is already open\n");
        return;
    }
    if (*nbmax < 0) {
        nb6_fatal(NB6_ERR_BAD_ARG);
        return;
    }
    R.open = true;
    R.nbodymax = *nbmax;
    const size_t npad = ((size_t)std::max(*nbmax, 1) + JT - 1) / JT * JT;
    R.posH.reserve(npad);
    R.posL.reserve(npad);
    R.vel.reserve(npad);
    R.jm.reserve(npad);
    R.jx.reserve(3 * npad);
    R.jv.reserve(3 * npad);
    if (!R.ev0) {
        NB6_CUDA_CHECK(cudaEventCreate(&R.ev0));
        NB6_CUDA_CHECK(cudaEventCreate(&R.ev1));
    }
    if (getenv("NB6_VERBOSE"))
        fprintf(stderr, "# Open GPU regular force - rank: %d; nbmax: %d\n", *irank, *nbmax);
}

void gpunb_close_() {
    if (!R.open) {
        fprintf(stderr, "gpunb: it is already close\n");
        return;
    }
    R.open = false;
    R.posH.release();
    R.posL.release();
    R.vel.release();
    R.jm.release();
    R.jx.release();
    R.jv.release();
    R.iin.release();
    R.part.release();
    R.nbcnt.release();
    R.nbbuf.release();
    R.outf.release();
    R.outl.release();
    R.hin.release();
    R.houtf.release();
    R.houtl.release();
    R.nbodymax = 0;
    R.nj = 0;
}

void gpunb_send_(int *nj, double *mj, double (*xj)[3], double (*vj)[3]) {
    if (!R.open) {
        nb6_fatal(NB6_ERR_NOT_OPEN);
        return;
    }
    const int n = *nj;
    if (n < 0 || n > R.nbodymax) {
        fprintf(stderr, "gpunb_send: nj=%d outside [0, nbmax=%d]\n", n, R.nbodymax);
        nb6_fatal(NB6_ERR_TOO_LARGE);
        return;
    }
    R.time_send -= nb6_wtime();
    R.isend++;
    cudaStream_t st = nb6_stream();
    R.nj = n;
    R.ntile = std::max(1, (n + JT - 1) / JT);
    const size_t npad = (size_t)R.ntile * JT;
    R.posH.reserve(npad);
    R.posL.reserve(npad);
    R.vel.reserve(npad);
    R.jm.reserve(npad);
    R.jx.reserve(3 * npad);
    R.jv.reserve(3 * npad);
    if (n > 0) {
        NB6_CUDA_CHECK(cudaMemcpyAsync(R.jm.ptr, mj, sizeof(double) * n, cudaMemcpyHostToDevice, st));
        NB6_CUDA_CHECK(cudaMemcpyAsync(R.jx.ptr, xj, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, st));
        NB6_CUDA_CHECK(cudaMemcpyAsync(R.jv.ptr, vj, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, st));
    }
    const int blocks = (int)std::min<size_t>((npad + 255) / 256, (size_t)nb6_num_sms() * 8);
    regf_pack_j<<<blocks, 256, 0, st>>>(n, (int)npad, R.jm.ptr, R.jx.ptr, R.jv.ptr, R.posH.ptr,
                                        R.posL.ptr, R.vel.ptr, nb6_dev_status());
    NB6_CUDA_CHECK(cudaGetLastError());
    R.time_send += nb6_wtime();
}

}  // extern "C"

// Internal hook for the device-resident predictor (predictor.cu): a send whose
// j data are produced on the device.  Sizes the j buffers for n bodies, makes
// them current, and hands out the arrays to fill (FP64 m, x, v for the exact
// neighbour recheck and the float4 tiles, padded to *npad with far massless
// bodies by the caller's kernel).
bool regular_bind_j(int n, double **jm, double **jx, double **jv, float4 **posH, float4 **posL,
                    float4 **vel, int *npad) {
    if (!R.open) {
        nb6_fatal(NB6_ERR_NOT_OPEN);
        return false;
    }
    if (n < 0 || n > R.nbodymax) {
        fprintf(stderr, "nb6_predict_send: n=%d outside [0, nbmax=%d]\n", n, R.nbodymax);
        nb6_fatal(NB6_ERR_TOO_LARGE);
        return false;
    }
    R.isend++;
    R.nj = n;
    R.ntile = std::max(1, (n + JT - 1) / JT);
    const size_t np = (size_t)R.ntile * JT;
    R.posH.reserve(np);
    R.posL.reserve(np);
    R.vel.reserve(np);
    R.jm.reserve(np);
    R.jx.reserve(3 * np);
    R.jv.reserve(3 * np);
    *jm = R.jm.ptr;
    *jx = R.jx.ptr;
    *jv = R.jv.ptr;
    *posH = R.posH.ptr;
    *posL = R.posL.ptr;
    *vel = R.vel.ptr;
    *npad = (int)np;
    return true;
}

extern "C" {

void gpunb_regf_(int *ni_, double *h2, double *dtr, double (*xi)[3], double (*vi)[3],
                 double (*acc)[3], double (*jrk)[3], double *pot, int *lmax_, int *nnbmax_,
                 int *list, int *m_flag) {
    if (!R.open) {
        nb6_fatal(NB6_ERR_NOT_OPEN);
        return;
    }
    const int ni = *ni_;
    const int lmax = *lmax_;
    const int nnbmax = *nnbmax_;
    if (ni <= 0 || lmax < 1 || std::min(nnbmax, lmax - 1) > 8191) {
        fprintf(stderr, "gpunb_regf: bad ni=%d, lmax=%d or list cap min(nnbmax,lmax-1) > 8191\n",
                ni, lmax);
        nb6_fatal(NB6_ERR_BAD_ARG);
        return;
    }
    if (any_nan(h2, ni) || any_nan(dtr, ni) || any_nan(&xi[0][0], 3 * (size_t)ni) ||
        any_nan(&vi[0][0], 3 * (size_t)ni)) {
        fprintf(stderr, "gpunb_regf: NaN in i-particle input\n");
        nb6_fatal(NB6_ERR_NAN_INPUT);
        return;
    }
    R.time_grav -= nb6_wtime();
    R.numInter += (long long)ni * R.nj;
    R.ini += ni;
    R.icall++;
    cudaStream_t st = nb6_stream();

    // stage i data: [h2 | dtr | x | v] in one pinned block, one H2D
    const size_t nin = (size_t)8 * ni;
    R.hin.reserve(nin);
    R.iin.reserve(nin);
    double *h = R.hin.ptr;
    memcpy(h, h2, sizeof(double) * ni);
    memcpy(h + ni, dtr, sizeof(double) * ni);
    memcpy(h + 2 * (size_t)ni, xi, sizeof(double) * 3 * ni);
    memcpy(h + 5 * (size_t)ni, vi, sizeof(double) * 3 * ni);
    NB6_CUDA_CHECK(cudaMemcpyAsync(R.iin.ptr, h, sizeof(double) * nin, cudaMemcpyHostToDevice, st));
    const double *d = R.iin.ptr;

    int W = 0;
    regf_device(ni, d, d + ni, d + 2 * (size_t)ni, d + 5 * (size_t)ni, lmax, nnbmax, *m_flag, st, W);

    R.houtf.reserve((size_t)ni * 8);
    R.houtl.reserve((size_t)ni * W);
    NB6_CUDA_CHECK(cudaMemcpyAsync(R.houtf.ptr, R.outf.ptr, sizeof(double) * 8 * ni,
                                   cudaMemcpyDeviceToHost, st));
    NB6_CUDA_CHECK(cudaMemcpyAsync(R.houtl.ptr, R.outl.ptr, sizeof(int) * (size_t)W * ni,
                                   cudaMemcpyDeviceToHost, st));
    NB6_CUDA_CHECK(cudaStreamSynchronize(st));
    NB6_CUDA_CHECK(cudaEventElapsedTime(&R.last_kernel_ms, R.ev0, R.ev1));
    const double wt = nb6_wtime();
    R.time_grav += wt;
    R.time_reduce -= wt;
    if (nb6_check_dev_status() != 0) return;

    const double *of = R.houtf.ptr;
    const int *ol = R.houtl.ptr;
    for (int i = 0; i < ni; ++i) {
        acc[i][0] = of[8 * i + 0];
        acc[i][1] = of[8 * i + 1];
        acc[i][2] = of[8 * i + 2];
        jrk[i][0] = of[8 * i + 3];
        jrk[i][1] = of[8 * i + 4];
        jrk[i][2] = of[8 * i + 5];
        pot[i] = of[8 * i + 6];
        const int *src = ol + (size_t)i * W;
        int *dst = list + (size_t)i * lmax;
        const int nnb = src[0];
        dst[0] = nnb;
        if (nnb > 0) memcpy(dst + 1, src + 1, sizeof(int) * nnb);
    }
    R.time_reduce += nb6_wtime();
}

void gpunb_profile_(int *irank) {
    if (R.icall) {
        const int per = R.isend ? R.ini / R.isend : R.ini;
        const double gf = R.time_grav > 0 ? 60.e-9 * (double)R.numInter / R.time_grav : 0.0;
        fprintf(stderr,
                "[R.%d GPU Reg.F ] Nsend %d  Ngrav %d  <Ni> %d   send(s) %f grav(s) %f  nb(s) %f  "
                "out(s) %f  Perf.(Gflops) %f\n",
                *irank, R.isend, R.icall, per, R.time_send, R.time_grav, R.time_reduce, R.time_out, gf);
    }
    R.time_send = R.time_grav = R.time_reduce = R.time_out = 0.0;
    R.numInter = 0;
    R.icall = R.ini = R.isend = 0;
}

// ---------------------------------------------------------------------------
// Extension entry points (no reference counterpart).
// ---------------------------------------------------------------------------

// Device-resident variant of gpunb_regf_ for benchmarking and for drivers
// that keep i data on the GPU: pointers are DEVICE pointers laid out as in
// gpunb_regf_; results stay in the library's device output buffers and are
// fetched with nb6_regf_fetch_.  Enqueued on the library stream, no sync.
void nb6_regf_device_(int *ni, const double *d_h2, const double *d_dtr, const double *d_x,
                      const double *d_v, int *lmax, int *nnbmax, int *m_flag) {
    int W;
    regf_device(*ni, d_h2, d_dtr, d_x, d_v, *lmax, *nnbmax, *m_flag, nb6_stream(), W);
}

// Device pointers of the last regf outputs: outf [ni][8] doubles
// (acc3, jrk3, pot, 0) and outl [ni][W] ints with W = min(nnbmax, lmax-1)+1.
void nb6_regf_outputs_(double **d_outf, int **d_outl) {
    *d_outf = R.outf.ptr;
    *d_outl = R.outl.ptr;
}

// Kernel-only device time (ms) of the last gpunb_regf_ call.
float nb6_regf_last_kernel_ms_() {
    if (!R.ev1) return 0.f;
    NB6_CUDA_CHECK(cudaEventSynchronize(R.ev1));
    NB6_CUDA_CHECK(cudaEventElapsedTime(&R.last_kernel_ms, R.ev0, R.ev1));
    return R.last_kernel_ms;
}

// Launch geometry of the last regf launch: i per thread, i-tiles, j-slices.
void nb6_regf_last_geometry_(int *geom) {
    geom[0] = R.last_geometry[0];
    geom[1] = R.last_geometry[1];
    geom[2] = R.last_geometry[2];
}

// Launch-geometry override for tuning sweeps: i per thread (1, 2, 4; 0 =
// automatic) and j-slice count (0 = automatic).
void nb6_regf_tune_(int *ni_per_thread, int *nslices) {
    R.forced_ni_per_thread = *ni_per_thread;
    R.forced_slices = *nslices;
}

void nb6_sync_() { NB6_CUDA_CHECK(cudaStreamSynchronize(nb6_stream())); nb6_check_dev_status(); }

void *nb6_stream_() { return (void *)nb6_stream(); }

}  // extern "C"
