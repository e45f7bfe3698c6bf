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
#include "copy_pool.h"
#include "mlp.cuh"

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <climits>
#include <map>
#include <mutex>
#include <vector>
#include <math.h>
#include <string.h>

MlpArgs nb6_mlp_args(const double *h2, const double *dtr);  // mlp.cu

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
// Minimum resident CTAs per SM requested for the packed kernel with one i
// per thread (halved for two): bounds its register allocation.
#ifndef X2_MINB
#define X2_MINB 4
#endif
// The rare candidate path is inlined: an out-of-line call forces the
// accumulators through a stack frame.
#ifndef FLUSH_INLINE
#define FLUSH_INLINE __forceinline__
#endif

struct RegArgs {
    const float4 *__restrict__ posH;  // (xH, yH, zH, m)
    const float4 *__restrict__ posL;  // (xL, yL, zL, 0)
    const float4 *__restrict__ vel;   // (vx, vy, vz, 0)
    const float *__restrict__ comp;   // component-major copy (NB6_NCOMP x npad)
    const double *__restrict__ compd; // FP64 positions, component-major (3 x npad)
    size_t npad;
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
    // spatially ordered j set: slot k holds body perm[k]; tile t's bounding
    // box is tbox[2t] = (centre xyz, max |v|), tbox[2t+1] = (half extent xyz,
    // max m).  Null: j slots are the caller's order, no boxes.
    const int *__restrict__ perm = nullptr;
    const float4 *__restrict__ tbox = nullptr;
    // packed kernel: thread slot s takes i-particle iperm[s] (the active set
    // in the same spatial order, so a warp covers a compact region); null =
    // slot order.  Every index into i data and outputs stays the caller's.
    const int *__restrict__ iperm = nullptr;
    // ordered j set only: positions relative to their tile's box centre,
    // fl32(x - c), component-major (3 x npad) -- the far-tile operands
    const float *__restrict__ comprel = nullptr;
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

// Exact FP64 decision for one candidate pair (i, j): record j as a neighbour
// or, if it is not one, add its contribution (which the hot loop masked).
// Operation order matches the FP64 rule of regint.f:41-65 with the strict
// "<" of gpunb.velocity.cu:188,236; no FMA contraction.
template <bool MFLAG>
NB6_DEV void reg_exact(const RegArgs &a, int i, int jslot, Sums &s, int joff = 0) {
    const int j = a.perm ? a.perm[jslot] : jslot;  // the caller's index of the body in this slot
    const double xi0 = a.ix[3 * i], xi1 = a.ix[3 * i + 1], xi2 = a.ix[3 * i + 2];
    const double vi0 = a.iv[3 * i], vi1 = a.iv[3 * i + 1], vi2 = a.iv[3 * i + 2];
    const double h2 = a.ih2[i], dt = a.idtr[i];
    {
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
            if (pos < a.lcap) a.nbbuf[(size_t)i * a.lcap + pos] = j - joff;
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
}

// Rare path for one i and one 32-j group that held at least one candidate:
// re-derive the candidates with the same FP32 test, decide each in FP64.
template <bool MFLAG>
__device__ FLUSH_INLINE Sums reg_flush(const RegArgs &a, const IPart ip, int i, const float4 *A,
                                       const float4 *B, const float4 *Cv, int jbase, Sums s) {
    for (int b = 0; b < 32; ++b) {
        if (!reg_geom<MFLAG>(ip, A[b], B[b], Cv[b]).cand) continue;
        const int j = jbase + b;
        if (j >= a.nj) continue;  // padding slots are never neighbours
        reg_exact<MFLAG>(a, i, j, s);
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
    __shared__ __align__(8) uint64_t ebar[NSTAGE];

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

    // Ring of NSTAGE tiles.  bar[st] completes when a tile's bulk copies have
    // landed; ebar[st] when every warp has finished reading it.  Warps release
    // stages independently, so they can drift up to NSTAGE-1 tiles apart and
    // only the producer (thread 0) ever waits for the slowest warp.
    const int lane = tid & 31;
    if (tid == 0) {
#pragma unroll
        for (int st = 0; st < NSTAGE; ++st) {
            mbar_init(&bar[st], 1);
            mbar_init(&ebar[st], NT / 32);
        }
        fence_mbar_init();
    }
    __syncthreads();
    int issued = 0;  // tiles issued so far (thread 0 only)
    if (tid == 0) {
        for (int st = 0; st < NSTAGE && st < nt; ++st) issue_tile(a, sj[st], &bar[st], t_begin + st);
        issued = min(nt, NSTAGE);
    }

    for (int t = 0; t < nt; ++t) {
        const int st = t % NSTAGE;
        const uint32_t par = (uint32_t)((t / NSTAGE) & 1);
        const bool ok = __all_sync(0xffffffffu, mbar_wait_timed(&bar[st], par, WAIT_NS));
        if (!ok) {
            set_status(a.status, NB6_ERR_WAIT_TIMEOUT);
            if (tid == 0)  // drain copies still in flight before the CTA's smem goes away
                for (int u = t; u < issued; ++u)
                    mbar_wait_timed(&bar[u % NSTAGE], (uint32_t)((u / NSTAGE) & 1), WAIT_NS / 8);
            return;
        }

        const float4 *A = sj[st][0];
        const float4 *B = sj[st][1];
        const float4 *C = sj[st][2];
        const int jt0 = (t_begin + t) * JT;
#pragma unroll 1
        for (int g = 0; g < JT / 32; ++g) {
            unsigned anyc[NI];
#pragma unroll
            for (int k = 0; k < NI; ++k) anyc[k] = 0u;
            const float4 *Ag = A + g * 32, *Bg = B + g * 32, *Cg = C + g * 32;
#pragma unroll kUnrollJ
            for (int q = 0; q < 32; ++q) {
                const float4 pa = Ag[q];
                const float4 pb = Bg[q];
                const float4 pc = Cg[q];
#pragma unroll
                for (int k = 0; k < NI; ++k) anyc[k] += reg_pair<MFLAG>(ip[k], pa, pb, pc, s[k]) ? 1u : 0u;
            }
#pragma unroll
            for (int k = 0; k < NI; ++k)
                if (anyc[k]) s[k] = reg_flush<MFLAG>(a, ip[k], ii[k], Ag, Bg, Cg, jt0 + g * 32, s[k]);
        }
        // this warp is done with the stage
        __syncwarp();
        if (lane == 0) mbar_arrive(&ebar[st]);
        if (tid == 0 && t + NSTAGE < nt) {
            // once every warp has released tile t, refill its stage
            if (!mbar_wait_timed(&ebar[st], par, WAIT_NS)) {
                set_status(a.status, NB6_ERR_WAIT_TIMEOUT);
                for (int u = t + 1; u < issued; ++u)
                    mbar_wait_timed(&bar[u % NSTAGE], (uint32_t)((u / NSTAGE) & 1), WAIT_NS / 8);
                return;
            }
            issue_tile(a, sj[st], &bar[st], t_begin + t + NSTAGE);
            issued = t + NSTAGE + 1;
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

// ----------------------------------------------------------------------------
// Packed variant: two j per instruction in the f32x2 lanes (fma/add/mul.f32x2
// of sm_100).  Each FP32 add/mul/fma of the pair math processes two pairs per
// issue slot, which moves the kernel from issue-bound to FMA-pipe-bound.  The
// j tile sits in shared memory component-major (NB6_NCOMP rows of JT floats),
// so one LDS.128 brings four consecutive j of one component.  The arithmetic
// is the scalar reg_pair's, operation for operation (negated i operands turn
// subtractions into adds; sums are kept negated), so candidates and results
// are bit-identical to the scalar kernels -- except on the far tiles of an
// ordered j set, which take tile-relative differences and 1/r without the
// Newton step (pair_x2_rel).
// ----------------------------------------------------------------------------
struct IP2 {
    float2 nxh, nyh, nzh, nxl, nyl, nzl, nvx, nvy, nvz, h2c, dt;  // i data, negated, duplicated
};

struct S2 {
    float2 ax, ay, az, jx, jy, jz, po;  // -(scaled sums), lane = j parity
};

NB6_DEV float2 dup2(float v) { return make_float2(v, v); }

NB6_DEV void zero2(S2 &s) {
    s.ax = s.ay = s.az = s.jx = s.jy = s.jz = s.po = make_float2(0.f, 0.f);
}

// Returns the candidate flags of the two lanes as bits 0 and 1.
template <bool MFLAG>
NB6_DEV unsigned pair_x2(const IP2 &ip, float2 xh, float2 yh, float2 zh, float2 m, float2 xl,
                         float2 yl, float2 zl, float2 vx, float2 vy, float2 vz, S2 &s) {
    const float2 dx = __fadd2_rn(__fadd2_rn(xh, ip.nxh), __fadd2_rn(xl, ip.nxl));
    const float2 dy = __fadd2_rn(__fadd2_rn(yh, ip.nyh), __fadd2_rn(yl, ip.nyl));
    const float2 dz = __fadd2_rn(__fadd2_rn(zh, ip.nzh), __fadd2_rn(zl, ip.nzl));
    const float2 dvx = __fadd2_rn(vx, ip.nvx);
    const float2 dvy = __fadd2_rn(vy, ip.nvy);
    const float2 dvz = __fadd2_rn(vz, ip.nvz);
    const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
    const float2 px = __ffma2_rn(ip.dt, dvx, dx);
    const float2 py = __ffma2_rn(ip.dt, dvy, dy);
    const float2 pz = __ffma2_rn(ip.dt, dvz, dz);
    const float2 rp2 = __ffma2_rn(pz, pz, __ffma2_rn(py, py, __fmul2_rn(px, px)));
    const float2 crit = MFLAG ? __fmul2_rn(m, ip.h2c) : ip.h2c;
    const bool c0 = fminf(r2.x, rp2.x) < crit.x;
    const bool c1 = fminf(r2.y, rp2.y) < crit.y;
    const float2 rv = __ffma2_rn(dz, dvz, __ffma2_rn(dy, dvy, __fmul2_rn(dx, dvx)));
    float2 y0;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y0.x) : "f"(r2.x));
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y0.y) : "f"(r2.y));
    const float2 ra = __fmul2_rn(r2, y0);
    const float2 nb = __ffma2_rn(ra, y0, dup2(-3.0f));   // -(3 - r2 y0^2)
    float2 ny = __fmul2_rn(y0, nb);                      // -2/r
    ny.x = c0 ? 0.0f : ny.x;
    ny.y = c1 ? 0.0f : ny.y;
    const float2 y2 = __fmul2_rn(ny, ny);
    const float2 nmy = __fmul2_rn(m, ny);
    const float2 nmy3 = __fmul2_rn(nmy, y2);
    const float2 al = __fmul2_rn(__fmul2_rn(y2, dup2(-0.75f)), rv);
    s.po = __fadd2_rn(s.po, nmy);
    s.ax = __ffma2_rn(nmy3, dx, s.ax);
    s.ay = __ffma2_rn(nmy3, dy, s.ay);
    s.az = __ffma2_rn(nmy3, dz, s.az);
    s.jx = __ffma2_rn(nmy3, __ffma2_rn(al, dx, dvx), s.jx);
    s.jy = __ffma2_rn(nmy3, __ffma2_rn(al, dy, dvy), s.jy);
    s.jz = __ffma2_rn(nmy3, __ffma2_rn(al, dz, dvz), s.jz);
    return (c0 ? 1u : 0u) | (c1 ? 2u : 0u);
}

// Far pair from tile-relative coordinates: xr = fl32(x_j - c) (stored with
// the ordered j set) and nxr = -fl32(x_i - c) (formed per tile in FP64), c
// the tile's box centre, so each difference is one FP32 add instead of
// three.  With the tile at least one half extent h away from i, the
// three roundings (of x_j - c, x_i - c and their difference) stay within
// u (|x_j - c| + |x_i - c| + r) <= u (2h + 2r) <= 4u r of the separation r
// (u = 2^-24): four FP32 ulps of an FP64-formed difference at most.
template <bool MFLAG>
NB6_DEV void pair_x2_rel(const IP2 &ip, float2 nxr, float2 nyr, float2 nzr, float2 xr, float2 yr, float2 zr,
                         float2 m, float2 vx, float2 vy, float2 vz, S2 &s) {
    const float2 dx = __fadd2_rn(xr, nxr);
    const float2 dy = __fadd2_rn(yr, nyr);
    const float2 dz = __fadd2_rn(zr, nzr);
    const float2 dvx = __fadd2_rn(vx, ip.nvx);
    const float2 dvy = __fadd2_rn(vy, ip.nvy);
    const float2 dvz = __fadd2_rn(vz, ip.nvz);
    const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
    const float2 rv = __ffma2_rn(dz, dvz, __ffma2_rn(dy, dvy, __fmul2_rn(dx, dvx)));
    float2 y0;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y0.x) : "f"(r2.x));
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y0.y) : "f"(r2.y));
    // No Newton step on a far pair: 1/r straight from the approximation.
    // A far pair is individually weak, so the approximation's relative
    // error enters the force as a near-uniform scaling of the far field;
    // the parity tests and the bench's FP64 check bound the result.
    // The sums of a far tile are kept unscaled and positive (m/r, m dx/r^3,
    // ...); the tile's fold applies the exact factors 2 and 8 of the
    // other paths' convention, so a far pair costs 27 lane operations.
    const float2 u = __fmul2_rn(m, y0);   // m/r
    const float2 w = __fmul2_rn(y0, y0);  // 1/r^2
    const float2 u3 = __fmul2_rn(u, w);   // m/r^3
    const float2 al = __fmul2_rn(__fmul2_rn(w, dup2(-3.0f)), rv);
    s.po = __fadd2_rn(s.po, u);
    s.ax = __ffma2_rn(u3, dx, s.ax);
    s.ay = __ffma2_rn(u3, dy, s.ay);
    s.az = __ffma2_rn(u3, dz, s.az);
    s.jx = __ffma2_rn(u3, __ffma2_rn(al, dx, dvx), s.jx);
    s.jy = __ffma2_rn(u3, __ffma2_rn(al, dy, dvy), s.jy);
    s.jz = __ffma2_rn(u3, __ffma2_rn(al, dz, dvz), s.jz);
}

// True when no body of tile box (bc, bh) can be a neighbour candidate of the
// i-particle: the box is farther than sqrt(crit) + dtr (|v_i| + max |v_j|),
// the farthest reach of min(r, |r + dtr dv|) < sqrt(crit) (triangle
// inequality), with margins for the FP32 rounding of positions, box and test.
template <bool MFLAG>
NB6_DEV bool tile_far(const IP2 &ip, float vabs, float4 bc, float4 bh) {
    const float xi = -ip.nxh.x, yi = -ip.nyh.x, zi = -ip.nzh.x;
    const float ex = fmaxf(fabsf(xi - bc.x) - bh.x, 0.f);
    const float ey = fmaxf(fabsf(yi - bc.y) - bh.y, 0.f);
    const float ez = fmaxf(fabsf(zi - bc.z) - bh.z, 0.f);
    const float d2 = ex * ex + ey * ey + ez * ez;
    const float crit = MFLAG ? bh.w * ip.h2c.x : ip.h2c.x;
    const float mag = fmaxf(fmaxf(fabsf(xi), fabsf(yi)), fabsf(zi)) +
                      fmaxf(fmaxf(fabsf(bc.x) + bh.x, fabsf(bc.y) + bh.y), fabsf(bc.z) + bh.z);
    const float reach = (sqrtf(crit) + ip.dt.x * (vabs + bc.w)) * 1.001f + mag * 1.0e-6f;
    // and, for the relative coordinates, at least one half extent away
    const float hmax = fmaxf(fmaxf(bh.x, bh.y), bh.z);
    return d2 > reach * reach && d2 > hmax * hmax;
}

// Same pair math with the coordinate differences formed in FP64 and rounded
// once to FP32 (DADD + F2F on the FP64 pipe instead of three FP32 adds per
// component on the FMA pipe).  xi/yi/zi are the i position in FP64.
template <bool MFLAG>
NB6_DEV unsigned pair_x2d(const IP2 &ip, double xi, double yi, double zi, double2 xj, double2 yj,
                          double2 zj, float2 m, float2 vx, float2 vy, float2 vz, S2 &s) {
    const float2 dx = make_float2(__double2float_rn(xj.x - xi), __double2float_rn(xj.y - xi));
    const float2 dy = make_float2(__double2float_rn(yj.x - yi), __double2float_rn(yj.y - yi));
    const float2 dz = make_float2(__double2float_rn(zj.x - zi), __double2float_rn(zj.y - zi));
    const float2 dvx = __fadd2_rn(vx, ip.nvx);
    const float2 dvy = __fadd2_rn(vy, ip.nvy);
    const float2 dvz = __fadd2_rn(vz, ip.nvz);
    const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
    const float2 px = __ffma2_rn(ip.dt, dvx, dx);
    const float2 py = __ffma2_rn(ip.dt, dvy, dy);
    const float2 pz = __ffma2_rn(ip.dt, dvz, dz);
    const float2 rp2 = __ffma2_rn(pz, pz, __ffma2_rn(py, py, __fmul2_rn(px, px)));
    const float2 crit = MFLAG ? __fmul2_rn(m, ip.h2c) : ip.h2c;
    const bool c0 = fminf(r2.x, rp2.x) < crit.x;
    const bool c1 = fminf(r2.y, rp2.y) < crit.y;
    const float2 rv = __ffma2_rn(dz, dvz, __ffma2_rn(dy, dvy, __fmul2_rn(dx, dvx)));
    float2 y0;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y0.x) : "f"(r2.x));
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y0.y) : "f"(r2.y));
    const float2 ra = __fmul2_rn(r2, y0);
    const float2 nb = __ffma2_rn(ra, y0, dup2(-3.0f));
    float2 ny = __fmul2_rn(y0, nb);
    ny.x = c0 ? 0.0f : ny.x;
    ny.y = c1 ? 0.0f : ny.y;
    const float2 y2 = __fmul2_rn(ny, ny);
    const float2 nmy = __fmul2_rn(m, ny);
    const float2 nmy3 = __fmul2_rn(nmy, y2);
    const float2 al = __fmul2_rn(__fmul2_rn(y2, dup2(-0.75f)), rv);
    s.po = __fadd2_rn(s.po, nmy);
    s.ax = __ffma2_rn(nmy3, dx, s.ax);
    s.ay = __ffma2_rn(nmy3, dy, s.ay);
    s.az = __ffma2_rn(nmy3, dz, s.az);
    s.jx = __ffma2_rn(nmy3, __ffma2_rn(al, dx, dvx), s.jx);
    s.jy = __ffma2_rn(nmy3, __ffma2_rn(al, dy, dvy), s.jy);
    s.jz = __ffma2_rn(nmy3, __ffma2_rn(al, dz, dvz), s.jz);
    return (c0 ? 1u : 0u) | (c1 ? 2u : 0u);
}

// Rare path: the candidates of one 32-j group, as recorded bit by bit by the
// hot loop, each decided exactly in FP64.
template <bool MFLAG>
NB6_DEV Sums reg_flush_mask(const RegArgs &a, int i, unsigned mask, int jbase, Sums s) {
    while (mask) {
        const int b = __ffs(mask) - 1;
        mask &= mask - 1;
        const int j = jbase + b;
        if (j >= a.nj) continue;  // padding slots are never neighbours
        reg_exact<MFLAG>(a, i, j, s);
    }
    return s;
}

// One tile into a stage of NB6_NCOMP float rows.  FP32 layout: the ten float
// components.  FP64 layout: x, y, z as doubles in row pairs (0,1) (2,3) (4,5),
// then m, vx, vy, vz in rows 6..9 -- the same 10*JT*4 bytes.
template <bool F64DX>
NB6_DEV void issue_tile_soa(const RegArgs &a, float (*stage)[JT], uint64_t *bar, int tile) {
    const size_t off = (size_t)tile * JT;
    // rows 10..12: the tile-relative positions of an ordered j set
    const bool rel = !F64DX && a.comprel != nullptr;
    mbar_arrive_expect_tx(bar, (uint32_t)((NB6_NCOMP + (rel ? 3 : 0)) * JT * sizeof(float)));
    if constexpr (F64DX) {
#pragma unroll
        for (int c = 0; c < 3; ++c)
            bulk_g2s(stage[2 * c], a.compd + (size_t)c * a.npad + off, JT * sizeof(double), bar);
        bulk_g2s(stage[6], a.comp + (size_t)3 * a.npad + off, JT * sizeof(float), bar);
#pragma unroll
        for (int c = 7; c < 10; ++c)
            bulk_g2s(stage[c], a.comp + (size_t)c * a.npad + off, JT * sizeof(float), bar);
    } else {
#pragma unroll
        for (int c = 0; c < NB6_NCOMP; ++c)
            bulk_g2s(stage[c], a.comp + (size_t)c * a.npad + off, JT * sizeof(float), bar);
        if (rel) {
#pragma unroll
            for (int c = 0; c < 3; ++c)
                bulk_g2s(stage[NB6_NCOMP + c], a.comprel + (size_t)c * a.npad + off, JT * sizeof(float), bar);
        }
    }
}

template <int NI, bool MFLAG, bool F64DX = false>
__global__ void __launch_bounds__(NT, X2_MINB / NI) regf_x2_kernel(const RegArgs a) {
    __shared__ __align__(128) float sj[NSTAGE][NB6_NCOMP + 3][JT];
    __shared__ __align__(8) uint64_t bar[NSTAGE];
    __shared__ __align__(8) uint64_t ebar[NSTAGE];
    // double-single accumulators, touched once per tile: kept in shared
    // memory (thread-private slots) to free registers for the pair math
    __shared__ float2 dsum[NI][7][NT];

    const int tid = threadIdx.x, lane = tid & 31;
    const int slice = blockIdx.y;
    // Tiles of this slice: a contiguous range, or with a spatially ordered j
    // set (a.tbox) every nslices-th tile, so that the tiles near a compact
    // group of i-particles -- the ones with neighbour candidates -- are
    // shared out among the slices instead of falling to one CTA.
    const bool strided = a.tbox != nullptr;
    const int t_begin = strided ? slice : (int)(((long long)slice * a.ntile) / a.nslices);
    const int t_step = strided ? a.nslices : 1;
    const int nt = strided ? (slice < a.ntile ? (a.ntile - slice + a.nslices - 1) / a.nslices : 0)
                           : (int)(((long long)(slice + 1) * a.ntile) / a.nslices) - t_begin;

    IP2 ip[NI];
    S2 s[NI];
    Sums fx[NI];
    int ii[NI];
    float vabs[NI];                 // |v_i|, for the tile reach test
    double xd[NI], yd[NI], zd[NI];  // FP64 i position (F64DX layout)
#pragma unroll
    for (int k = 0; k < NI; ++k) {
        const int slot = blockIdx.x * (NT * NI) + k * NT + tid;
        const int i = (a.iperm && slot < a.ni) ? a.iperm[slot] : slot;
        ii[k] = i;
        zero2(s[k]);
        zero(fx[k]);
#pragma unroll
        for (int c = 0; c < 7; ++c) dsum[k][c][tid] = make_float2(0.f, 0.f);
        xd[k] = i < a.ni ? a.ix[3 * i] : 0.0;
        yd[k] = i < a.ni ? a.ix[3 * i + 1] : 0.0;
        zd[k] = i < a.ni ? a.ix[3 * i + 2] : 0.0;
        IPart p;
        if (i < a.ni) {
            split_hl(a.ix[3 * i], p.xh, p.xl);
            split_hl(a.ix[3 * i + 1], p.yh, p.yl);
            split_hl(a.ix[3 * i + 2], p.zh, p.zl);
            p.vx = (float)a.iv[3 * i];
            p.vy = (float)a.iv[3 * i + 1];
            p.vz = (float)a.iv[3 * i + 2];
            p.h2c = (float)a.ih2[i] * CAND_SLACK;
            p.dt = (float)a.idtr[i];
        } else {
            p.xh = p.yh = p.zh = p.xl = p.yl = p.zl = p.vx = p.vy = p.vz = 0.f;
            p.h2c = 0.f;  // padding lanes: never a candidate
            p.dt = 0.f;
        }
        ip[k].nxh = dup2(-p.xh);
        ip[k].nyh = dup2(-p.yh);
        ip[k].nzh = dup2(-p.zh);
        ip[k].nxl = dup2(-p.xl);
        ip[k].nyl = dup2(-p.yl);
        ip[k].nzl = dup2(-p.zl);
        ip[k].nvx = dup2(-p.vx);
        ip[k].nvy = dup2(-p.vy);
        ip[k].nvz = dup2(-p.vz);
        ip[k].h2c = dup2(p.h2c);
        ip[k].dt = dup2(p.dt);
        vabs[k] = sqrtf(p.vx * p.vx + p.vy * p.vy + p.vz * p.vz);
    }

    if (tid == 0) {
#pragma unroll
        for (int st = 0; st < NSTAGE; ++st) {
            mbar_init(&bar[st], 1);
            mbar_init(&ebar[st], NT / 32);
        }
        fence_mbar_init();
    }
    __syncthreads();
    int issued = 0;
    if (tid == 0) {
        for (int st = 0; st < NSTAGE && st < nt; ++st)
            issue_tile_soa<F64DX>(a, sj[st], &bar[st], t_begin + st * t_step);
        issued = min(nt, NSTAGE);
    }

    for (int t = 0; t < nt; ++t) {
        const int st = t % NSTAGE;
        const uint32_t par = (uint32_t)((t / NSTAGE) & 1);
        const bool ok = __all_sync(0xffffffffu, mbar_wait_timed(&bar[st], par, WAIT_NS));
        if (!ok) {
            set_status(a.status, NB6_ERR_WAIT_TIMEOUT);
            if (tid == 0)
                for (int u = t; u < issued; ++u)
                    mbar_wait_timed(&bar[u % NSTAGE], (uint32_t)((u / NSTAGE) & 1), WAIT_NS / 8);
            return;
        }
        const float(*S)[JT] = sj[st];
        const int tile = t_begin + t * t_step;
        const int jt0 = tile * JT;
        // whole warp out of reach of this tile: no candidates, short loop
        bool far = false;
        float2 nxr[NI], nyr[NI], nzr[NI];  // -fl32(x_i - c) of this tile (far path)
        if constexpr (!F64DX && NI == 1) {  // (two i per thread: no registers left for it)
            if (a.comprel) {
                const float4 bc = __ldg(&a.tbox[2 * tile]);
                const float4 bh = __ldg(&a.tbox[2 * tile + 1]);
                bool f = true;
#pragma unroll
                for (int k = 0; k < NI; ++k) f = f && (ii[k] >= a.ni || tile_far<MFLAG>(ip[k], vabs[k], bc, bh));
                far = __all_sync(0xffffffffu, f);
                if (far) {
#pragma unroll
                    for (int k = 0; k < NI; ++k) {
                        nxr[k] = dup2(-__double2float_rn(xd[k] - (double)bc.x));
                        nyr[k] = dup2(-__double2float_rn(yd[k] - (double)bc.y));
                        nzr[k] = dup2(-__double2float_rn(zd[k] - (double)bc.z));
                    }
                }
            }
        }
        if constexpr (!F64DX && NI == 1) {
          if (far) {
#pragma unroll 1
            for (int g = 0; g < JT / 32; ++g) {
#pragma unroll
                for (int u = 0; u < 32; u += 4) {
                    const int q = g * 32 + u;
                    const float4 MM = *reinterpret_cast<const float4 *>(&S[3][q]);
                    const float4 VX = *reinterpret_cast<const float4 *>(&S[7][q]);
                    const float4 VY = *reinterpret_cast<const float4 *>(&S[8][q]);
                    const float4 VZ = *reinterpret_cast<const float4 *>(&S[9][q]);
                    const float4 XR = *reinterpret_cast<const float4 *>(&S[NB6_NCOMP][q]);
                    const float4 YR = *reinterpret_cast<const float4 *>(&S[NB6_NCOMP + 1][q]);
                    const float4 ZR = *reinterpret_cast<const float4 *>(&S[NB6_NCOMP + 2][q]);
#pragma unroll
                    for (int k = 0; k < NI; ++k) {
                        pair_x2_rel<MFLAG>(ip[k], nxr[k], nyr[k], nzr[k], make_float2(XR.x, XR.y),
                                           make_float2(YR.x, YR.y), make_float2(ZR.x, ZR.y),
                                           make_float2(MM.x, MM.y), make_float2(VX.x, VX.y),
                                           make_float2(VY.x, VY.y), make_float2(VZ.x, VZ.y), s[k]);
                        pair_x2_rel<MFLAG>(ip[k], nxr[k], nyr[k], nzr[k], make_float2(XR.z, XR.w),
                                           make_float2(YR.z, YR.w), make_float2(ZR.z, ZR.w),
                                           make_float2(MM.z, MM.w), make_float2(VX.z, VX.w),
                                           make_float2(VY.z, VY.w), make_float2(VZ.z, VZ.w), s[k]);
                    }
                }
            }
          }
        }
#pragma unroll 1
        for (int g = 0; g < (far ? 0 : JT / 32); ++g) {
            unsigned cnt[NI];
#pragma unroll
            for (int k = 0; k < NI; ++k) cnt[k] = 0u;
            // fully unrolled: every candidate flag lands on a fixed mask bit
#pragma unroll
            for (int u = 0; u < 32; u += 4) {
                const int q = g * 32 + u;
                if constexpr (F64DX) {
                    const double *SX = reinterpret_cast<const double *>(S[0]);
                    const double *SY = reinterpret_cast<const double *>(S[2]);
                    const double *SZ = reinterpret_cast<const double *>(S[4]);
                    const double2 X0 = *reinterpret_cast<const double2 *>(SX + q);
                    const double2 X1 = *reinterpret_cast<const double2 *>(SX + q + 2);
                    const double2 Y0 = *reinterpret_cast<const double2 *>(SY + q);
                    const double2 Y1 = *reinterpret_cast<const double2 *>(SY + q + 2);
                    const double2 Z0 = *reinterpret_cast<const double2 *>(SZ + q);
                    const double2 Z1 = *reinterpret_cast<const double2 *>(SZ + q + 2);
                    const float4 MM = *reinterpret_cast<const float4 *>(&S[6][q]);
                    const float4 VX = *reinterpret_cast<const float4 *>(&S[7][q]);
                    const float4 VY = *reinterpret_cast<const float4 *>(&S[8][q]);
                    const float4 VZ = *reinterpret_cast<const float4 *>(&S[9][q]);
#pragma unroll
                    for (int k = 0; k < NI; ++k) {
                        const unsigned c01 = pair_x2d<MFLAG>(
                            ip[k], xd[k], yd[k], zd[k], X0, Y0, Z0, make_float2(MM.x, MM.y),
                            make_float2(VX.x, VX.y), make_float2(VY.x, VY.y), make_float2(VZ.x, VZ.y), s[k]);
                        const unsigned c23 = pair_x2d<MFLAG>(
                            ip[k], xd[k], yd[k], zd[k], X1, Y1, Z1, make_float2(MM.z, MM.w),
                            make_float2(VX.z, VX.w), make_float2(VY.z, VY.w), make_float2(VZ.z, VZ.w), s[k]);
                        cnt[k] |= (c01 | (c23 << 2)) << u;
                    }
                    continue;
                }
                const float4 XH = *reinterpret_cast<const float4 *>(&S[0][q]);
                const float4 YH = *reinterpret_cast<const float4 *>(&S[1][q]);
                const float4 ZH = *reinterpret_cast<const float4 *>(&S[2][q]);
                const float4 MM = *reinterpret_cast<const float4 *>(&S[3][q]);
                const float4 XL = *reinterpret_cast<const float4 *>(&S[4][q]);
                const float4 YL = *reinterpret_cast<const float4 *>(&S[5][q]);
                const float4 ZL = *reinterpret_cast<const float4 *>(&S[6][q]);
                const float4 VX = *reinterpret_cast<const float4 *>(&S[7][q]);
                const float4 VY = *reinterpret_cast<const float4 *>(&S[8][q]);
                const float4 VZ = *reinterpret_cast<const float4 *>(&S[9][q]);
#pragma unroll
                for (int k = 0; k < NI; ++k) {
                    const unsigned c01 =
                        pair_x2<MFLAG>(ip[k], make_float2(XH.x, XH.y), make_float2(YH.x, YH.y),
                                       make_float2(ZH.x, ZH.y), make_float2(MM.x, MM.y),
                                       make_float2(XL.x, XL.y), make_float2(YL.x, YL.y),
                                       make_float2(ZL.x, ZL.y), make_float2(VX.x, VX.y),
                                       make_float2(VY.x, VY.y), make_float2(VZ.x, VZ.y), s[k]);
                    const unsigned c23 =
                        pair_x2<MFLAG>(ip[k], make_float2(XH.z, XH.w), make_float2(YH.z, YH.w),
                                       make_float2(ZH.z, ZH.w), make_float2(MM.z, MM.w),
                                       make_float2(XL.z, XL.w), make_float2(YL.z, YL.w),
                                       make_float2(ZL.z, ZL.w), make_float2(VX.z, VX.w),
                                       make_float2(VY.z, VY.w), make_float2(VZ.z, VZ.w), s[k]);
                    cnt[k] |= (c01 | (c23 << 2)) << u;
                }
            }
#pragma unroll
            for (int k = 0; k < NI; ++k)
                if (cnt[k]) fx[k] = reg_flush_mask<MFLAG>(a, ii[k], cnt[k], jt0 + g * 32, fx[k]);
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&ebar[st]);
        if (tid == 0 && t + NSTAGE < nt) {
            if (!mbar_wait_timed(&ebar[st], par, WAIT_NS)) {
                set_status(a.status, NB6_ERR_WAIT_TIMEOUT);
                for (int u = t + 1; u < issued; ++u)
                    mbar_wait_timed(&bar[u % NSTAGE], (uint32_t)((u / NSTAGE) & 1), WAIT_NS / 8);
                return;
            }
            issue_tile_soa<F64DX>(a, sj[st], &bar[st], t_begin + (t + NSTAGE) * t_step);
            issued = t + NSTAGE + 1;
        }
        // fold: positive partial = rare-path sums - packed (negated) lane
        // sums; a far tile's lane sums are unscaled and positive (x8, x2)
        const float fa = far ? 8.0f : -1.0f, fp = far ? 2.0f : -1.0f;
#pragma unroll
        for (int k = 0; k < NI; ++k) {
            const float p[7] = {fx[k].ax + fa * (s[k].ax.x + s[k].ax.y), fx[k].ay + fa * (s[k].ay.x + s[k].ay.y),
                                fx[k].az + fa * (s[k].az.x + s[k].az.y), fx[k].jx + fa * (s[k].jx.x + s[k].jx.y),
                                fx[k].jy + fa * (s[k].jy.x + s[k].jy.y), fx[k].jz + fa * (s[k].jz.x + s[k].jz.y),
                                fx[k].po + fp * (s[k].po.x + s[k].po.y)};
#pragma unroll
            for (int c = 0; c < 7; ++c) {
                float2 d = dsum[k][c][tid];
                ds_fold(d.x, d.y, p[c]);
                dsum[k][c][tid] = d;
            }
            zero2(s[k]);
            zero(fx[k]);
        }
    }

#pragma unroll
    for (int k = 0; k < NI; ++k) {
        const int i = ii[k];
        if (i < a.ni) {
            float2 d[7];
#pragma unroll
            for (int c = 0; c < 7; ++c) d[c] = dsum[k][c][tid];
            float4 *p = a.part + ((size_t)slice * a.ni_pad + i) * 4;
            p[0] = make_float4(d[0].x, d[0].y, d[1].x, d[1].y);
            p[1] = make_float4(d[2].x, d[2].y, d[3].x, d[3].y);
            p[2] = make_float4(d[4].x, d[4].y, d[5].x, d[5].y);
            p[3] = make_float4(d[6].x, d[6].y, 0.f, 0.f);
        }
    }
}

// j-parallel variant for few active particles (blocksteps with small
// N_active): a CTA takes IB i-particles (hi/lo split into shared memory) and
// a j-slice; each thread streams its own j's straight from global memory
// (coalesced float4 loads) and runs them against all IB i's, so every SM is
// busy even for ni = 1.  Same pair math, candidate test and exact FP64 rare
// path as regf_kernel; the per-thread FP32 partials are reduced over the CTA
// in FP64 and written as (hi, lo) slice partials for regf_finalize.
constexpr int JPAR_NT = 256;

// The i-particles of a j-parallel CTA in shared memory: sip[k] = (xH, yH, zH,
// 1.01 h2), (xL, yL, zL, dtr), (vx, vy, vz, 0) of particle k, and, for the
// packed loop, the same data as IP2 pairs (particles 2p and 2p+1 in the two
// lanes, negated as pair_x2 takes them).  Padding particles (k >= nvalid)
// have h2 = 0: never a candidate, results unused.
template <int IB> struct JparI {
    float4 sip[IB][3];
    IP2 sip2[IB > 1 ? IB / 2 : 1];
    // packed loop: each warp's queue of neighbour candidates (j << 3 | k)
    // awaiting the exact FP64 decision; fewer than 32 wait between j
    // iterations, and one iteration adds at most 32 IB
    unsigned queue[IB > 1 ? JPAR_NT / 32 : 1][IB > 1 ? 32 + 32 * IB : 1];
};

template <int IB, bool X2>
NB6_DEV void jpar_stage_i(const RegArgs &a, JparI<IB> &S, int i0, int nvalid) {
    const int k = threadIdx.x;
    if (k >= IB) return;
    float4 p = make_float4(0.f, 0.f, 0.f, 0.f), q = p, r = p;
    if (k < nvalid) {
        const int i = i0 + k;
        split_hl(a.ix[3 * i], p.x, q.x);
        split_hl(a.ix[3 * i + 1], p.y, q.y);
        split_hl(a.ix[3 * i + 2], p.z, q.z);
        p.w = (float)a.ih2[i] * CAND_SLACK;
        q.w = (float)a.idtr[i];
        r = make_float4((float)a.iv[3 * i], (float)a.iv[3 * i + 1], (float)a.iv[3 * i + 2], 0.f);
    }
    S.sip[k][0] = p;
    S.sip[k][1] = q;
    S.sip[k][2] = r;
    if constexpr (X2 && IB > 1) {
        IP2 &d = S.sip2[k >> 1];
        float *l = reinterpret_cast<float *>(&d) + (k & 1);  // lane k & 1 of every float2
        const float v[11] = {-p.x, -p.y, -p.z, -q.x, -q.y, -q.z, -r.x, -r.y, -r.z, p.w, q.w};
#pragma unroll
        for (int c = 0; c < 11; ++c) l[2 * c] = v[c];
    }
}

// The j-parallel inner loop: this thread's j's of [j_begin, j_end) against
// the IB staged i-particles, results into s[k] (scaled as reg_pair keeps
// them).  X2 (IB >= 2): two i-particles per f32x2 instruction (pair_x2 on
// IP2 pairs, the j operands duplicated into both lanes; pair_x2 is reg_pair
// operation for operation).  Neighbour candidates of the packed loop wait
// in a per-warp queue and are decided 32 at a time, one per lane: in a small
// cluster a sizeable share of all pairs are neighbours, and deciding them
// where they arise would hold the whole warp for every lane that has one.
// Any lane may decide any queued pair: its contribution joins that lane's
// partial sum of particle k, which the CTA reduction adds up with the rest.
// The order is fixed by the data, so results are deterministic; they differ
// from the scalar loop's (X2 false) in the order of those sums.
template <int IB, bool MFLAG, bool X2>
NB6_DEV void jpar_loop(const RegArgs &a, const JparI<IB> &S, int j_begin, int j_end, int i0, int nvalid,
                       int jbase, Sums *s) {
    if constexpr (X2 && IB > 1) {
        constexpr int NP = IB / 2;
        S2 acc[NP];
#pragma unroll
        for (int p = 0; p < NP; ++p) zero2(acc[p]);
        const int lane = threadIdx.x & 31;
        unsigned *qw = const_cast<unsigned *>(S.queue[threadIdx.x >> 5]);
        int qn = 0;  // queued candidates of this warp (warp-uniform)
        // decide queued entry e on this lane: its exact contribution (or its
        // neighbour record) into lane k & 1 of acc[k / 2]
        auto decide = [&](unsigned e) {
            const int k = (int)(e & 7u), jj = (int)(e >> 3);
            Sums t;
            zero(t);
            reg_exact<MFLAG>(a, i0 + k, jj, t, jbase);
#pragma unroll
            for (int kk = 0; kk < IB; ++kk) {
                if (kk != k) continue;
                S2 &q = acc[kk >> 1];
                if (kk & 1) {
                    q.ax.y -= t.ax; q.ay.y -= t.ay; q.az.y -= t.az;
                    q.jx.y -= t.jx; q.jy.y -= t.jy; q.jz.y -= t.jz; q.po.y -= t.po;
                } else {
                    q.ax.x -= t.ax; q.ay.x -= t.ay; q.az.x -= t.az;
                    q.jx.x -= t.jx; q.jy.x -= t.jy; q.jz.x -= t.jz; q.po.x -= t.po;
                }
            }
        };
        const int j_stop = j_begin + (int)((j_end - j_begin + JPAR_NT - 1) / JPAR_NT) * JPAR_NT;
        for (int j = j_begin + lane + (int)(threadIdx.x & ~31u); j < j_stop; j += JPAR_NT) {
            // every lane of the warp takes every iteration (the queue is the
            // warp's); lanes past j_end compute nothing
            unsigned cm = 0u;
            if (j < j_end) {
                const float4 pa = __ldg(a.posH + j);
                const float4 pb = __ldg(a.posL + j);
                const float4 pc = __ldg(a.vel + j);
#pragma unroll
                for (int p = 0; p < NP; ++p) {
                    const IP2 ip = S.sip2[p];
                    cm |= pair_x2<MFLAG>(ip, dup2(pa.x), dup2(pa.y), dup2(pa.z), dup2(pa.w), dup2(pb.x),
                                         dup2(pb.y), dup2(pb.z), dup2(pc.x), dup2(pc.y), dup2(pc.z), acc[p])
                          << (2 * p);
                }
            }
            if (__any_sync(0xffffffffu, cm != 0u)) {
                // append this lane's candidates after those of the lanes below
                const int c = __popc(cm);
                int pre = c;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int t = __shfl_up_sync(0xffffffffu, pre, o);
                    if (lane >= o) pre += t;
                }
                const int tot = __shfl_sync(0xffffffffu, pre, 31);
                int w = qn + pre - c;
                for (unsigned m = cm; m; m &= m - 1) qw[w++] = ((unsigned)j << 3) | (unsigned)(__ffs(m) - 1);
                __syncwarp();
                qn += tot;
                while (qn >= 32) {  // warp-uniform
                    const unsigned e = qw[qn - 32 + lane];
                    __syncwarp();
                    qn -= 32;
                    decide(e);
                }
            }
        }
        if (qn > 0) {
            const unsigned e = lane < qn ? qw[lane] : 0u;
            __syncwarp();
            if (lane < qn) decide(e);
        }
#pragma unroll
        for (int k = 0; k < IB; ++k) {
            const S2 &q = acc[k >> 1];
            const bool hi = k & 1;
            s[k].ax = -(hi ? q.ax.y : q.ax.x);
            s[k].ay = -(hi ? q.ay.y : q.ay.x);
            s[k].az = -(hi ? q.az.y : q.az.x);
            s[k].jx = -(hi ? q.jx.y : q.jx.x);
            s[k].jy = -(hi ? q.jy.y : q.jy.x);
            s[k].jz = -(hi ? q.jz.y : q.jz.x);
            s[k].po = -(hi ? q.po.y : q.po.x);
        }
    } else {
#pragma unroll
        for (int k = 0; k < IB; ++k) zero(s[k]);
        for (int j = j_begin + (int)threadIdx.x; j < j_end; j += JPAR_NT) {
            const float4 pa = __ldg(a.posH + j);
            const float4 pb = __ldg(a.posL + j);
            const float4 pc = __ldg(a.vel + j);
            bool any = false;
#pragma unroll
            for (int k = 0; k < IB; ++k) {
                const float4 p = S.sip[k][0], q = S.sip[k][1], r = S.sip[k][2];
                IPart ip;
                ip.xh = p.x; ip.yh = p.y; ip.zh = p.z; ip.h2c = p.w;
                ip.xl = q.x; ip.yl = q.y; ip.zl = q.z; ip.dt = q.w;
                ip.vx = r.x; ip.vy = r.y; ip.vz = r.z;
                any |= reg_pair<MFLAG>(ip, pa, pb, pc, s[k]);
            }
            if (any) {
                for (int k = 0; k < IB && k < nvalid; ++k) {
                    const float4 p = S.sip[k][0], q = S.sip[k][1], r = S.sip[k][2];
                    IPart ip;
                    ip.xh = p.x; ip.yh = p.y; ip.zh = p.z; ip.h2c = p.w;
                    ip.xl = q.x; ip.yl = q.y; ip.zl = q.z; ip.dt = q.w;
                    ip.vx = r.x; ip.vy = r.y; ip.vz = r.z;
                    if (reg_geom<MFLAG>(ip, pa, pb, pc).cand) reg_exact<MFLAG>(a, i0 + k, j, s[k], jbase);
                }
            }
        }
    }
}

template <int IB, bool MFLAG, bool X2 = false>
__global__ void __launch_bounds__(JPAR_NT) regf_jpar_kernel(const RegArgs a) {
    __shared__ __align__(16) JparI<IB> S;
    __shared__ double red[JPAR_NT / 32][IB][7];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int i0 = blockIdx.x * IB;
    jpar_stage_i<IB, X2>(a, S, i0, a.ni - i0);
    __syncthreads();
    const int j_begin = (int)(((long long)blockIdx.y * a.nj) / a.nslices);
    const int j_end = (int)(((long long)(blockIdx.y + 1) * a.nj) / a.nslices);
    Sums s[IB];
    jpar_loop<IB, MFLAG, X2>(a, S, j_begin, j_end, i0, a.ni - i0, 0, s);
    // CTA reduction in FP64: warp shuffles, then across warps in shared memory
#pragma unroll
    for (int k = 0; k < IB; ++k) {
        double v[7] = {s[k].ax, s[k].ay, s[k].az, s[k].jx, s[k].jy, s[k].jz, s[k].po};
#pragma unroll
        for (int c = 0; c < 7; ++c) {
            const double w = warp_sum_d(v[c]);
            if (lane == 0) red[warp][k][c] = w;
        }
    }
    __syncthreads();
    if (tid < IB * 7) {
        const int k = tid / 7, c = tid % 7;
        double w = 0.0;
#pragma unroll
        for (int q = 0; q < JPAR_NT / 32; ++q) w += red[q][k][c];
        red[0][k][c] = w;
    }
    __syncthreads();
    if (tid < IB) {
        const int i = i0 + tid;
        if (i < a.ni) {
            float hv[7], lv[7];
#pragma unroll
            for (int c = 0; c < 7; ++c) {
                const double w = red[0][tid][c];
                hv[c] = (float)w;
                lv[c] = (float)(w - (double)hv[c]);
            }
            float4 *p = a.part + ((size_t)blockIdx.y * a.ni_pad + i) * 4;
            p[0] = make_float4(hv[0], lv[0], hv[1], lv[1]);
            p[1] = make_float4(hv[2], lv[2], hv[3], lv[3]);
            p[2] = make_float4(hv[4], lv[4], hv[5], lv[5]);
            p[3] = make_float4(hv[6], lv[6], 0.f, 0.f);
        }
    }
}

// Accumulate one (hi, lo) slice partial into FP64 sums.
NB6_DEV void add_partial(const float4 *p, double *v) {
    const float4 q0 = p[0], q1 = p[1], q2 = p[2], q3 = p[3];
    v[0] += (double)q0.x + (double)q0.y;
    v[1] += (double)q0.z + (double)q0.w;
    v[2] += (double)q1.x + (double)q1.y;
    v[3] += (double)q1.z + (double)q1.w;
    v[4] += (double)q2.x + (double)q2.y;
    v[5] += (double)q2.z + (double)q2.w;
    v[6] += (double)q3.x + (double)q3.y;
}

// Second half of a finalize row (one warp, one i): reduce the lanes' FP64
// sums, write outf, reset the neighbour counter, and write the list row
// sorted ascending (warp bitonic sort in shared memory) or -nnb on overflow.
NB6_DEV void finalize_row(int i, int lane, double *v, int *__restrict__ nbcnt,
                          const int *__restrict__ nbbuf, int lcap, int cap, int W, int *sb,
                          double *__restrict__ outf, int *__restrict__ outl, const MlpArgs &mlp,
                          const __nv_bfloat16 *sw) {
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
    __syncwarp();
    if (lane == 0) nbcnt[i] = 0;
    if (mlp.on) {
        // learned radius proposal from this call's own results (out slot 7)
        float fe[MLP_IN];
        const double ax = v[0] * 0.125, ay = v[1] * 0.125, az = v[2] * 0.125;
        mlp_features((double)n, mlp.h2[i], ax * ax + ay * ay + az * az, mlp.dtr[i], fe);
        MlpAct act;
        const float out = mlp_forward_warp(sw, mlp.norm, fe, lane, act);
        if (lane == 0) outf[(size_t)i * 8 + 7] = (double)(out * mlp.norm[2 * MLP_IN + 1] + mlp.norm[2 * MLP_IN]);
    }
    int *row = outl + (size_t)i * W;
    if (n > cap) {
        if (lane == 0) row[0] = -n;
        return;
    }
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

// One warp per i: FP64 sum over slices in a fixed order, then the neighbour
// ids sorted ascending.  outf row = (ax, ay, az, jx, jy, jz, pot, 0).  The
// neighbour counter of i is reset to zero once read, so the next call starts
// from clean counters without a memset.
__global__ void __launch_bounds__(FIN_WARPS * 32)
    regf_finalize(const float4 *__restrict__ part, int nslices, int ni, int ni_pad,
                  int *__restrict__ nbcnt, const int *__restrict__ nbbuf, int lcap,
                  int cap, int W, int pmax, double *__restrict__ outf,
                  int *__restrict__ outl, const MlpArgs mlp) {
    extern __shared__ __align__(16) int sbuf[];
    __nv_bfloat16 *sw = reinterpret_cast<__nv_bfloat16 *>(sbuf + FIN_WARPS * pmax);
    if (mlp.on) {
        mlp_load(sw, mlp.w);
        __syncthreads();
    }
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * FIN_WARPS + warp;
    if (i >= ni) return;
    double v[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int sl = lane; sl < nslices; sl += 32) add_partial(part + ((size_t)sl * ni_pad + i) * 4, v);
    finalize_row(i, lane, v, nbcnt, nbbuf, lcap, cap, W, sbuf + warp * pmax, outf, outl, mlp, sw);
}

// ----------------------------------------------------------------------------
// Segmented regular force (ensembles of independent clusters in one call).
//
// The j set holds several clusters back to back; segment c is the j range
// [seg_j0[c], seg_j0[c+1]).  Every active i belongs to one segment and sees
// only that segment's j: the same force, jerk, potential and neighbour rule
// as gpunb_regf_ with that cluster alone sent, list ids relative to the
// segment's first j.  The work is a list of items (segment, group of up to IB
// consecutive i of that segment, j chunk), built on the host with the costly
// items first; one persistent launch of SMs x occupancy CTAs walks the list
// (grid-stride), each item running the j-parallel inner loop of
// regf_jpar_kernel (threads over j, the IB i in shared memory).  Item q of an
// i writes its (hi, lo) partial to slot pinfo[i].x + q; regf_finalize_seg
// sums the pinfo[i].y slots of each i in order.
// ----------------------------------------------------------------------------
struct SegItem {
    int i0, ni, j0, j1, jbase, q, pad0, pad1;
};

template <int IB, bool MFLAG, bool X2 = false>
__global__ void __launch_bounds__(JPAR_NT)
    regf_seg_kernel(const RegArgs a, const SegItem *__restrict__ items, const int *__restrict__ nitems_p,
                    const int2 *__restrict__ pinfo) {
    __shared__ __align__(16) JparI<IB> S;
    __shared__ double red[JPAR_NT / 32][IB][7];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nitems = *nitems_p;
    for (int w = blockIdx.x; w < nitems; w += gridDim.x) {
        const SegItem it = items[w];
        __syncthreads();  // the previous item is done with the staged i and red
        jpar_stage_i<IB, X2>(a, S, it.i0, it.ni);
        __syncthreads();
        Sums s[IB];
        jpar_loop<IB, MFLAG, X2>(a, S, it.j0, it.j1, it.i0, it.ni, it.jbase, s);
#pragma unroll
        for (int k = 0; k < IB; ++k) {
            double v[7] = {s[k].ax, s[k].ay, s[k].az, s[k].jx, s[k].jy, s[k].jz, s[k].po};
#pragma unroll
            for (int c = 0; c < 7; ++c) {
                const double wsum = warp_sum_d(v[c]);
                if (lane == 0) red[warp][k][c] = wsum;
            }
        }
        __syncthreads();
        if (tid < IB * 7) {
            const int k = tid / 7, c = tid % 7;
            double wsum = 0.0;
#pragma unroll
            for (int q = 0; q < JPAR_NT / 32; ++q) wsum += red[q][k][c];
            red[0][k][c] = wsum;
        }
        __syncthreads();
        if (tid < it.ni && tid < IB) {
            const int i = it.i0 + tid;
            float hv[7], lv[7];
#pragma unroll
            for (int c = 0; c < 7; ++c) {
                const double wsum = red[0][tid][c];
                hv[c] = (float)wsum;
                lv[c] = (float)(wsum - (double)hv[c]);
            }
            float4 *p = a.part + ((size_t)pinfo[i].x + it.q) * 4;
            p[0] = make_float4(hv[0], lv[0], hv[1], lv[1]);
            p[1] = make_float4(hv[2], lv[2], hv[3], lv[3]);
            p[2] = make_float4(hv[4], lv[4], hv[5], lv[5]);
            p[3] = make_float4(hv[6], lv[6], 0.f, 0.f);
        }
    }
}

__global__ void __launch_bounds__(FIN_WARPS * 32)
    regf_finalize_seg(const float4 *__restrict__ part, const int2 *__restrict__ pinfo, int ni,
                      int *__restrict__ nbcnt, const int *__restrict__ nbbuf, int lcap, int cap, int W,
                      int pmax, double *__restrict__ outf, int *__restrict__ outl, const MlpArgs mlp) {
    extern __shared__ __align__(16) int sbuf[];
    __nv_bfloat16 *sw = reinterpret_cast<__nv_bfloat16 *>(sbuf + FIN_WARPS * pmax);
    if (mlp.on) {
        mlp_load(sw, mlp.w);
        __syncthreads();
    }
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * FIN_WARPS + warp;
    if (i >= ni) return;
    const int2 pi = pinfo[i];
    double v[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int q = lane; q < pi.y; q += 32) add_partial(part + ((size_t)pi.x + q) * 4, v);
    finalize_row(i, lane, v, nbcnt, nbbuf, lcap, cap, W, sbuf + warp * pmax, outf, outl, mlp, sw);
}

// FP64 (m, x, v) -> SoA float4 tiles; padding slots are massless and far.
__global__ void regf_pack_j(int nj, JSetOut o, const double *__restrict__ m,
                            const double *__restrict__ x, const double *__restrict__ v, int *status) {
    for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < o.npad;
         j += (size_t)gridDim.x * blockDim.x) {
        if (j < (size_t)nj) {
            const double x0 = x[3 * j], x1 = x[3 * j + 1], x2 = x[3 * j + 2];
            const double v0 = v[3 * j], v1 = v[3 * j + 1], v2 = v[3 * j + 2];
            const double mj = m[j];
            if (x0 != x0 || x1 != x1 || x2 != x2 || v0 != v0 || v1 != v1 || v2 != v2 ||
                mj != mj)
                set_status(status, NB6_ERR_NAN_INPUT);
            write_j(o, j, true, x0, x1, x2, mj, v0, v1, v2);
        } else {
            write_j(o, j, false, 0, 0, 0, 0, 0, 0, 0);
        }
    }
}

// ----------------------------------------------------------------------------
// host state
// ----------------------------------------------------------------------------

// Measured autotuner keyed on (log2 N_active, log2 N_j, m_flag): the first
// call in a bucket times every admissible variant on the caller's own data
// (kernel-only CUDA events) and caches the fastest.  NB6_AUTOTUNE=0 turns it
// off (default_variant is used); nb6_regf_tune_ forces a variant.
struct TuneKey {
    int li, lj, mf;
    bool operator<(const TuneKey &o) const {
        return li != o.li ? li < o.li : lj != o.lj ? lj < o.lj : mf < o.mf;
    }
};

struct RegState {
    bool open = false;
    int nbodymax = 0;
    int nj = 0;
    int ntile = 0;
    DevBuf<float4> posH, posL, vel;
    DevBuf<float> comp;              // NB6_NCOMP x npad, component-major
    DevBuf<double> compd;            // 3 x npad FP64 positions, component-major
    size_t npad = 0;
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
    int forced_ni_per_thread = 0;   // forced variant (see Plan); 0 = automatic
    int forced_slices = 0;
    int last_geometry[3] = {0, 0, 0};  // variant, i-grid, j-slices of the last launch
    int autotune = -1;                 // -1 = read NB6_AUTOTUNE on first use
    std::map<TuneKey, int> tuned;      // bucket -> best variant
    cudaEvent_t tev0 = nullptr, tev1 = nullptr;
    // CUDA graphs of one call: [0] device-resident i data, [1] host i data
    // with the copies in the graph.  Built once, then re-parameterised per
    // call (launch geometry, kernel, pointers, copy sizes).
    struct Graph {
        cudaGraph_t g = nullptr;
        cudaGraphExec_t x = nullptr;
        cudaGraphNode_t h2d = nullptr, kmain = nullptr, kfin = nullptr, d2hf = nullptr, d2hl = nullptr;
    } graph[2];
    int use_graphs = -1;               // -1 = read NB6_GRAPHS on first use
    long long graph_builds = 0, graph_launches = 0;
    bool nbcnt_dirty = true;           // neighbour counters not known to be zero
    // segmented calls: work list and per-i partial slots, staged as ints
    HostBuf<int> hseg;
    DevBuf<int> dseg;
    // spatially ordered copy of the j set (see jset_keys)
    int use_jsort = -1;                // -1 = read NB6_JSORT on first use
    long long jver = 0, sorted_ver = -1;
    DevBuf<float4> posH_s, posL_s, vel_s, tbox;
    DevBuf<float> comp_s, comprel;  // ordered layout; tile-relative positions (3 x npad)
    DevBuf<double> compd_s;
    DevBuf<int> perm, vals_in, iperm;
    DevBuf<unsigned> keys_in, keys_out, ext;
    DevBuf<unsigned char> sort_tmp;
    // NB6_SELFCHECK=1: host copy of the last send, to re-derive sample rows
    int selfcheck = -1;
    std::vector<double> chk_m, chk_x, chk_v;
    long long chk_rows = 0, chk_bad = 0;
};
RegState R;

// A launch plan.  variant > 0: regf_kernel with NI = variant i per thread
// (i-parallel tiles); variant < 0: regf_jpar_kernel with IB = -variant
// i-particles per CTA (j-parallel).
struct Plan {
    int variant = 1;
    int igrid = 1;   // i-tiles or i-groups
    int nslices = 1;
};

template <class K> int occ_of(K kern, int threads) {
    int occ = 0;
    NB6_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, threads, 0));
    return occ < 1 ? 1 : occ;
}

// Variants: 1, 2, 4 = regf_kernel with that many i per thread; 11, 12 =
// regf_x2_kernel (packed f32x2) with 1 or 2 i per thread; -1, -2, -4, -8 =
// regf_jpar_kernel with that many i per CTA.
bool valid_variant(int v) {
    return v == 1 || v == 2 || v == 4 || v == 11 || v == 12 || v == 13 || v == -1 || v == -2 || v == -4 ||
           v == -8;
}

int i_per_thread(int v) { return v == 13 ? 1 : v > 10 ? v - 10 : v; }

// The j-parallel and segmented kernels with two or more i per CTA run the
// packed (f32x2) inner loop; NB6_JPAR_X2=0 in the environment selects the
// scalar loop (the same bits, for comparison).
bool jpar_x2() {
    static const bool on = [] {
        const char *e = getenv("NB6_JPAR_X2");
        return !(e && atoi(e) == 0);
    }();
    return on;
}

template <bool MF> int occupancy_t(int variant) {
    switch (variant) {
        case 1: return occ_of(regf_kernel<1, MF>, NT);
        case 2: return occ_of(regf_kernel<2, MF>, NT);
        case 4: return occ_of(regf_kernel<4, MF>, NT);
        case 11: return occ_of(regf_x2_kernel<1, MF>, NT);
        case 12: return occ_of(regf_x2_kernel<2, MF>, NT);
        case 13: return occ_of(regf_x2_kernel<1, MF, true>, NT);
        case -1: return occ_of(regf_jpar_kernel<1, MF>, JPAR_NT);
        case -2: return jpar_x2() ? occ_of(regf_jpar_kernel<2, MF, true>, JPAR_NT) : occ_of(regf_jpar_kernel<2, MF>, JPAR_NT);
        case -4: return jpar_x2() ? occ_of(regf_jpar_kernel<4, MF, true>, JPAR_NT) : occ_of(regf_jpar_kernel<4, MF>, JPAR_NT);
        default: return jpar_x2() ? occ_of(regf_jpar_kernel<8, MF, true>, JPAR_NT) : occ_of(regf_jpar_kernel<8, MF>, JPAR_NT);
    }
}

int occupancy(int variant, bool mf) {
    static std::map<int, int> cache;
    const int key = variant * 2 + (mf ? 1 : 0);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    const int c = mf ? occupancy_t<true>(variant) : occupancy_t<false>(variant);
    cache[key] = c;
    return c;
}

// Geometry of one variant: enough CTAs for one full wave.
Plan make_plan(int variant, int ni, int nj, int ntile, bool mf, int forced_slices) {
    Plan p;
    p.variant = variant;
    const int target = nb6_num_sms() * occupancy(variant, mf);
    if (variant > 0) {
        const int tile = NT * i_per_thread(variant);
        p.igrid = (ni + tile - 1) / tile;
        p.nslices = std::max(1, target / p.igrid);
        p.nslices = std::min(p.nslices, ntile);
    } else {
        const int ib = -variant;
        p.igrid = (ni + ib - 1) / ib;
        // at least 4 j per thread so the per-CTA set-up and reduction amortise
        const int maxsl = std::max(1, nj / (JPAR_NT * 4));
        p.nslices = std::max(1, std::min(target / p.igrid, maxsl));
    }
    if (forced_slices > 0) p.nslices = variant > 0 ? std::min(forced_slices, ntile) : forced_slices;
    p.nslices = std::max(p.nslices, 1);
    return p;
}

// Default plan without measurement: the packed i-parallel kernel with one i
// per thread once a 128-thread tile is full, otherwise the j-parallel kernel
// with the smallest CTA i-group that covers ni (at most 8).
int default_variant(int ni) {
    if (ni >= NT) return 11;
    int ib = 1;
    while (ib < ni && ib < 8) ib <<= 1;
    return -ib;
}

template <bool MF> void launch_plan(const Plan &p, const RegArgs &a, cudaStream_t st) {
    dim3 grid(p.igrid, p.nslices);
    switch (p.variant) {
        case 1: regf_kernel<1, MF><<<grid, NT, 0, st>>>(a); break;
        case 2: regf_kernel<2, MF><<<grid, NT, 0, st>>>(a); break;
        case 4: regf_kernel<4, MF><<<grid, NT, 0, st>>>(a); break;
        case 11: regf_x2_kernel<1, MF><<<grid, NT, 0, st>>>(a); break;
        case 12: regf_x2_kernel<2, MF><<<grid, NT, 0, st>>>(a); break;
        case 13: regf_x2_kernel<1, MF, true><<<grid, NT, 0, st>>>(a); break;
        case -1: regf_jpar_kernel<1, MF><<<grid, JPAR_NT, 0, st>>>(a); break;
        case -2:
            if (jpar_x2()) regf_jpar_kernel<2, MF, true><<<grid, JPAR_NT, 0, st>>>(a);
            else regf_jpar_kernel<2, MF><<<grid, JPAR_NT, 0, st>>>(a);
            break;
        case -4:
            if (jpar_x2()) regf_jpar_kernel<4, MF, true><<<grid, JPAR_NT, 0, st>>>(a);
            else regf_jpar_kernel<4, MF><<<grid, JPAR_NT, 0, st>>>(a);
            break;
        default:
            if (jpar_x2()) regf_jpar_kernel<8, MF, true><<<grid, JPAR_NT, 0, st>>>(a);
            else regf_jpar_kernel<8, MF><<<grid, JPAR_NT, 0, st>>>(a);
            break;
    }
}

// The kernel launch_plan would launch, as a function handle for graph nodes.
template <bool MF> const void *kernel_of(int variant) {
    switch (variant) {
        case 1: return (const void *)regf_kernel<1, MF>;
        case 2: return (const void *)regf_kernel<2, MF>;
        case 4: return (const void *)regf_kernel<4, MF>;
        case 11: return (const void *)regf_x2_kernel<1, MF>;
        case 12: return (const void *)regf_x2_kernel<2, MF>;
        case 13: return (const void *)regf_x2_kernel<1, MF, true>;
        case -1: return (const void *)regf_jpar_kernel<1, MF>;
        case -2: return jpar_x2() ? (const void *)regf_jpar_kernel<2, MF, true> : (const void *)regf_jpar_kernel<2, MF>;
        case -4: return jpar_x2() ? (const void *)regf_jpar_kernel<4, MF, true> : (const void *)regf_jpar_kernel<4, MF>;
        default: return jpar_x2() ? (const void *)regf_jpar_kernel<8, MF, true> : (const void *)regf_jpar_kernel<8, MF>;
    }
}

int ilog2(int v) {
    int r = 0;
    while ((1 << (r + 1)) <= v) ++r;
    return r;
}

bool any_nan(const double *p, size_t n) {
    for (size_t k = 0; k < n; ++k)
        if (p[k] != p[k]) return true;
    return false;
}

// ----------------------------------------------------------------------------
// Spatial order of the j set.  After every send the bodies are put in Morton
// (Z-curve) order of their positions, so that the 128 bodies of a tile are
// close together, and each tile gets a bounding box.  The packed kernel then
// skips the neighbour-candidate arithmetic for every (warp, tile) whose box is
// provably out of reach of all the warp's i-particles.  Slot k of the ordered
// set holds the caller's body perm[k]; the exact FP64 path maps slots back, so
// neighbour ids are the caller's.
// ----------------------------------------------------------------------------

// ext[0..2] = min x, y, z and ext[3..5] = max (order-preserving uints).
__global__ void jset_extent(int nj, const double *__restrict__ jx, unsigned *__restrict__ ext) {
    unsigned mn[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, mx[3] = {0u, 0u, 0u};
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nj; j += gridDim.x * blockDim.x)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const unsigned o = f2ord((float)jx[3 * (size_t)j + k]);
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


// 30-bit Morton key of each body on a 1024^3 grid over the extent.
__global__ void jset_keys(int nj, const double *__restrict__ jx, const unsigned *__restrict__ ext,
                          unsigned *__restrict__ keys, int *__restrict__ vals) {
    float lo[3], sc[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        lo[k] = ord2f(ext[k]);
        const float w = ord2f(ext[3 + k]) - lo[k];
        sc[k] = w > 0.f ? 1023.99f / w : 0.f;
    }
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nj; j += gridDim.x * blockDim.x) {
        unsigned key = 0;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float q = ((float)jx[3 * (size_t)j + k] - lo[k]) * sc[k];
            const unsigned c = q <= 0.f ? 0u : (q >= 1023.f ? 1023u : (unsigned)q);
            key |= spread10(c) << k;
        }
        keys[j] = key;
        vals[j] = j;
    }
}

// Ordered copies of the float layouts (slot k <- body perm[k]; padding slots
// k >= nj are copied in place).
__global__ void jset_permute(int nj, JSetOut src, JSetOut dst, const int *__restrict__ perm) {
    const size_t np = src.npad;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < np; k += (size_t)gridDim.x * blockDim.x) {
        const size_t o = k < (size_t)nj ? (size_t)perm[k] : k;
        dst.posH[k] = src.posH[o];
        dst.posL[k] = src.posL[o];
        dst.vel[k] = src.vel[o];
#pragma unroll
        for (int c = 0; c < NB6_NCOMP; ++c) dst.comp[c * np + k] = src.comp[c * np + o];
#pragma unroll
        for (int c = 0; c < 3; ++c) dst.compd[c * np + k] = src.compd[c * np + o];
    }
}

// One warp per tile: bounding box of the hi positions of its real bodies
// (centre rounded to nearest, half extent, speeds and masses rounded up).
__global__ void jset_tile_boxes(int nj, int ntile, const float4 *__restrict__ posH, const float4 *__restrict__ vel,
                                float4 *__restrict__ tbox) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= ntile) return;
    double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300}, vm = 0.0, mm = 0.0;
    for (int q = lane; q < JT; q += 32) {
        const int k = warp * JT + q;
        if (k >= nj) break;
        const float4 p = posH[k], v = vel[k];
        const double c[3] = {p.x, p.y, p.z};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            mn[d] = fmin(mn[d], c[d]);
            mx[d] = fmax(mx[d], c[d]);
        }
        vm = fmax(vm, sqrt((double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z));
        mm = fmax(mm, (double)p.w);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            mn[d] = fmin(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
            mx[d] = fmax(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o));
        }
        vm = fmax(vm, __shfl_xor_sync(0xffffffffu, vm, o));
        mm = fmax(mm, __shfl_xor_sync(0xffffffffu, mm, o));
    }
    if (lane == 0) {
        tbox[2 * warp] = make_float4(__double2float_rn(0.5 * (mn[0] + mx[0])), __double2float_rn(0.5 * (mn[1] + mx[1])),
                                     __double2float_rn(0.5 * (mn[2] + mx[2])), __double2float_ru(vm));
        tbox[2 * warp + 1] = make_float4(__double2float_ru(0.5 * (mx[0] - mn[0])), __double2float_ru(0.5 * (mx[1] - mn[1])),
                                         __double2float_ru(0.5 * (mx[2] - mn[2])), __double2float_ru(mm));
    }
}

// Tile-relative positions of the ordered j set: xr = fl32(x - c) with c the
// box centre of the body's tile (an FP32 number, so x - c is formed exactly
// in FP64 up to one rounding).  Padding slots keep their far-away marker.
__global__ void jset_rel(int npad, int ntile, const double *__restrict__ compd, const float4 *__restrict__ tbox,
                         float *__restrict__ comprel) {
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < (size_t)npad;
         q += (size_t)gridDim.x * blockDim.x) {
        const int t = (int)(q / JT);
        const float4 c = t < ntile ? tbox[2 * t] : make_float4(0.f, 0.f, 0.f, 0.f);
        comprel[q] = __double2float_rn(compd[q] - (double)c.x);
        comprel[(size_t)npad + q] = __double2float_rn(compd[(size_t)npad + q] - (double)c.y);
        comprel[2 * (size_t)npad + q] = __double2float_rn(compd[2 * (size_t)npad + q] - (double)c.z);
    }
}

// Spatial order of the active set of one call (ni <= ISORT_MAX): Morton keys
// on the j set's grid, bitonic sort of (key, index) in one CTA.
constexpr int ISORT_MAX = 4096;
__global__ void __launch_bounds__(1024) iset_order(int ni, const double *__restrict__ ix,
                                                   const unsigned *__restrict__ ext, int *__restrict__ iperm) {
    __shared__ unsigned long long kv[ISORT_MAX];
    float lo[3], sc[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        lo[k] = ord2f(ext[k]);
        const float w = ord2f(ext[3 + k]) - lo[k];
        sc[k] = w > 0.f ? 1023.99f / w : 0.f;
    }
    int P = 1;
    while (P < ni) P <<= 1;
    for (int s = threadIdx.x; s < P; s += blockDim.x) {
        unsigned long long v = ~0ull;  // padding sorts last
        if (s < ni) {
            unsigned key = 0;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float q = ((float)ix[3 * (size_t)s + k] - lo[k]) * sc[k];
                const unsigned c = q <= 0.f ? 0u : (q >= 1023.f ? 1023u : (unsigned)q);
                key |= spread10(c) << k;
            }
            v = ((unsigned long long)key << 32) | (unsigned)s;
        }
        kv[s] = v;
    }
    __syncthreads();
    for (int kk = 2; kk <= P; kk <<= 1)
        for (int jj = kk >> 1; jj > 0; jj >>= 1) {
            for (int x = threadIdx.x; x < P; x += blockDim.x) {
                const int y = x ^ jj;
                if (y > x) {
                    const unsigned long long p0 = kv[x], p1 = kv[y];
                    if ((p0 > p1) == ((x & kk) == 0)) {
                        kv[x] = p1;
                        kv[y] = p0;
                    }
                }
            }
            __syncthreads();
        }
    for (int s = threadIdx.x; s < ni; s += blockDim.x) iperm[s] = (int)(kv[s] & 0xffffffffu);
}

}  // namespace

// Make n bodies the current j set: tile count, padded length and buffers for
// both float layouts plus the FP64 copies.
static JSetOut size_j_buffers(int n) {
    R.jver++;  // a producer is about to write a new j set
    R.nj = n;
    R.ntile = std::max(1, (n + JT - 1) / JT);
    R.npad = (size_t)R.ntile * JT;
    R.posH.reserve(R.npad);
    R.posL.reserve(R.npad);
    R.vel.reserve(R.npad);
    R.comp.reserve((size_t)NB6_NCOMP * R.npad);
    R.compd.reserve((size_t)3 * R.npad);
    R.jm.reserve(R.npad);
    R.jx.reserve(3 * R.npad);
    R.jv.reserve(3 * R.npad);
    JSetOut o;
    o.posH = R.posH.ptr;
    o.posL = R.posL.ptr;
    o.vel = R.vel.ptr;
    o.comp = R.comp.ptr;
    o.compd = R.compd.ptr;
    o.npad = R.npad;
    return o;
}

// Build (once per j set) the spatially ordered copy used by the tile and
// j-parallel kernels.  Stream-ordered after the producer's kernels.
static bool ensure_sorted(cudaStream_t st) {
    if (R.use_jsort < 0) {
        const char *e = getenv("NB6_JSORT");
        R.use_jsort = (e && atoi(e) == 0) ? 0 : 1;
    }
    // small sets: the j-parallel kernel serves them and tiles span the whole
    // system, so the order would only cost the sort (NB6_JSORT_MIN overrides)
    static const int jsort_min = [] {
        const char *e = getenv("NB6_JSORT_MIN");
        return e ? atoi(e) : 32768;
    }();
    if (!R.use_jsort || R.nj < 1 || R.nj < jsort_min) return false;
    if (R.sorted_ver == R.jver) return true;
    const int nj = R.nj;
    const size_t np = R.npad;
    R.posH_s.reserve(np);
    R.posL_s.reserve(np);
    R.vel_s.reserve(np);
    R.comp_s.reserve((size_t)NB6_NCOMP * np);
    R.compd_s.reserve((size_t)3 * np);
    R.perm.reserve(nj);
    R.vals_in.reserve(nj);
    R.keys_in.reserve(nj);
    R.keys_out.reserve(nj);
    R.ext.reserve(6);
    R.tbox.reserve((size_t)2 * R.ntile);
    const unsigned init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    NB6_CUDA_CHECK(cudaMemcpyAsync(R.ext.ptr, init, sizeof(init), cudaMemcpyHostToDevice, st));
    const int blocks = std::max(1, std::min((nj + 255) / 256, nb6_num_sms() * 8));
    jset_extent<<<blocks, 256, 0, st>>>(nj, R.jx.ptr, R.ext.ptr);
    jset_keys<<<blocks, 256, 0, st>>>(nj, R.jx.ptr, R.ext.ptr, R.keys_in.ptr, R.vals_in.ptr);
    NB6_CUDA_CHECK(cudaGetLastError());
    size_t tmp = 0;
    NB6_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, tmp, R.keys_in.ptr, R.keys_out.ptr, R.vals_in.ptr,
                                                   R.perm.ptr, nj, 0, 30, st));
    R.sort_tmp.reserve(tmp + 16);
    NB6_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(R.sort_tmp.ptr, tmp, R.keys_in.ptr, R.keys_out.ptr,
                                                   R.vals_in.ptr, R.perm.ptr, nj, 0, 30, st));
    JSetOut src{R.posH.ptr, R.posL.ptr, R.vel.ptr, R.comp.ptr, R.compd.ptr, np};
    JSetOut dst{R.posH_s.ptr, R.posL_s.ptr, R.vel_s.ptr, R.comp_s.ptr, R.compd_s.ptr, np};
    const int pblocks = (int)std::min<size_t>((np + 255) / 256, (size_t)nb6_num_sms() * 8);
    jset_permute<<<pblocks, 256, 0, st>>>(nj, src, dst, R.perm.ptr);
    jset_tile_boxes<<<(R.ntile * 32 + 255) / 256, 256, 0, st>>>(nj, R.ntile, R.posH_s.ptr, R.vel_s.ptr, R.tbox.ptr);
    R.comprel.reserve((size_t)3 * np);
    jset_rel<<<pblocks, 256, 0, st>>>((int)np, R.ntile, R.compd_s.ptr, R.tbox.ptr, R.comprel.ptr);
    NB6_CUDA_CHECK(cudaGetLastError());
    R.sorted_ver = R.jver;
    return true;
}

// ----------------------------------------------------------------------------
// One regular-force call on resident i data, in three steps:
//   regf_prepare  pick the launch plan (autotuner), size the buffers;
//   regf_eager    memset + force kernel + finalize (+ copies) as launches;
//   regf_submit   the same work as one CUDA graph launch.
// The graph of each call kind is built once and re-parameterised per call
// (cudaGraphExec*SetParams: kernel, grid, arguments, copy sizes), so calls
// of any ni replay it without a new capture.  The neighbour counters are
// zeroed by regf_finalize itself, which keeps memsets out of the graph.
// ----------------------------------------------------------------------------
struct RegLaunch {
    Plan plan;
    RegArgs a;
    int ni = 0, W = 1, cap = 0, pmax = 32, fblocks = 1;
    size_t smem = 0;
    bool mf = false;
    MlpArgs mlp{};
    // host staging (graph node of kind 1)
    const double *hin = nullptr;
    size_t in_bytes = 0;
    // where regf_finalize writes: the device buffers, or (host calls under
    // unified addressing) the pinned host staging itself, so only the used
    // part of each list row crosses the bus and no copy-back is needed
    double *outf = nullptr;
    int *outl = nullptr;
    bool direct = false;
};

// Arguments of regf_finalize, addressable for a kernel node.
struct FinArgs {
    const float4 *part;
    int nslices, ni, ni_pad;
    int *nbcnt;
    const int *nbbuf;
    int lcap, cap, W, pmax;
    double *outf;
    int *outl;
    MlpArgs mlp;
    void *p[13];
    explicit FinArgs(const RegLaunch &L)
        : part(L.a.part), nslices(L.plan.nslices), ni(L.ni), ni_pad(L.a.ni_pad), nbcnt(L.a.nbcnt),
          nbbuf(L.a.nbbuf), lcap(L.a.lcap), cap(L.cap), W(L.W), pmax(L.pmax), outf(L.outf),
          outl(L.outl), mlp(L.mlp) {
        void *q[13] = {&part, &nslices, &ni, &ni_pad, &nbcnt, &nbbuf, &lcap, &cap, &W, &pmax, &outf, &outl, &mlp};
        memcpy(p, q, sizeof(q));
    }
};

// The neighbour counters of ni rows.  A new buffer is cleared over its
// whole capacity: the kernels count into rows [0, ni) of every call and
// regf_finalize resets the rows it reads, so rows beyond the calls so far
// must start at zero too (a later, larger call reads them without a
// clear).  Returns whether the buffer was replaced.
static bool nbcnt_reserve(int ni, cudaStream_t st) {
    const int *before = R.nbcnt.ptr;
    const size_t cap_before = R.nbcnt.cap;
    R.nbcnt.reserve(ni);
    if (R.nbcnt.ptr == before && R.nbcnt.cap == cap_before) return false;
    NB6_CUDA_CHECK(cudaMemsetAsync(R.nbcnt.ptr, 0, sizeof(int) * R.nbcnt.cap, st));
    return true;
}

static void regf_prepare(int ni, const double *d_h2, const double *d_dtr, const double *d_x,
                         const double *d_v, int lmax, int nnbmax, int mflag, cudaStream_t st,
                         RegLaunch &L) {
    const int cap = std::max(0, std::min(nnbmax, lmax - 1));
    const int W = cap + 1;
    const int ni_pad = ni;
    const bool mf = mflag != 0;
    if (R.autotune < 0) {
        const char *e = getenv("NB6_AUTOTUNE");
        R.autotune = (e && atoi(e) == 0) ? 0 : 1;
    }
    int variant = default_variant(ni);
    // calls above TUNE_NI rows share one bucket, tuned on their first
    // TUNE_NI rows: the choice no longer changes with ni there, and trials on
    // every row of a very large call would cost seconds
    constexpr int TUNE_NI = 8192;
    static_assert(ISORT_MAX <= TUNE_NI, "an ordered call must be tuned on all its rows");
    const int nt = std::min(ni, TUNE_NI);
    const TuneKey key{ilog2(std::max(nt, 1)), ilog2(std::max(R.nj, 1)), mf ? 1 : 0};
    bool tune_now = false;
    if (R.forced_ni_per_thread != 0) {
        variant = R.forced_ni_per_thread;
    } else if (R.autotune) {
        auto it = R.tuned.find(key);
        if (it != R.tuned.end()) variant = it->second;
        else tune_now = true;
    }
    // admissible variants for this bucket
    int cands[12], ncand = 0;
    if (tune_now) {
        if (ni >= NT / 2) {
            cands[ncand++] = 1;
            cands[ncand++] = 11;
            cands[ncand++] = 13;
            if (ni >= NT * 2) {
                cands[ncand++] = 2;
                cands[ncand++] = 12;
            }
        }
        if (ni <= 2048)
            for (int ib : {1, 2, 4, 8})
                if (ib <= 2 * ni) cands[ncand++] = -ib;
        if (ncand == 0) tune_now = false;
    }
    Plan plan = make_plan(variant, ni, R.nj, R.ntile, mf, R.forced_slices);
    size_t part_need = (size_t)plan.nslices * ni_pad;
    if (tune_now)
        for (int c = 0; c < ncand; ++c)
            part_need = std::max<size_t>(part_need, (size_t)make_plan(cands[c], nt, R.nj, R.ntile, mf, 0).nslices * nt);
    R.part.reserve(part_need * 4);
    nbcnt_reserve(ni, st);
    R.nbbuf.reserve((size_t)ni * std::max(cap, 1));
    R.outf.reserve((size_t)ni * 8);
    R.outl.reserve((size_t)ni * W);

    // the spatial order serves the packed tile kernels (far tiles); a call
    // that runs the j-parallel kernel does not wait for it
    const bool sorted = (tune_now || variant > 0) && ensure_sorted(st);
    RegArgs a;
    a.posH = sorted ? R.posH_s.ptr : R.posH.ptr;
    a.posL = sorted ? R.posL_s.ptr : R.posL.ptr;
    a.vel = sorted ? R.vel_s.ptr : R.vel.ptr;
    a.comp = sorted ? R.comp_s.ptr : R.comp.ptr;
    a.compd = sorted ? R.compd_s.ptr : R.compd.ptr;
    a.perm = sorted ? R.perm.ptr : nullptr;
    static const int far_path = [] {
        const char *e = getenv("NB6_FARPATH");
        return (e && atoi(e) == 0) ? 0 : 1;
    }();
    a.tbox = (sorted && far_path) ? R.tbox.ptr : nullptr;
    a.comprel = (sorted && far_path) ? R.comprel.ptr : nullptr;
    static const int i_order = [] {
        const char *e = getenv("NB6_IORDER");
        return (e && atoi(e) == 0) ? 0 : 1;
    }();
    if (i_order && a.tbox && ni > NT && ni <= ISORT_MAX) {
        R.iperm.reserve(ni);
        // the order reads this call's i positions: a host call's staging
        // must be on the device first (the submission copies it again)
        if (L.hin)
            NB6_CUDA_CHECK(cudaMemcpyAsync(R.iin.ptr, L.hin, L.in_bytes, cudaMemcpyHostToDevice, st));
        iset_order<<<1, 1024, 0, st>>>(ni, d_x, R.ext.ptr, R.iperm.ptr);
        NB6_CUDA_CHECK(cudaGetLastError());
        a.iperm = R.iperm.ptr;
    }
    a.npad = R.npad;
    a.jm = R.jm.ptr;
    a.jx = R.jx.ptr;
    a.jv = R.jv.ptr;
    a.nj = R.nj;
    a.ntile = R.ntile;
    a.nslices = plan.nslices;
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
    if (!R.tev0) {
        NB6_CUDA_CHECK(cudaEventCreate(&R.tev0));
        NB6_CUDA_CHECK(cudaEventCreate(&R.tev1));
    }
    if (tune_now) {
        // the trials read the i data: stage it first when the call brings it
        if (L.hin)
            NB6_CUDA_CHECK(cudaMemcpyAsync(R.iin.ptr, L.hin, L.in_bytes, cudaMemcpyHostToDevice, st));
        // time each candidate three times and keep its best (after one
        // warm-up launch whose time is not compared); when the warm-up took
        // 2 ms or more, once: the noise of so long a launch is well inside
        // the 3% tie below, and the trials of a large bucket would
        // otherwise cost ~16 such launches.  Neighbour counters are reset
        // before every trial.
        float best = 1e30f, tdefault = 1e30f, twarm = 0.f;
        int bestv = variant;
        const int vdefault = default_variant(nt);
        for (int c = -1; c < ncand; ++c) {
            const int v = cands[c < 0 ? 0 : c];
            Plan p = make_plan(v, nt, R.nj, R.ntile, mf, 0);
            RegArgs t = a;
            t.nslices = p.nslices;
            t.ni = t.ni_pad = nt;
            float vbest = 1e30f;
            const int reps = c < 0 ? 1 : (twarm >= 2.0f ? 1 : 3);
            for (int rep = 0; rep < reps; ++rep) {
                NB6_CUDA_CHECK(cudaMemsetAsync(R.nbcnt.ptr, 0, sizeof(int) * nt, st));
                NB6_CUDA_CHECK(cudaEventRecord(R.tev0, st));
                if (mf) launch_plan<true>(p, t, st);
                else launch_plan<false>(p, t, st);
                NB6_CUDA_CHECK(cudaGetLastError());
                NB6_CUDA_CHECK(cudaEventRecord(R.tev1, st));
                NB6_CUDA_CHECK(cudaEventSynchronize(R.tev1));
                float ms = 0.f;
                NB6_CUDA_CHECK(cudaEventElapsedTime(&ms, R.tev0, R.tev1));
                vbest = std::min(vbest, ms);
            }
            if (c < 0) twarm = vbest;
            if (c >= 0 && vbest < best) {
                best = vbest;
                bestv = v;
            }
            if (c >= 0 && v == vdefault) tdefault = vbest;
        }
        // timings within 3% are a tie, and a tie keeps the default: the
        // choice then no longer flips between processes on timing noise
        if (tdefault <= 1.03f * best) {
            bestv = vdefault;
            best = tdefault;
        }
        R.nbcnt_dirty = true;
        R.tuned[key] = bestv;
        variant = bestv;
        plan = make_plan(variant, ni, R.nj, R.ntile, mf, R.forced_slices);
        a.nslices = plan.nslices;
        if (getenv("NB6_VERBOSE"))
            fprintf(stderr, "# nb6 autotune: ni~2^%d nj~2^%d mflag %d -> variant %d (%.3f ms)\n",
                    key.li, key.lj, key.mf, bestv, best);
    }
    if (plan.variant < 0 && a.perm) {
        // the j-parallel kernel takes the j set in its sent order, whether
        // or not this call's trials needed the spatial order: the same
        // variant always sums in the same order
        a.posH = R.posH.ptr;
        a.posL = R.posL.ptr;
        a.vel = R.vel.ptr;
        a.comp = R.comp.ptr;
        a.compd = R.compd.ptr;
        a.perm = nullptr;
        a.tbox = nullptr;
        a.iperm = nullptr;
        a.comprel = nullptr;
    }
    R.last_geometry[0] = plan.variant;
    R.last_geometry[1] = plan.igrid;
    R.last_geometry[2] = plan.nslices;

    int pmax = 32;
    while (pmax < cap) pmax <<= 1;
    const MlpArgs mlp = nb6_mlp_args(d_h2, d_dtr);
    const size_t smem = (size_t)FIN_WARPS * pmax * sizeof(int) + (mlp.on ? MLP_SMEM_BYTES : 0);
    if (smem > 48 * 1024)
        NB6_CUDA_CHECK(cudaFuncSetAttribute(regf_finalize, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)smem));
    L.mlp = mlp;
    if (L.hin) {
        R.houtf.reserve((size_t)ni * 8);
        R.houtl.reserve((size_t)ni * W);
    }
    L.direct = L.hin != nullptr && nb6_uva();
    L.outf = L.direct ? R.houtf.ptr : R.outf.ptr;
    L.outl = L.direct ? R.houtl.ptr : R.outl.ptr;
    L.plan = plan;
    L.a = a;
    L.ni = ni;
    L.W = W;
    L.cap = cap;
    L.pmax = pmax;
    L.smem = smem;
    L.fblocks = (ni + FIN_WARPS - 1) / FIN_WARPS;
    L.mf = mf;
}

// Copies back to the host staging buffers (kind 1 only).
static void regf_copy_out(const RegLaunch &L, cudaStream_t st) {
    NB6_CUDA_CHECK(cudaMemcpyAsync(R.houtf.ptr, R.outf.ptr, sizeof(double) * 8 * L.ni,
                                   cudaMemcpyDeviceToHost, st));
    NB6_CUDA_CHECK(cudaMemcpyAsync(R.houtl.ptr, R.outl.ptr, sizeof(int) * (size_t)L.W * L.ni,
                                   cudaMemcpyDeviceToHost, st));
}

static void regf_eager(const RegLaunch &L, cudaStream_t st) {
    if (L.hin)
        NB6_CUDA_CHECK(cudaMemcpyAsync(R.iin.ptr, L.hin, L.in_bytes, cudaMemcpyHostToDevice, st));
    NB6_CUDA_CHECK(cudaMemsetAsync(R.nbcnt.ptr, 0, sizeof(int) * (R.nbcnt_dirty ? R.nbcnt.cap : (size_t)L.ni), st));
    // kernel-only timing of the main force kernel (read by
    // nb6_regf_last_kernel_ms_ after the stream has drained)
    NB6_CUDA_CHECK(cudaEventRecord(R.ev0, st));
    if (L.mf) launch_plan<true>(L.plan, L.a, st);
    else launch_plan<false>(L.plan, L.a, st);
    NB6_CUDA_CHECK(cudaGetLastError());
    NB6_CUDA_CHECK(cudaEventRecord(R.ev1, st));
    regf_finalize<<<L.fblocks, FIN_WARPS * 32, L.smem, st>>>(
        L.a.part, L.plan.nslices, L.ni, L.a.ni_pad, R.nbcnt.ptr, R.nbbuf.ptr, L.a.lcap, L.cap, L.W,
        L.pmax, L.outf, L.outl, L.mlp);
    NB6_CUDA_CHECK(cudaGetLastError());
    if (L.hin && !L.direct) regf_copy_out(L, st);
    R.nbcnt_dirty = false;
}

static cudaKernelNodeParams main_node(const RegLaunch &L, void **args) {
    cudaKernelNodeParams k{};
    k.func = (void *)(L.mf ? kernel_of<true>(L.plan.variant) : kernel_of<false>(L.plan.variant));
    k.gridDim = dim3(L.plan.igrid, L.plan.nslices);
    k.blockDim = dim3(L.plan.variant > 0 ? NT : JPAR_NT);
    k.sharedMemBytes = 0;
    k.kernelParams = args;
    return k;
}

static cudaKernelNodeParams fin_node(const RegLaunch &L, FinArgs &f) {
    cudaKernelNodeParams k{};
    k.func = (void *)regf_finalize;
    k.gridDim = dim3(L.fblocks);
    k.blockDim = dim3(FIN_WARPS * 32);
    k.sharedMemBytes = (unsigned)L.smem;
    k.kernelParams = f.p;
    return k;
}

#define NB6_GRAPH_TRY(call)              \
    do {                                 \
        if ((call) != cudaSuccess) return false; \
    } while (0)

static bool graph_build(RegState::Graph &G, const RegLaunch &L) {
    const bool io = L.hin != nullptr;
    NB6_GRAPH_TRY(cudaGraphCreate(&G.g, 0));
    cudaGraphNode_t prev = nullptr, n = nullptr;
    auto deps = [&]() { return prev ? &prev : (cudaGraphNode_t *)nullptr; };
    auto ndeps = [&]() { return (size_t)(prev ? 1 : 0); };
    if (io) {
        NB6_GRAPH_TRY(cudaGraphAddMemcpyNode1D(&G.h2d, G.g, deps(), ndeps(), R.iin.ptr, L.hin, L.in_bytes,
                                               cudaMemcpyHostToDevice));
        prev = G.h2d;
    }
    NB6_GRAPH_TRY(cudaGraphAddEventRecordNode(&n, G.g, deps(), ndeps(), R.ev0));
    prev = n;
    RegArgs a = L.a;
    void *margs[1] = {&a};
    const cudaKernelNodeParams km = main_node(L, margs);
    NB6_GRAPH_TRY(cudaGraphAddKernelNode(&G.kmain, G.g, deps(), ndeps(), &km));
    prev = G.kmain;
    NB6_GRAPH_TRY(cudaGraphAddEventRecordNode(&n, G.g, deps(), ndeps(), R.ev1));
    prev = n;
    FinArgs f(L);
    const cudaKernelNodeParams kf = fin_node(L, f);
    NB6_GRAPH_TRY(cudaGraphAddKernelNode(&G.kfin, G.g, deps(), ndeps(), &kf));
    prev = G.kfin;
    if (io && !L.direct) {
        NB6_GRAPH_TRY(cudaGraphAddMemcpyNode1D(&G.d2hf, G.g, deps(), ndeps(), R.houtf.ptr, R.outf.ptr,
                                               sizeof(double) * 8 * L.ni, cudaMemcpyDeviceToHost));
        prev = G.d2hf;
        NB6_GRAPH_TRY(cudaGraphAddMemcpyNode1D(&G.d2hl, G.g, deps(), ndeps(), R.houtl.ptr, R.outl.ptr,
                                               sizeof(int) * (size_t)L.W * L.ni, cudaMemcpyDeviceToHost));
    }
    NB6_GRAPH_TRY(cudaGraphInstantiate(&G.x, G.g, 0));
    R.graph_builds++;
    return true;
}

static bool graph_update(RegState::Graph &G, const RegLaunch &L) {
    const bool io = L.hin != nullptr;
    if (io)
        NB6_GRAPH_TRY(cudaGraphExecMemcpyNodeSetParams1D(G.x, G.h2d, R.iin.ptr, L.hin, L.in_bytes,
                                                         cudaMemcpyHostToDevice));
    RegArgs a = L.a;
    void *margs[1] = {&a};
    const cudaKernelNodeParams km = main_node(L, margs);
    NB6_GRAPH_TRY(cudaGraphExecKernelNodeSetParams(G.x, G.kmain, &km));
    FinArgs f(L);
    const cudaKernelNodeParams kf = fin_node(L, f);
    NB6_GRAPH_TRY(cudaGraphExecKernelNodeSetParams(G.x, G.kfin, &kf));
    if (io && !L.direct) {
        NB6_GRAPH_TRY(cudaGraphExecMemcpyNodeSetParams1D(G.x, G.d2hf, R.houtf.ptr, R.outf.ptr,
                                                         sizeof(double) * 8 * L.ni, cudaMemcpyDeviceToHost));
        NB6_GRAPH_TRY(cudaGraphExecMemcpyNodeSetParams1D(G.x, G.d2hl, R.houtl.ptr, R.outl.ptr,
                                                         sizeof(int) * (size_t)L.W * L.ni,
                                                         cudaMemcpyDeviceToHost));
    }
    return true;
}
#undef NB6_GRAPH_TRY

static void clear_graphs() {
    for (auto &G : R.graph) {
        if (G.x) cudaGraphExecDestroy(G.x);
        if (G.g) cudaGraphDestroy(G.g);
        G = RegState::Graph{};
    }
}

// Enqueue one call: as a graph launch when graphs are on (NB6_GRAPHS=0 or
// nb6_regf_graphs_(0) turns them off), else as individual launches.  A graph
// API error turns graphs off for the rest of the run and falls back to
// launches for this call.
static void regf_submit(const RegLaunch &L, cudaStream_t st) {
    if (R.use_graphs < 0) {
        const char *e = getenv("NB6_GRAPHS");
        R.use_graphs = (e && atoi(e) == 0) ? 0 : 1;
    }
    if (!R.use_graphs) {
        regf_eager(L, st);
        return;
    }
    RegState::Graph &G = R.graph[L.hin ? 1 : 0];
    bool ok = G.x ? graph_update(G, L) : graph_build(G, L);
    if (ok) {
        // (a call that failed or the tuner's trials may have left any row
        // counted: clear them all)
        if (R.nbcnt_dirty) NB6_CUDA_CHECK(cudaMemsetAsync(R.nbcnt.ptr, 0, sizeof(int) * R.nbcnt.cap, st));
        ok = cudaGraphLaunch(G.x, st) == cudaSuccess;
    }
    if (!ok) {
        const cudaError_t e = cudaGetLastError();
        fprintf(stderr, "libnb6b200: CUDA graph path unavailable (%s); using plain launches\n",
                cudaGetErrorName(e));
        clear_graphs();
        R.use_graphs = 0;
        regf_eager(L, st);
        return;
    }
    R.nbcnt_dirty = false;
    R.graph_launches++;
}

// Device-resident regular force (i data already on the device).
static void regf_device(int ni, const double *d_h2, const double *d_dtr, const double *d_x,
                        const double *d_v, int lmax, int nnbmax, int mflag, cudaStream_t st,
                        int &W) {
    RegLaunch L;
    regf_prepare(ni, d_h2, d_dtr, d_x, d_v, lmax, nnbmax, mflag, st, L);
    W = L.W;
    regf_submit(L, st);
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
    nb6_lib_opened();
    R.nbodymax = *nbmax;
    size_j_buffers(std::max(*nbmax, 1));
    R.nj = 0;
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
    clear_graphs();
    R.nbcnt_dirty = true;
    R.posH.release();
    R.posL.release();
    R.vel.release();
    R.comp.release();
    R.compd.release();
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
    nb6_lib_closed();
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
    if (R.selfcheck < 0) {
        const char *e = getenv("NB6_SELFCHECK");
        R.selfcheck = (e && atoi(e) != 0) ? 1 : 0;
    }
    if (R.selfcheck) {
        R.chk_m.assign(mj, mj + n);
        R.chk_x.assign(&xj[0][0], &xj[0][0] + 3 * (size_t)n);
        R.chk_v.assign(&vj[0][0], &vj[0][0] + 3 * (size_t)n);
    }
    cudaStream_t st = nb6_stream();
    const JSetOut o = size_j_buffers(n);
    if (n > 0) {
        NB6_CUDA_CHECK(cudaMemcpyAsync(R.jm.ptr, mj, sizeof(double) * n, cudaMemcpyHostToDevice, st));
        NB6_CUDA_CHECK(cudaMemcpyAsync(R.jx.ptr, xj, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, st));
        NB6_CUDA_CHECK(cudaMemcpyAsync(R.jv.ptr, vj, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, st));
    }
    const int blocks = (int)std::min<size_t>((o.npad + 255) / 256, (size_t)nb6_num_sms() * 8);
    regf_pack_j<<<blocks, 256, 0, st>>>(n, o, R.jm.ptr, R.jx.ptr, R.jv.ptr, nb6_dev_status());
    NB6_CUDA_CHECK(cudaGetLastError());
    R.time_send += nb6_wtime();
}

}  // extern "C"

// Internal hook for the device-resident predictor (predictor.cu): a send whose
// j data are produced on the device.  Sizes the j buffers for n bodies, makes
// them current, and hands out the arrays to fill: FP64 m, x, v for the exact
// neighbour recheck and the float layouts (JSetOut), which the caller's
// kernel writes for j < npad with write_j.
bool regular_bind_j(int n, double **jm, double **jx, double **jv, JSetOut *out) {
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
    *out = size_j_buffers(n);
    *jm = R.jm.ptr;
    *jx = R.jx.ptr;
    *jv = R.jv.ptr;
    return true;
}

// Results of a finished call, from the pinned staging into the caller's
// arrays (reference layout: acc/jrk [ni][3], pot [ni], list rows of lmax).
// Calls of at least this many bodies stage their inputs and unpack their
// results on the library's copy threads (copy_pool.h).
constexpr int POOL_MIN_NI = 256;

static void unpack_rows(int lo, int hi, int W, int lmax, double (*acc)[3], double (*jrk)[3], double *pot,
                        int *list) {
    const double *of = R.houtf.ptr;
    const int *ol = R.houtl.ptr;
    for (int i = lo; i < hi; ++i) {
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
}

static void unpack_results(int ni, int W, int lmax, double (*acc)[3], double (*jrk)[3], double *pot,
                           int *list) {
    if (ni < POOL_MIN_NI) {
        unpack_rows(0, ni, W, lmax, acc, jrk, pot, list);
        return;
    }
    CopyPool &pool = nb6_copy_pool();
    const int np = pool.parts();
    pool.run([&](int p) {
        unpack_rows((int)((long long)ni * p / np), (int)((long long)ni * (p + 1) / np), W, lmax, acc, jrk, pot,
                    list);
    });
}

// Stage a call's i data as [h2 | dtr | x | v] in the pinned block h and
// report whether any value is NaN, in one pass (split over the copy threads
// for large calls).
static bool stage_inputs(int ni, double *h, const double *h2, const double *dtr, const double *xi,
                         const double *vi) {
    auto part = [&](int lo, int hi) {
        bool nan = false;
        for (int k = lo; k < hi; ++k) {
            h[k] = h2[k];
            h[ni + k] = dtr[k];
            nan |= (h2[k] != h2[k]) | (dtr[k] != dtr[k]);
        }
        for (int k = 3 * lo; k < 3 * hi; ++k) {
            h[2 * (size_t)ni + k] = xi[k];
            h[5 * (size_t)ni + k] = vi[k];
            nan |= (xi[k] != xi[k]) | (vi[k] != vi[k]);
        }
        return nan;
    };
    if (ni < POOL_MIN_NI) return part(0, ni);
    CopyPool &pool = nb6_copy_pool();
    const int np = pool.parts();
    bool nan[64] = {};
    pool.run([&](int p) { nan[p] = part((int)((long long)ni * p / np), (int)((long long)ni * (p + 1) / np)); });
    bool any = false;
    for (int p = 0; p < np; ++p) any |= nan[p];
    return any;
}

// Diagnostic (NB6_SELFCHECK=1, off by default): re-derive sample rows of a
// finished gpunb_regf_ call on the host in FP64 with the rule of
// regint.f:41-65 (strict "<") and report rows whose neighbour list differs or
// whose force/jerk/potential is off by more than 1e-5 relative.
static void selfcheck_rows(int ni, const double *h2, const double *dtr, const double (*xi)[3],
                           const double (*vi)[3], const double (*acc)[3], const double (*jrk)[3],
                           const double *pot, const int *list, int lmax, int nnbmax, int mflag) {
    const int nj = (int)R.chk_m.size();
    if (nj != R.nj) return;
    const int cap = std::max(0, std::min(nnbmax, lmax - 1));
    int rows[4] = {0, ni / 3, (2 * ni) / 3, ni - 1};
    for (int r : rows) {
        if (r < 0 || r >= ni) continue;
        double a[3] = {0, 0, 0}, jk[3] = {0, 0, 0}, po = 0;
        std::vector<int> ids;
        for (int j = 0; j < nj; ++j) {
            double d[3], dv[3], r2 = 0, r2p = 0, rv = 0;
            for (int k = 0; k < 3; ++k) {
                d[k] = R.chk_x[3 * (size_t)j + k] - xi[r][k];
                dv[k] = R.chk_v[3 * (size_t)j + k] - vi[r][k];
            }
            r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            const double p0 = d[0] + dtr[r] * dv[0], p1 = d[1] + dtr[r] * dv[1], p2 = d[2] + dtr[r] * dv[2];
            r2p = p0 * p0 + p1 * p1 + p2 * p2;
            const double crit = mflag ? R.chk_m[j] * h2[r] : h2[r];
            if ((r2 < r2p ? r2 : r2p) < crit) {
                ids.push_back(j);
                continue;
            }
            rv = d[0] * dv[0] + d[1] * dv[1] + d[2] * dv[2];
            const double ri2 = 1.0 / r2, ri = sqrt(ri2), mr = R.chk_m[j] * ri, mr3 = mr * ri2;
            const double al = -3.0 * rv * ri2;
            po += mr;
            for (int k = 0; k < 3; ++k) {
                a[k] += mr3 * d[k];
                jk[k] += mr3 * (dv[k] + al * d[k]);
            }
        }
        R.chk_rows++;
        const int *row = list + (size_t)r * lmax;
        const int nnb = (int)ids.size();
        bool bad = (nnb > cap) ? (row[0] != -nnb) : (row[0] != nnb);
        if (!bad && nnb <= cap)
            for (int k = 0; k < nnb; ++k) bad = bad || row[1 + k] != ids[k];
        double ea = 0, ej = 0, na = 0, nj2 = 0;
        for (int k = 0; k < 3; ++k) {
            ea += (acc[r][k] - a[k]) * (acc[r][k] - a[k]);
            na += a[k] * a[k];
            ej += (jrk[r][k] - jk[k]) * (jrk[r][k] - jk[k]);
            nj2 += jk[k] * jk[k];
        }
        const double era = sqrt(ea / (na > 0 ? na : 1)), erj = sqrt(ej / (nj2 > 0 ? nj2 : 1));
        const double erp = fabs(pot[r] - po) / (po > 0 ? po : 1);
        if (nnb <= cap && (era > 1e-5 || erj > 1e-4 || erp > 1e-5)) bad = true;
        if (bad) {
            R.chk_bad++;
            fprintf(stderr,
                    "# nb6 selfcheck: call ni=%d nj=%d variant %d grid (%d,%d) row %d: nnb %d (fp64 %d), acc err %.2e,"
                    " jrk err %.2e, pot err %.2e\n",
                    ni, nj, R.last_geometry[0], R.last_geometry[1], R.last_geometry[2], r, row[0], nnb, era, erj,
                    erp);
        }
    }
}

// Set while regular_seg_on_device runs nb6_regf_seg_: results stay in the
// device buffers and nothing is synchronised or unpacked.
static bool g_seg_keep_device = false;

template <bool MF> static const void *seg_kernel_of(int ib) {
    switch (ib) {
        case 1: return (const void *)regf_seg_kernel<1, MF>;
        case 2: return jpar_x2() ? (const void *)regf_seg_kernel<2, MF, true> : (const void *)regf_seg_kernel<2, MF>;
        default: return jpar_x2() ? (const void *)regf_seg_kernel<4, MF, true> : (const void *)regf_seg_kernel<4, MF>;
    }
}

static int seg_occupancy(int ib, bool mf) {
    static std::map<int, int> cache;
    const int key = ib * 2 + (mf ? 1 : 0);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    int occ = 0;
    NB6_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &occ, mf ? seg_kernel_of<true>(ib) : seg_kernel_of<false>(ib), JPAR_NT, 0));
    occ = std::max(occ, 1);
    cache[key] = occ;
    return occ;
}

template <int IB, bool MF>
static void launch_seg_t(int grid, const RegArgs &a, const SegItem *items, const int *nit,
                         const int2 *pinfo, cudaStream_t st) {
    if (IB > 1 && jpar_x2()) regf_seg_kernel<IB, MF, true><<<grid, JPAR_NT, 0, st>>>(a, items, nit, pinfo);
    else regf_seg_kernel<IB, MF><<<grid, JPAR_NT, 0, st>>>(a, items, nit, pinfo);
}

static void launch_seg(int ib, bool mf, int grid, const RegArgs &a, const SegItem *items, const int *nit,
                       const int2 *pinfo, cudaStream_t st) {
    switch (ib * 2 + (mf ? 1 : 0)) {
        case 2: launch_seg_t<1, false>(grid, a, items, nit, pinfo, st); break;
        case 3: launch_seg_t<1, true>(grid, a, items, nit, pinfo, st); break;
        case 4: launch_seg_t<2, false>(grid, a, items, nit, pinfo, st); break;
        case 5: launch_seg_t<2, true>(grid, a, items, nit, pinfo, st); break;
        case 8: launch_seg_t<4, false>(grid, a, items, nit, pinfo, st); break;
        default: launch_seg_t<4, true>(grid, a, items, nit, pinfo, st); break;
    }
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
    // stage i data: [h2 | dtr | x | v] in one pinned block, one H2D
    const size_t nin = (size_t)8 * ni;
    R.hin.reserve(nin);
    R.iin.reserve(nin);
    double *h = R.hin.ptr;
    if (stage_inputs(ni, h, h2, dtr, &xi[0][0], &vi[0][0])) {
        fprintf(stderr, "gpunb_regf: NaN in i-particle input\n");
        nb6_fatal(NB6_ERR_NAN_INPUT);
        return;
    }
    R.time_grav -= nb6_wtime();
    R.numInter += (long long)ni * R.nj;
    R.ini += ni;
    R.icall++;
    cudaStream_t st = nb6_stream();
    const double *d = R.iin.ptr;

    // one submission: H2D of the staged i data, force kernel, finalize and
    // the D2H of the results (a graph launch unless graphs are off)
    RegLaunch L;
    L.hin = h;
    L.in_bytes = sizeof(double) * nin;
    regf_prepare(ni, d, d + ni, d + 2 * (size_t)ni, d + 5 * (size_t)ni, lmax, nnbmax, *m_flag, st, L);
    const int W = L.W;
    regf_submit(L, st);
    nb6_status_fetch(st);
    if (ni >= POOL_MIN_NI) nb6_copy_pool().arm();   // the helpers spin while the GPU works
    NB6_CUDA_CHECK(cudaStreamSynchronize(st));
    NB6_CUDA_CHECK(cudaEventElapsedTime(&R.last_kernel_ms, R.ev0, R.ev1));
    const double wt = nb6_wtime();
    R.time_grav += wt;
    R.time_reduce -= wt;
    if (nb6_check_dev_status() != 0) {
        R.nbcnt_dirty = true;
        return;
    }

    unpack_results(ni, W, lmax, acc, jrk, pot, list);
    R.time_reduce += nb6_wtime();
    if (R.selfcheck > 0)
        selfcheck_rows(ni, h2, dtr, xi, vi, acc, jrk, pot, list, lmax, nnbmax, *m_flag);
}

// Segmented regular force: gpunb_regf_ for an ensemble of independent
// clusters sent together.  Segment c is the j range [seg_j0[c], seg_j0[c+1])
// of the last send; active particle k belongs to segment iseg[k] (iseg
// non-decreasing, so each cluster's active particles are contiguous) and
// interacts with that segment only.  Outputs as gpunb_regf_, neighbour ids
// relative to seg_j0[iseg[k]].  One persistent kernel launch covers every
// cluster.
void nb6_regf_seg_(int *ni_, int *iseg, double *h2, double *dtr, double (*xi)[3], double (*vi)[3],
                   double (*acc)[3], double (*jrk)[3], double *pot, int *lmax_, int *nnbmax_,
                   int *list, int *m_flag, int *nseg_, int *seg_j0) {
    if (!R.open) {
        nb6_fatal(NB6_ERR_NOT_OPEN);
        return;
    }
    const int ni = *ni_, lmax = *lmax_, nnbmax = *nnbmax_, nseg = *nseg_;
    bool bad = ni <= 0 || lmax < 1 || std::min(nnbmax, lmax - 1) > 8191 || nseg <= 0 ||
               seg_j0[0] < 0 || seg_j0[nseg] > R.nj;
    for (int c = 0; c < nseg && !bad; ++c) bad = seg_j0[c + 1] < seg_j0[c];
    for (int k = 0; k < ni && !bad; ++k)
        bad = iseg[k] < 0 || iseg[k] >= nseg || (k > 0 && iseg[k] < iseg[k - 1]);
    if (bad) {
        fprintf(stderr, "nb6_regf_seg: bad ni, lmax, list cap, segment bounds or segment order\n");
        nb6_fatal(NB6_ERR_BAD_ARG);
        return;
    }
    if (any_nan(h2, ni) || any_nan(dtr, ni) || any_nan(&xi[0][0], 3 * (size_t)ni) ||
        any_nan(&vi[0][0], 3 * (size_t)ni)) {
        fprintf(stderr, "nb6_regf_seg: NaN in i-particle input\n");
        nb6_fatal(NB6_ERR_NAN_INPUT);
        return;
    }
    const double t_start = nb6_wtime();
    R.ini += ni;
    R.icall++;
    cudaStream_t st = nb6_stream();
    const int cap = std::max(0, std::min(nnbmax, lmax - 1));
    const int W = cap + 1;
    const bool mf = *m_flag != 0;

    // i data: [h2 | dtr | x | v], as in gpunb_regf_
    const size_t nin = (size_t)8 * ni;
    R.hin.reserve(nin);
    R.iin.reserve(nin);
    double *h = R.hin.ptr;
    memcpy(h, h2, sizeof(double) * ni);
    memcpy(h + ni, dtr, sizeof(double) * ni);
    memcpy(h + 2 * (size_t)ni, xi, sizeof(double) * 3 * ni);
    memcpy(h + 5 * (size_t)ni, vi, sizeof(double) * 3 * ni);

    // One segment spanning a large j set (one big cluster): the tuned tile
    // kernels of gpunb_regf_ (packed pair math, spatial order, far tiles)
    // beat the segmented kernel's j-parallel loop there; the results are the
    // same rows (ids relative to the segment = to the first j sent).
    static const int seg_tile_min = [] {
        const char *e = getenv("NB6_SEG_TILE_MIN");
        return e ? atoi(e) : 32768;
    }();
    if (nseg == 1 && seg_j0[0] == 0 && seg_j0[1] == R.nj && R.nj >= seg_tile_min) {
        R.time_out += nb6_wtime() - t_start;
        R.time_grav -= nb6_wtime();
        R.numInter += (long long)ni * R.nj;
        NB6_CUDA_CHECK(cudaMemcpyAsync(R.iin.ptr, h, sizeof(double) * nin, cudaMemcpyHostToDevice, st));
        const double *d = R.iin.ptr;
        int Wt = W;
        regf_device(ni, d, d + ni, d + 2 * (size_t)ni, d + 5 * (size_t)ni, lmax, nnbmax, *m_flag, st, Wt);
        if (g_seg_keep_device) {
            R.time_grav += nb6_wtime();
            return;
        }
        R.houtf.reserve((size_t)ni * 8);
        R.houtl.reserve((size_t)ni * W);
        NB6_CUDA_CHECK(cudaMemcpyAsync(R.houtf.ptr, R.outf.ptr, sizeof(double) * 8 * ni, cudaMemcpyDeviceToHost,
                                       st));
        NB6_CUDA_CHECK(cudaMemcpyAsync(R.houtl.ptr, R.outl.ptr, sizeof(int) * (size_t)W * ni,
                                       cudaMemcpyDeviceToHost, st));
        nb6_status_fetch(st);
        NB6_CUDA_CHECK(cudaStreamSynchronize(st));
        NB6_CUDA_CHECK(cudaEventElapsedTime(&R.last_kernel_ms, R.ev0, R.ev1));
        const double wt2 = nb6_wtime();
        R.time_grav += wt2;
        R.time_reduce -= wt2;
        if (nb6_check_dev_status() != 0) {
            R.nbcnt_dirty = true;
            return;
        }
        unpack_results(ni, W, lmax, acc, jrk, pot, list);
        R.time_reduce += nb6_wtime();
        return;
    }

    // runs of active particles per segment, and the CTA i-group size
    std::vector<int> run_k0, run_c;
    for (int k = 0; k < ni; ++k)
        if (k == 0 || iseg[k] != iseg[k - 1]) {
            run_k0.push_back(k);
            run_c.push_back(iseg[k]);
        }
    const int nrun = (int)run_k0.size();
    run_k0.push_back(ni);
    // at most 4: the IB = 8 form needs 184 registers (one CTA of 8 warps per
    // SM) against 112 for IB = 4 (two CTAs), and ran 15-17% slower on
    // ensembles of 2-100% active bodies
    int ib = 1;
    while (ib < 4 && ib * nrun < ni) ib <<= 1;
    const int grid_max = nb6_num_sms() * seg_occupancy(ib, mf);
    double work = 0.0;
    for (int r = 0; r < nrun; ++r)
        work += (double)(run_k0[r + 1] - run_k0[r]) * (seg_j0[run_c[r] + 1] - seg_j0[run_c[r]]);
    R.numInter += (long long)work;
    // items of about a quarter wave's share of the work each, at least 4 j
    // per thread
    const double wt = std::max(work / (4.0 * grid_max), (double)ib * JPAR_NT * 4);
    std::vector<SegItem> items;
    std::vector<int2> pinfo(ni);
    long long slots = 0;
    for (int r = 0; r < nrun; ++r) {
        const int c = run_c[r], k0 = run_k0[r], k1 = run_k0[r + 1];
        const int j0 = seg_j0[c], nc = seg_j0[c + 1] - seg_j0[c];
        const int g = std::min(ib, k1 - k0);
        int Q = 0;
        if (nc > 0) {
            const int qmax = (nc + JPAR_NT * 4 - 1) / (JPAR_NT * 4);
            Q = std::max(1, std::min(qmax, (int)std::ceil((double)g * nc / wt)));
        }
        for (int k = k0; k < k1; ++k) pinfo[k] = make_int2((int)(slots + (long long)(k - k0) * Q), Q);
        slots += (long long)(k1 - k0) * Q;
        for (int i0 = k0; i0 < k1; i0 += ib)
            for (int q = 0; q < Q; ++q) {
                SegItem it;
                it.i0 = i0;
                it.ni = std::min(ib, k1 - i0);
                it.j0 = j0 + (int)((long long)nc * q / Q);
                it.j1 = j0 + (int)((long long)nc * (q + 1) / Q);
                it.jbase = j0;
                it.q = q;
                it.pad0 = it.pad1 = 0;
                items.push_back(it);
            }
    }
    std::stable_sort(items.begin(), items.end(), [](const SegItem &x, const SegItem &y) {
        return (long long)x.ni * (x.j1 - x.j0) > (long long)y.ni * (y.j1 - y.j0);
    });
    const int nitems = (int)items.size();
    if (slots > INT_MAX / 4) {
        fprintf(stderr, "nb6_regf_seg: too many partial slots (%lld)\n", slots);
        nb6_fatal(NB6_ERR_TOO_LARGE);
        return;
    }
    // int staging: [nitems, 0, 0, 0 | items (8 ints each) | pinfo (2 ints each)]
    const size_t nint = 4 + (size_t)8 * nitems + (size_t)2 * ni;
    R.hseg.reserve(nint);
    R.dseg.reserve(nint);
    int *hs = R.hseg.ptr;
    hs[0] = nitems;
    hs[1] = hs[2] = hs[3] = 0;
    if (nitems) memcpy(hs + 4, items.data(), sizeof(SegItem) * nitems);
    memcpy(hs + 4 + (size_t)8 * nitems, pinfo.data(), sizeof(int2) * ni);
    const SegItem *d_items = reinterpret_cast<const SegItem *>(R.dseg.ptr + 4);
    const int2 *d_pinfo = reinterpret_cast<const int2 *>(R.dseg.ptr + 4 + (size_t)8 * nitems);

    R.part.reserve((size_t)std::max<long long>(slots, 1) * 4);
    nbcnt_reserve(ni, st);
    R.nbbuf.reserve((size_t)ni * std::max(cap, 1));
    R.outf.reserve((size_t)ni * 8);
    R.outl.reserve((size_t)ni * W);
    R.houtf.reserve((size_t)ni * 8);
    R.houtl.reserve((size_t)ni * W);
    if (!R.ev0) {
        NB6_CUDA_CHECK(cudaEventCreate(&R.ev0));
        NB6_CUDA_CHECK(cudaEventCreate(&R.ev1));
    }
    RegArgs a{};
    a.posH = R.posH.ptr;
    a.posL = R.posL.ptr;
    a.vel = R.vel.ptr;
    a.comp = R.comp.ptr;
    a.compd = R.compd.ptr;
    a.npad = R.npad;
    a.jm = R.jm.ptr;
    a.jx = R.jx.ptr;
    a.jv = R.jv.ptr;
    a.nj = R.nj;
    a.ntile = R.ntile;
    a.nslices = 1;
    const double *d = R.iin.ptr;
    a.ih2 = d;
    a.idtr = d + ni;
    a.ix = d + 2 * (size_t)ni;
    a.iv = d + 5 * (size_t)ni;
    a.ni = ni;
    a.ni_pad = ni;
    a.part = R.part.ptr;
    a.nbcnt = R.nbcnt.ptr;
    a.nbbuf = R.nbbuf.ptr;
    a.lcap = std::max(cap, 1);
    a.status = nb6_dev_status();

    // host preparation (staging, work list) shows as out(s) in the profile,
    // copies + kernels + sync as grav(s), unpacking as nb(s)
    const double t_prep = nb6_wtime();
    R.time_out += t_prep - t_start;
    R.time_grav -= t_prep;
    NB6_CUDA_CHECK(cudaMemcpyAsync(R.iin.ptr, h, sizeof(double) * nin, cudaMemcpyHostToDevice, st));
    NB6_CUDA_CHECK(cudaMemcpyAsync(R.dseg.ptr, hs, sizeof(int) * nint, cudaMemcpyHostToDevice, st));
    NB6_CUDA_CHECK(cudaMemsetAsync(R.nbcnt.ptr, 0, sizeof(int) * ni, st));
    NB6_CUDA_CHECK(cudaEventRecord(R.ev0, st));
    if (nitems > 0)
        launch_seg(ib, mf, std::min(nitems, grid_max), a, d_items, R.dseg.ptr, d_pinfo, st);
    NB6_CUDA_CHECK(cudaGetLastError());
    NB6_CUDA_CHECK(cudaEventRecord(R.ev1, st));
    R.last_geometry[0] = -ib;
    R.last_geometry[1] = std::min(nitems, grid_max);
    R.last_geometry[2] = nitems;
    int pmax = 32;
    while (pmax < cap) pmax <<= 1;
    const MlpArgs mlp = nb6_mlp_args(a.ih2, a.idtr);
    const size_t smem = (size_t)FIN_WARPS * pmax * sizeof(int) + (mlp.on ? MLP_SMEM_BYTES : 0);
    if (smem > 48 * 1024)
        NB6_CUDA_CHECK(cudaFuncSetAttribute(regf_finalize_seg, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)smem));
    // finalize writes the pinned host staging in place, unless a device
    // kernel consumes the results (regular_seg_on_device)
    const bool direct = nb6_uva() && !g_seg_keep_device;
    regf_finalize_seg<<<(ni + FIN_WARPS - 1) / FIN_WARPS, FIN_WARPS * 32, smem, st>>>(
        R.part.ptr, d_pinfo, ni, R.nbcnt.ptr, R.nbbuf.ptr, a.lcap, cap, W, pmax,
        direct ? R.houtf.ptr : R.outf.ptr, direct ? R.houtl.ptr : R.outl.ptr, mlp);
    NB6_CUDA_CHECK(cudaGetLastError());
    if (g_seg_keep_device) {
        R.time_grav += nb6_wtime();
        return;
    }
    if (!direct) {
        NB6_CUDA_CHECK(cudaMemcpyAsync(R.houtf.ptr, R.outf.ptr, sizeof(double) * 8 * ni, cudaMemcpyDeviceToHost,
                                       st));
        NB6_CUDA_CHECK(cudaMemcpyAsync(R.houtl.ptr, R.outl.ptr, sizeof(int) * (size_t)W * ni,
                                       cudaMemcpyDeviceToHost, st));
    }
    nb6_status_fetch(st);
    NB6_CUDA_CHECK(cudaStreamSynchronize(st));
    NB6_CUDA_CHECK(cudaEventElapsedTime(&R.last_kernel_ms, R.ev0, R.ev1));
    const double wt2 = nb6_wtime();
    R.time_grav += wt2;
    R.time_reduce -= wt2;
    if (nb6_check_dev_status() != 0) {
        R.nbcnt_dirty = true;
        return;
    }
    unpack_results(ni, W, lmax, acc, jrk, pot, list);
    R.time_reduce += nb6_wtime();
}

}  // extern "C"

// Segmented regular force for a following device kernel: everything is
// enqueued on the library stream, the results stay in the device output
// buffers (described in *out); the caller synchronises.
bool regular_seg_on_device(int ni, int *iseg, double *h2, double *dtr, double (*xi)[3], double (*vi)[3], int lmax,
                           int nnbmax, int mflag, int nseg, int *seg_j0, RegDeviceOut *out) {
    int n = ni, lm = lmax, nm = nnbmax, mf = mflag, ns = nseg;
    g_seg_keep_device = true;
    nb6_regf_seg_(&n, iseg, h2, dtr, xi, vi, nullptr, nullptr, nullptr, &lm, &nm, nullptr, &mf, &ns, seg_j0);
    g_seg_keep_device = false;
    out->outf = R.outf.ptr;
    out->outl = R.outl.ptr;
    out->W = std::max(0, std::min(nnbmax, lmax - 1)) + 1;
    out->jm = R.jm.ptr;
    out->jx = R.jx.ptr;
    out->jv = R.jv.ptr;
    return nb6_last_status_() == 0;
}

extern "C" {

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
void nb6_regf_tune_(int *variant, int *nslices) {
    const int v = *variant;
    const bool ok = v == 0 || valid_variant(v);
    if (!ok || *nslices < 0) {
        nb6_fatal(NB6_ERR_BAD_ARG);
        return;
    }
    R.forced_ni_per_thread = v;
    R.forced_slices = *nslices;
}

// Enable (1) or disable (0) the measured autotuner; -1 clears its cache.
void nb6_regf_autotune_(int *flag) {
    if (*flag < 0) {
        R.tuned.clear();
        return;
    }
    R.autotune = *flag ? 1 : 0;
}

// The autotuner's choices so far: *n = number of buckets; out[4k..4k+3] =
// (log2 N_active, log2 N_j, m_flag, variant) of bucket k, for the first
// *cap buckets (ascending).
void nb6_regf_tuned_(int *n, int *cap, int *out) {
    int k = 0;
    for (const auto &e : R.tuned) {
        if (k < *cap) {
            out[4 * k] = e.first.li;
            out[4 * k + 1] = e.first.lj;
            out[4 * k + 2] = e.first.mf;
            out[4 * k + 3] = e.second;
        }
        ++k;
    }
    *n = k;
}

// Spatial ordering of the j set for the tile kernels: 1 on (default;
// NB6_JSORT=0 in the environment for off), 0 off, other values query.
// Returns the setting.
int nb6_regf_jsort_(int *flag) {
    if (R.use_jsort < 0) {
        const char *e = getenv("NB6_JSORT");
        R.use_jsort = (e && atoi(e) == 0) ? 0 : 1;
    }
    if (flag && (*flag == 0 || *flag == 1)) {
        R.use_jsort = *flag;
        R.sorted_ver = -1;  // rebuild on the next call if turned on
    }
    return R.use_jsort;
}

// Learned radius proposals of the last gpunb_regf_ / nb6_regf_seg_ call:
// out[k] = dlog RS for active particle k (0 when proposals are off).
void nb6_regf_proposals_(int *ni, double *out) {
    for (int k = 0; k < *ni; ++k) out[k] = R.houtf.ptr ? R.houtf.ptr[8 * (size_t)k + 7] : 0.0;
}

// CUDA-graph submission of regular-force calls: flag 1 turns it on, 0 off
// (plain launches), any other value leaves it as it is.  counts receives
// {graphs built, graph launches, 1 if on else 0}.
void nb6_regf_graphs_(int *flag, long long *counts) {
    if (R.use_graphs < 0) {
        const char *e = getenv("NB6_GRAPHS");
        R.use_graphs = (e && atoi(e) == 0) ? 0 : 1;
    }
    if (flag && (*flag == 0 || *flag == 1)) {
        if (*flag == 0) clear_graphs();
        R.use_graphs = *flag;
    }
    if (counts) {
        counts[0] = R.graph_builds;
        counts[1] = R.graph_launches;
        counts[2] = R.use_graphs;
    }
}

void nb6_sync_() { NB6_CUDA_CHECK(cudaStreamSynchronize(nb6_stream())); nb6_check_dev_status(); }

void *nb6_stream_() { return (void *)nb6_stream(); }

}  // extern "C"

// ============================================================================
// Regular force without any device allocation.
//
// Some callers cannot let this library allocate device memory: a simulation
// whose GPU memory is entirely owned by another allocator (a framework's
// caching pool, or a fixed per-rank budget set when the run starts), or a
// driver that must not change the device's allocation state in the middle of
// a run.  nb6_regf_noalloc_ serves them: the caller passes device-accessible
// inputs and outputs, and the only working memory is the fixed array below,
// which is part of the library image.  Nothing is allocated or freed, not
// even a stream or an event.
//
// The array is NB6_NOALLOC_SCRATCH_BYTES (12 MiB) per GPU and stays resident
// on every GPU that loads the library until the process exits.  It bounds a
// call to ni <= 1024 active particles and a list cap min(nnbmax, lmax-1) <=
// 511; larger requests are rejected.  Every call shares it and it keeps the
// previous call's contents (the neighbour counters are cleared at the start
// of each call): calls that overlap on the GPU -- different streams, or
// different host threads without ordering -- race on it and must not be
// issued.
// ============================================================================

constexpr size_t NB6_NOALLOC_SCRATCH_BYTES = 12u << 20;
constexpr int NA_NIMAX = 1024;
constexpr int NA_CAPMAX = 511;
constexpr int NA_SLICES_MAX = 128;
constexpr int NA_IB = 4;  // i-particles per CTA of the j-parallel kernel

// Layout inside the array: neighbour counters [NA_NIMAX], neighbour ids
// [NA_NIMAX][NA_CAPMAX], slice partials [NA_SLICES_MAX][NA_NIMAX][4] float4.
constexpr size_t NA_OFF_CNT = 0;
constexpr size_t NA_OFF_IDS = 4096;
constexpr size_t NA_OFF_PART = NA_OFF_IDS + (size_t)NA_NIMAX * NA_CAPMAX * sizeof(int) + 4096;
static_assert(NA_OFF_PART % 256 == 0, "alignment");
static_assert(NA_OFF_PART + (size_t)NA_SLICES_MAX * NA_NIMAX * 4 * sizeof(float4) <=
                  NB6_NOALLOC_SCRATCH_BYTES,
              "scratch layout exceeds the array");

static __device__ __align__(256) unsigned char nb6_noalloc_scratch[NB6_NOALLOC_SCRATCH_BYTES];

namespace {

__global__ void na_clear_counts(int *cnt, int ni) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ni) cnt[i] = 0;
}

// j-parallel regular force reading the caller's FP64 j arrays directly
// (hi/lo split on the fly); pair math, candidate test and exact FP64
// re-decision are those of the other regular kernels.
template <bool MFLAG>
__global__ void __launch_bounds__(JPAR_NT) regf_na_kernel(const RegArgs a) {
    __shared__ float4 sip[NA_IB][3];
    __shared__ double red[JPAR_NT / 32][NA_IB][7];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int i0 = blockIdx.x * NA_IB;
    if (tid < NA_IB) {
        const int i = i0 + tid;
        float4 p = make_float4(0.f, 0.f, 0.f, 0.f), q = p, r = p;  // padding: never a candidate
        if (i < a.ni) {
            split_hl(a.ix[3 * i], p.x, q.x);
            split_hl(a.ix[3 * i + 1], p.y, q.y);
            split_hl(a.ix[3 * i + 2], p.z, q.z);
            p.w = (float)a.ih2[i] * CAND_SLACK;
            q.w = (float)a.idtr[i];
            r = make_float4((float)a.iv[3 * i], (float)a.iv[3 * i + 1], (float)a.iv[3 * i + 2], 0.f);
        }
        sip[tid][0] = p;
        sip[tid][1] = q;
        sip[tid][2] = r;
    }
    __syncthreads();
    const int j_begin = (int)(((long long)blockIdx.y * a.nj) / a.nslices);
    const int j_end = (int)(((long long)(blockIdx.y + 1) * a.nj) / a.nslices);
    Sums s[NA_IB];
#pragma unroll
    for (int k = 0; k < NA_IB; ++k) zero(s[k]);
    for (int j = j_begin + tid; j < j_end; j += JPAR_NT) {
        float4 pa, pb;
        split_hl(a.jx[3 * (size_t)j], pa.x, pb.x);
        split_hl(a.jx[3 * (size_t)j + 1], pa.y, pb.y);
        split_hl(a.jx[3 * (size_t)j + 2], pa.z, pb.z);
        pa.w = (float)a.jm[j];
        pb.w = 0.f;
        const float4 pc = make_float4((float)a.jv[3 * (size_t)j], (float)a.jv[3 * (size_t)j + 1],
                                      (float)a.jv[3 * (size_t)j + 2], 0.f);
        bool any = false;
        IPart ips[NA_IB];
#pragma unroll
        for (int k = 0; k < NA_IB; ++k) {
            const float4 p = sip[k][0], q = sip[k][1], r = sip[k][2];
            IPart &ip = ips[k];
            ip.xh = p.x; ip.yh = p.y; ip.zh = p.z; ip.h2c = p.w;
            ip.xl = q.x; ip.yl = q.y; ip.zl = q.z; ip.dt = q.w;
            ip.vx = r.x; ip.vy = r.y; ip.vz = r.z;
            any |= reg_pair<MFLAG>(ip, pa, pb, pc, s[k]);
        }
        if (any) {
            for (int k = 0; k < NA_IB; ++k)
                if (reg_geom<MFLAG>(ips[k], pa, pb, pc).cand) reg_exact<MFLAG>(a, i0 + k, j, s[k]);
        }
    }
#pragma unroll
    for (int k = 0; k < NA_IB; ++k) {
        double v[7] = {s[k].ax, s[k].ay, s[k].az, s[k].jx, s[k].jy, s[k].jz, s[k].po};
#pragma unroll
        for (int c = 0; c < 7; ++c) {
            const double w = warp_sum_d(v[c]);
            if (lane == 0) red[warp][k][c] = w;
        }
    }
    __syncthreads();
    if (tid < NA_IB * 7) {
        const int k = tid / 7, c = tid % 7;
        double w = 0.0;
#pragma unroll
        for (int q = 0; q < JPAR_NT / 32; ++q) w += red[q][k][c];
        const int i = i0 + k;
        if (i < a.ni) {
            float *p = reinterpret_cast<float *>(a.part + ((size_t)blockIdx.y * a.ni_pad + i) * 4);
            const float hi = (float)w;
            p[2 * c] = hi;
            p[2 * c + 1] = (float)(w - (double)hi);
        }
    }
}

// One warp per i: FP64 sum of the slice partials into the caller's acc, jrk
// and pot rows, and the sorted neighbour ids into the caller's list row.
__global__ void __launch_bounds__(FIN_WARPS * 32)
    regf_na_finalize(const float4 *__restrict__ part, int nslices, int ni,
                     const int *__restrict__ nbcnt, const int *__restrict__ nbbuf, int lcap, int cap,
                     int lmax, double *__restrict__ acc, double *__restrict__ jrk,
                     double *__restrict__ pot, int *__restrict__ list) {
    __shared__ int sbuf[FIN_WARPS][512];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.x * FIN_WARPS + warp;
    if (i >= ni) return;
    double v[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int sl = lane; sl < nslices; sl += 32) {
        const float *p = reinterpret_cast<const float *>(part + ((size_t)sl * ni + i) * 4);
#pragma unroll
        for (int c = 0; c < 7; ++c) v[c] += (double)p[2 * c] + (double)p[2 * c + 1];
    }
#pragma unroll
    for (int c = 0; c < 7; ++c) v[c] = warp_sum_d(v[c]);
    if (lane == 0) {
        acc[3 * (size_t)i] = v[0] * 0.125;
        acc[3 * (size_t)i + 1] = v[1] * 0.125;
        acc[3 * (size_t)i + 2] = v[2] * 0.125;
        jrk[3 * (size_t)i] = v[3] * 0.125;
        jrk[3 * (size_t)i + 1] = v[4] * 0.125;
        jrk[3 * (size_t)i + 2] = v[5] * 0.125;
        pot[i] = v[6] * 0.5;
    }
    const int n = nbcnt[i];
    int *row = list + (size_t)i * lmax;
    if (n > cap) {
        if (lane == 0) row[0] = -n;
        return;
    }
    int *sb = sbuf[warp];
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

// Device address of the scratch array, looked up once per device (up to 64
// devices) with that device current.  The lookup is serialised, so host
// threads making their first calls at the same time all get the address.
unsigned char *na_scratch_address(int dev) {
    static unsigned char *addr[64] = {nullptr};
    static std::mutex mu;
    if (dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, nb6_noalloc_scratch);
        if (e != cudaSuccess) {
            fprintf(stderr, "nb6_regf_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
            return nullptr;
        }
        addr[dev] = static_cast<unsigned char *>(p);
    }
    return addr[dev];
}

}  // namespace

extern "C" {

// Regular force + jerk + potential + neighbour list (gpunb_regf_ semantics)
// that allocates nothing.  All array arguments are device-accessible
// pointers in the gpunb_regf_ layouts: j set m[nj], x[nj][3], v[nj][3];
// i set h2[ni], dtr[ni], x[ni][3], v[ni][3]; outputs acc[ni][3], jrk[ni][3],
// pot[ni] and list[ni][lmax] (list[i*lmax] = nnb or -nnb, ids 0-based and
// ascending after it).  Work is enqueued on `stream` (0 = the legacy default
// stream) and the call returns without waiting.  The first call on a device
// looks up the scratch array's device address (cudaGetSymbolAddress, with
// that device current); make that first call before any stream capture.
// Limits: ni <= 1024, min(nnbmax, lmax-1) <= 511.
void nb6_regf_noalloc_(int *nj_, const double *d_mj, const double *d_xj, const double *d_vj,
                       int *ni_, const double *d_h2, const double *d_dtr, const double *d_xi,
                       const double *d_vi, double *d_acc, double *d_jrk, double *d_pot, int *lmax_,
                       int *nnbmax_, int *d_list, int *m_flag, void *stream) {
    const int nj = *nj_, ni = *ni_, lmax = *lmax_, nnbmax = *nnbmax_;
    const int cap = std::max(0, std::min(nnbmax, lmax - 1));
    if (ni <= 0 || ni > NA_NIMAX || nj <= 0 || lmax < 1 || cap > NA_CAPMAX) {
        fprintf(stderr,
                "nb6_regf_noalloc: ni=%d (1..%d), nj=%d (>=1), list cap min(nnbmax,lmax-1)=%d (<=%d) "
                "outside the fixed scratch limits\n",
                ni, NA_NIMAX, nj, cap, NA_CAPMAX);
        nb6_fatal(NB6_ERR_TOO_LARGE);
        return;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        nb6_fatal(NB6_ERR_CUDA);
        return;
    }
    unsigned char *base = na_scratch_address(dev);
    if (!base) {
        nb6_fatal(NB6_ERR_CUDA);
        return;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        nb6_fatal(NB6_ERR_CUDA);
        return;
    }
    RegArgs a = {};
    a.jm = d_mj;
    a.jx = d_xj;
    a.jv = d_vj;
    a.nj = nj;
    a.ih2 = d_h2;
    a.idtr = d_dtr;
    a.ix = d_xi;
    a.iv = d_vi;
    a.ni = ni;
    a.ni_pad = ni;
    a.nbcnt = reinterpret_cast<int *>(base + NA_OFF_CNT);
    a.nbbuf = reinterpret_cast<int *>(base + NA_OFF_IDS);
    a.lcap = std::max(cap, 1);
    a.part = reinterpret_cast<float4 *>(base + NA_OFF_PART);
    const int igroups = (ni + NA_IB - 1) / NA_IB;
    // Two waves of CTAs, and at most 64 j per thread and slice: each
    // thread's FP32 sums then cover as few pairs as a tile of the other
    // kernels before they reach FP64 (up to 2M j within NA_SLICES_MAX).
    const int by_waves = std::min(2 * sms / igroups, nj / (JPAR_NT * 4));
    const int by_sums = (int)(((long long)nj + JPAR_NT * 64 - 1) / (JPAR_NT * 64));
    a.nslices = std::max(1, std::min(std::max(by_waves, by_sums), NA_SLICES_MAX));

    na_clear_counts<<<(ni + 255) / 256, 256, 0, st>>>(a.nbcnt, ni);
    dim3 grid(igroups, a.nslices);
    if (*m_flag) regf_na_kernel<true><<<grid, JPAR_NT, 0, st>>>(a);
    else regf_na_kernel<false><<<grid, JPAR_NT, 0, st>>>(a);
    regf_na_finalize<<<(ni + FIN_WARPS - 1) / FIN_WARPS, FIN_WARPS * 32, 0, st>>>(
        a.part, a.nslices, ni, a.nbcnt, a.nbbuf, a.lcap, cap, lmax, d_acc, d_jrk, d_pot, d_list);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "nb6_regf_noalloc: launch failed: %s\n", cudaGetErrorString(e));
        nb6_fatal(NB6_ERR_CUDA);
    }
}

}  // extern "C"
