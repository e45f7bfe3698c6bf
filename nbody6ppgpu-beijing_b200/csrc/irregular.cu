// irregular.cu -- irregular (neighbour) force + jerk + nearest neighbour
// behind the reference's irr_simd_* C ABI (irr.avx.cpp:568-606), with the
// GPUIRR_* names of the NBODY6/GPU interface as aliases (the calls the
// reference keeps commented out in fpoly0.F:42,70,202,383).
//
// State lives on the device: one 128-byte record per particle
// (x0, x0dot, F = a/2, FDOT = adot/6, mass, t0, all FP64) and one neighbour
// row per particle ([nnb, 0-based ids...], stride lmax).  irr_simd_set_jp_ /
// irr_simd_set_list_ are called once per particle by the Fortran driver, so
// they only write into pinned host staging (a later call for the same
// particle overwrites its staged entry); irr_simd_firr_vec_ uploads what is
// staged, scatters it, and runs one warp per active particle: lanes walk the
// list, predict each j to ti in FP64 (jpred_int.f:16-25) and do the pair
// math and the sums in FP64 -- the walk is bound by the 128-byte record
// gathers, so FP64 costs nothing here and is more accurate than the
// reference's FP32 (irr.avx.cpp:303-332); the nearest neighbour is the minimum FP64 r2 with the
// smallest index on ties (irr.avx.cpp:320-323 packs (r2, idx) the same way).
#include "nb6_common.cuh"
#include "copy_pool.h"

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <climits>
#include <string.h>
#include <vector>

bool regular_bind_j(int n, double **jm, double **jx, double **jv, JSetOut *out);

namespace {

constexpr int IRR_WARPS = 4;
// A large irr_simd_firr_vec_ call runs in up to IRR_CHUNKS launches of at
// least IRR_CHUNK_MIN bodies, so that each chunk's results are downloaded
// and copied into the caller's arrays while the next chunks compute.
constexpr int IRR_CHUNKS = 4, IRR_CHUNK_MIN = 8192;

struct Rec {           // 16 doubles = 128 bytes, one cache line per gather
    double x[3], v[3], f[3], fd[3], m, t0, pad0, pad1;
};

NB6_DEV void predict(const Rec &r, double ti, double *x, double *v) {
    const double s = ti - r.t0;
    const double s1 = 1.5 * s, s2 = 2.0 * s;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        x[k] = ((r.fd[k] * s + r.f[k]) * s + r.v[k]) * s + r.x[k];
        v[k] = (r.fd[k] * s1 + r.f[k]) * s2 + r.v[k];
    }
}

// CG: load through L2 only (ld.global.cg), for records that other CTAs of
// the same launch write (the persistent block kernel); else the read-only
// path.
template <bool CG = false>
NB6_DEV double2 ld_d2(const double2 *q) {
    return CG ? __ldcg(q) : __ldg(q);
}

template <bool CG = false>
NB6_DEV void load_rec(const Rec *__restrict__ p, Rec &r) {
    const double2 *q = reinterpret_cast<const double2 *>(p);
    double2 a = ld_d2<CG>(q + 0), b = ld_d2<CG>(q + 1), c = ld_d2<CG>(q + 2), d = ld_d2<CG>(q + 3);
    double2 e = ld_d2<CG>(q + 4), f = ld_d2<CG>(q + 5), g = ld_d2<CG>(q + 6);
    r.x[0] = a.x; r.x[1] = a.y; r.x[2] = b.x;
    r.v[0] = b.y; r.v[1] = c.x; r.v[2] = c.y;
    r.f[0] = d.x; r.f[1] = d.y; r.f[2] = e.x;
    r.fd[0] = e.y; r.fd[1] = f.x; r.fd[2] = f.y;
    r.m = g.x; r.t0 = g.y;
}

// Perturbed KS pairs whose components the irregular force resolves
// (nb6_ks_set_): slot[a] = pair p of c.m. body a (0-based) or -1; pair p
// has component positions xk[6p..6p+5] and velocities vk[6p..] at the
// block time (first component, then second), masses mk[2p], mk[2p+1], and
// perturbers plist[pofs[p] .. pofs[p+1]) (0-based).  slot == nullptr: no
// table, no corrections.
struct KsArgs {
    const int *slot;
    const double *xk, *vk, *mk;
    const int *pofs, *plist;
};

// Force and jerk on (xi, vi) from a point mass m at (xj, vj), operation
// order of cmfirr_cor.f:47-93.
NB6_DEV void cm_pair(const double *xi, const double *vi, const double *xj, const double *vj, double m, double *f,
                     double *fd) {
    double dx[3], dv[3], dr2 = 0.0, drdv = 0.0;
#pragma unroll
    for (int l = 0; l < 3; ++l) {
        dx[l] = xj[l] - xi[l];
        dv[l] = vj[l] - vi[l];
        dr2 += dx[l] * dx[l];
        drdv += dx[l] * dv[l];
    }
    const double dr2i = 1.0 / dr2;
    const double dr3i = m * dr2i * sqrt(dr2i);
    drdv = 3.0 * drdv * dr2i;
#pragma unroll
    for (int l = 0; l < 3; ++l) {
        f[l] = dx[l] * dr3i;
        fd[l] = (dv[l] - dx[l] * drdv) * dr3i;
    }
}

// The lanes' sums reduced into every lane; the nearest neighbour is the
// smallest r2, the smallest index on ties (1-based, -1 for an empty list).
NB6_DEV void irr_warp_finish(double ax, double ay, double az, double jx, double jy, double jz, double rmin, int jmin,
                             int nnb, double *a, double *jd, int &nnbid) {
    a[0] = warp_sum_d(ax);
    a[1] = warp_sum_d(ay);
    a[2] = warp_sum_d(az);
    jd[0] = warp_sum_d(jx);
    jd[1] = warp_sum_d(jy);
    jd[2] = warp_sum_d(jz);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double r2 = __shfl_xor_sync(0xffffffffu, rmin, o);
        const int j2 = __shfl_xor_sync(0xffffffffu, jmin, o);
        if (r2 < rmin || (r2 == rmin && j2 < jmin)) {
            rmin = r2;
            jmin = j2;
        }
    }
    nnbid = (nnb > 0 && jmin != 0x7fffffff) ? jmin + 1 : -1;
}

// One warp, one active particle i: neighbour force, jerk and nearest
// neighbour (1-based, -1 for an empty list), reduced into every lane.
// With a KS pair table the force includes the c.m. corrections NBINT_COR
// adds on the host (nbint_cor.f:37-65): for a neighbour that is a
// perturbed pair, the sum over its two components replaces its point-mass
// term (cmfirr_ucor.f:14-116); for i itself the c.m. of a perturbed pair,
// the perturbation terms over its perturber list are added instead
// (cmfirr_cor.f:13-130).  An empty list gets no corrections.
// DEEP: the ids of two rounds are loaded with the list header and the
// records of both rounds before their arithmetic -- fewer dependent round
// trips for one body's walk (the block clock's small blocks are bound by
// that latency) at the cost of registers (the bulk calls keep the plain
// walk's occupancy).  Each lane sums its entries l = lane, lane + 32, ...
// in that order either way, so both forms give the same bits.
template <bool KS, bool CG = false, bool DEEP = false>
NB6_DEV void irr_force_warp(int i, int lane, double ti, const Rec *__restrict__ rec,
                            const int *__restrict__ lists, int ls, int nmax, const KsArgs &ks, double *a,
                            double *jd, int &nnbid) {
    Rec ri;
    load_rec<CG>(rec + i, ri);
    double xi[3], vi[3];
    predict(ri, ti, xi, vi);
    const int *row = lists + (size_t)i * ls;
    const int nnb = row[0];
    const int pi = KS ? ks.slot[i] : -1;
    const bool resolve = KS && pi < 0;  // components of perturbed neighbours
    double ax = 0, ay = 0, az = 0, jx = 0, jy = 0, jz = 0;
    double rmin = 1.0e300;
    int jmin = 0x7fffffff;
    auto add = [&](const Rec &rj, int j) {
        double xj[3], vj[3];
        predict(rj, ti, xj, vj);
        const double dxd = xj[0] - xi[0], dyd = xj[1] - xi[1], dzd = xj[2] - xi[2];
        const double r2d = dxd * dxd + dyd * dyd + dzd * dzd;
        if (r2d < rmin || (r2d == rmin && j < jmin)) {
            rmin = r2d;
            jmin = j;
        }
        const int q = resolve ? ks.slot[j] : -1;
        if (q >= 0) {
            double f[3], fd[3];
            for (int c = 0; c < 2; ++c) {
                cm_pair(xi, vi, ks.xk + 6 * (size_t)q + 3 * c, ks.vk + 6 * (size_t)q + 3 * c, ks.mk[2 * q + c], f,
                        fd);
                ax += f[0];
                ay += f[1];
                az += f[2];
                jx += fd[0];
                jy += fd[1];
                jz += fd[2];
            }
            return;
        }
        // The list walk is bound by the record gathers, not by arithmetic,
        // so the pair math stays in FP64 (nbint.F:143-158).
        const double dvx = vj[0] - vi[0], dvy = vj[1] - vi[1], dvz = vj[2] - vi[2];
        const double rinv = rsqrt(r2d);
        const double rinv2 = rinv * rinv;
        const double mr3 = rj.m * rinv * rinv2;
        const double al = -3.0 * (dxd * dvx + dyd * dvy + dzd * dvz) * rinv2;
        ax += mr3 * dxd;
        ay += mr3 * dyd;
        az += mr3 * dzd;
        jx += mr3 * (dvx + al * dxd);
        jy += mr3 * (dvy + al * dyd);
        jz += mr3 * (dvz + al * dzd);
    };
    if (DEEP) {
        int jn0 = 1 + lane < ls ? row[1 + lane] : -1;
        int jn1 = 33 + lane < ls ? row[33 + lane] : -1;
        for (int base = 0; base < nnb; base += 64) {
            const int j0 = base + lane < nnb ? jn0 : -1;
            const int j1 = base + 32 + lane < nnb ? jn1 : -1;
            if (base + 64 < nnb) {
                const int l = base + 65 + lane;
                jn0 = l < ls ? row[l] : -1;
                jn1 = l + 32 < ls ? row[l + 32] : -1;
            }
            const bool v0 = j0 >= 0 && j0 < nmax, v1 = j1 >= 0 && j1 < nmax;   // ids are checked at set_list time
            Rec r0, r1;
            if (v0) load_rec<CG>(rec + j0, r0);
            if (v1) load_rec<CG>(rec + j1, r1);
            if (v0) add(r0, j0);
            if (v1) add(r1, j1);
        }
    } else {
        for (int l = lane; l < nnb; l += 32) {
            const int j = row[1 + l];
            if (j < 0 || j >= nmax) continue;   // ids are checked at set_list time
            Rec rj;
            load_rec<CG>(rec + j, rj);
            add(rj, j);
        }
    }
    if (KS && pi >= 0 && nnb > 0) {
        // i is the c.m. of a perturbed pair: perturbation of its components
        // by each perturber (itself resolved when it is a perturbed pair)
        // minus the perturber's c.m. force on the c.m.
        const double *x1 = ks.xk + 6 * (size_t)pi, *x2 = x1 + 3;
        const double *v1 = ks.vk + 6 * (size_t)pi, *v2 = v1 + 3;
        const double m1 = ks.mk[2 * pi], m2 = ks.mk[2 * pi + 1], mi = ri.m;
        for (int l = ks.pofs[pi] + lane; l < ks.pofs[pi + 1]; l += 32) {
            const int j = ks.plist[l];
            if (j < 0 || j >= nmax) continue;   // ids are checked at set time
            Rec rj;
            load_rec<CG>(rec + j, rj);
            double xj[3], vj[3], fcm[3], fcmd[3];
            predict(rj, ti, xj, vj);
            cm_pair(xi, vi, xj, vj, rj.m, fcm, fcmd);
            const int q = ks.slot[j];
            for (int c = 0; c < (q >= 0 ? 2 : 1); ++c) {
                const double *xs = q >= 0 ? ks.xk + 6 * (size_t)q + 3 * c : xj;
                const double *vs = q >= 0 ? ks.vk + 6 * (size_t)q + 3 * c : vj;
                const double ms = q >= 0 ? ks.mk[2 * q + c] : rj.m;
                double f1[3], fd1[3], f2[3], fd2[3];
                cm_pair(x1, v1, xs, vs, ms, f1, fd1);
                cm_pair(x2, v2, xs, vs, ms, f2, fd2);
                const double s = c == 0 ? 1.0 : 0.0;  // the c.m. term once
                ax += (m1 * f1[0] + m2 * f2[0]) / mi - s * fcm[0];
                ay += (m1 * f1[1] + m2 * f2[1]) / mi - s * fcm[1];
                az += (m1 * f1[2] + m2 * f2[2]) / mi - s * fcm[2];
                jx += (m1 * fd1[0] + m2 * fd2[0]) / mi - s * fcmd[0];
                jy += (m1 * fd1[1] + m2 * fd2[1]) / mi - s * fcmd[1];
                jz += (m1 * fd1[2] + m2 * fd2[2]) / mi - s * fcmd[2];
            }
        }
    }
    irr_warp_finish(ax, ay, az, jx, jy, jz, rmin, jmin, nnb, a, jd, nnbid);
}

// A body predicted to the time of one call: x, m, v in 64 bytes, so a
// neighbour gather moves two 32-byte sectors instead of the record's four.
struct Pv {
    double x[3], m, v[3], pad;
};

// Every record predicted to ti by predict(), the function the record walk
// applies to each neighbour, so the predicted set holds the same bits the
// record walk computes.  A CTA takes PS_NT consecutive records: the threads
// read them as consecutive 16-byte pieces into shared memory, each thread
// predicts one record from there, and the 64-byte bodies leave through
// shared memory the same way, so every global access of a warp is one
// contiguous 512-byte run.  The 16-byte pieces are stored XOR-swizzled so
// that a quarter-warp's accesses fall in distinct bank groups.
constexpr int PS_NT = 128;
__global__ void __launch_bounds__(PS_NT) irr_predict_set(int n, double ti, const Rec *__restrict__ rec,
                                                        Pv *__restrict__ pv) {
    __shared__ double2 sm[PS_NT * 8];   // PS_NT records of 8 pieces; later PS_NT bodies of 4
    const int t = threadIdx.x;
    const int b0 = blockIdx.x * PS_NT;
    const int nb = min(PS_NT, n - b0);
    const double2 *src = reinterpret_cast<const double2 *>(rec + b0);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int q = t + PS_NT * k;   // piece q & 7 of record q >> 3
        if (q < nb * 8) sm[(q & ~7) | ((q & 7) ^ ((q >> 3) & 7))] = __ldg(src + q);
    }
    __syncthreads();
    double x[3], v[3], m = 0.0;
    if (t < nb) {
        const int sw = t & 7;
        const double2 a = sm[t * 8 + (0 ^ sw)], b = sm[t * 8 + (1 ^ sw)], c = sm[t * 8 + (2 ^ sw)];
        const double2 d = sm[t * 8 + (3 ^ sw)], e = sm[t * 8 + (4 ^ sw)], f = sm[t * 8 + (5 ^ sw)];
        const double2 g = sm[t * 8 + (6 ^ sw)];
        Rec r;   // the piece order of load_rec
        r.x[0] = a.x; r.x[1] = a.y; r.x[2] = b.x;
        r.v[0] = b.y; r.v[1] = c.x; r.v[2] = c.y;
        r.f[0] = d.x; r.f[1] = d.y; r.f[2] = e.x;
        r.fd[0] = e.y; r.fd[1] = f.x; r.fd[2] = f.y;
        r.m = g.x; r.t0 = g.y;
        predict(r, ti, x, v);
        m = r.m;
    }
    __syncthreads();
    if (t < nb) {
        const int sw = (t >> 1) & 3;
        sm[t * 4 + (0 ^ sw)] = make_double2(x[0], x[1]);
        sm[t * 4 + (1 ^ sw)] = make_double2(x[2], m);
        sm[t * 4 + (2 ^ sw)] = make_double2(v[0], v[1]);
        sm[t * 4 + (3 ^ sw)] = make_double2(v[2], 0.0);
    }
    __syncthreads();
    double2 *dst = reinterpret_cast<double2 *>(pv + b0);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int q = t + PS_NT * k;   // piece q & 3 of body q >> 2
        if (q < nb * 4) dst[q] = sm[(q & ~3) | ((q & 3) ^ ((q >> 3) & 3))];
    }
}

NB6_DEV void load_pv(const Pv *__restrict__ p, double *x, double *v, double &m) {
    const double2 *q = reinterpret_cast<const double2 *>(p);
    const double2 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2), d = __ldg(q + 3);
    x[0] = a.x;
    x[1] = a.y;
    x[2] = b.x;
    m = b.y;
    v[0] = c.x;
    v[1] = c.y;
    v[2] = d.x;
}

// irr_force_warp without a pair table, over the predicted set: the same
// pair terms in the same order per lane, so the same bits.
NB6_DEV void irr_force_warp_pv(int i, int lane, const Pv *__restrict__ pv, const int *__restrict__ lists, int ls,
                               int nmax, double *a, double *jd, int &nnbid) {
    double xi[3], vi[3], mi;
    load_pv(pv + i, xi, vi, mi);
    const int *row = lists + (size_t)i * ls;
    const int nnb = row[0];
    double ax = 0, ay = 0, az = 0, jx = 0, jy = 0, jz = 0;
    double rmin = 1.0e300;
    int jmin = 0x7fffffff;
    auto add = [&](const double *xj, const double *vj, double m, int j) {
        const double dxd = xj[0] - xi[0], dyd = xj[1] - xi[1], dzd = xj[2] - xi[2];
        const double r2d = dxd * dxd + dyd * dyd + dzd * dzd;
        if (r2d < rmin || (r2d == rmin && j < jmin)) {
            rmin = r2d;
            jmin = j;
        }
        const double dvx = vj[0] - vi[0], dvy = vj[1] - vi[1], dvz = vj[2] - vi[2];
        const double rinv = rsqrt(r2d);
        const double rinv2 = rinv * rinv;
        const double mr3 = m * rinv * rinv2;
        const double al = -3.0 * (dxd * dvx + dyd * dvy + dzd * dvz) * rinv2;
        ax += mr3 * dxd;
        ay += mr3 * dyd;
        az += mr3 * dzd;
        jx += mr3 * (dvx + al * dxd);
        jy += mr3 * (dvy + al * dyd);
        jz += mr3 * (dvz + al * dzd);
    };
    for (int l = lane; l < nnb; l += 32) {
        const int j = row[1 + l];
        if (j < 0 || j >= nmax) continue;   // ids are checked at set_list time
        double xj[3], vj[3], m;
        load_pv(pv + j, xj, vj, m);
        add(xj, vj, m, j);
    }
    irr_warp_finish(ax, ay, az, jx, jy, jz, rmin, jmin, nnb, a, jd, nnbid);
}

// out row k = (ax, ay, az, jx, jy, jz, nnbid, 0) (the correctors' rows),
// or, with out null, the caller's layout in fv: acc[ni][3] | jrk[ni][3]
// (doubles) | nnbid[ni] | nnb[ni] (ints), one download per call and plain
// block copies into the caller's arrays.
// KS: with the pair table (a separate instance: the corrections double the
// registers of the plain walk).  PV (no pair table): the walk over the
// predicted set pv instead of the records.
template <bool KS, bool PV = false>
__global__ void __launch_bounds__(IRR_WARPS * 32)
    irr_kernel(int ni, const int *__restrict__ addr, double ti, const Rec *__restrict__ rec,
               const Pv *__restrict__ pv, const int *__restrict__ lists, int ls, int nmax, KsArgs ks,
               double *__restrict__ out, double *__restrict__ fv) {
    static_assert(!(KS && PV), "the predicted-set walk has no pair table");
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int k = blockIdx.x * IRR_WARPS + warp;
    if (k >= ni) return;
    double a[3], jd[3];
    int id;
    if (PV)
        irr_force_warp_pv(addr[k] - 1, lane, pv, lists, ls, nmax, a, jd, id);
    else
        irr_force_warp<KS>(addr[k] - 1, lane, ti, rec, lists, ls, nmax, ks, a, jd, id);
    if (lane == 0 && !out) {
        // the caller's layout, in the blocks of the output staging:
        // acc[ni][3] | jrk[ni][3] (doubles) | nnbid[ni] | nnb[ni] (ints)
        double *oa = fv;
        int *oi = reinterpret_cast<int *>(oa + 6 * (size_t)ni);
        oa[3 * (size_t)k] = a[0];
        oa[3 * (size_t)k + 1] = a[1];
        oa[3 * (size_t)k + 2] = a[2];
        oa[3 * (size_t)ni + 3 * (size_t)k] = jd[0];
        oa[3 * (size_t)ni + 3 * (size_t)k + 1] = jd[1];
        oa[3 * (size_t)ni + 3 * (size_t)k + 2] = jd[2];
        oi[k] = id;
        oi[ni + k] = max(lists[(size_t)(addr[k] - 1) * ls], 0);
    }
    if (lane == 0 && out) {
        double *o = out + (size_t)k * 8;
        o[0] = a[0];
        o[1] = a[1];
        o[2] = a[2];
        o[3] = jd[0];
        o[4] = jd[1];
        o[5] = jd[2];
        o[6] = (double)id;
        o[7] = 0.0;
    }
}

// ----------------------------------------------------------------------------
// Device-resident irregular corrector (nb6_irr_correct_).  Beside each 128-byte
// record the device keeps an Aux record with the rest of a body's Hermite
// state; irr_kernel computes the neighbour force of each active body, then
// irr_apply_corrector applies the irregular corrector and the new irregular step of
// nbint_cor.f:113-173,215-236 (tstep.f), the regular-due test and the F/FDOT
// extrapolation of intgrt.F:570-578.  Every operation is rounded separately
// in the order of the host restatement (driver/hermite.h, Bodies::irr_correct),
// so device and host give the same bits.
// ----------------------------------------------------------------------------
struct Aux {  // 16 doubles
    double fi[3], fid[3], fr[3], frd[3], step, t0r, stepr, rs;
};

struct HermiteParams {
    double eta_i, smax, dtmin;
};

NB6_DEV double dadd(double a, double b) { return __dadd_rn(a, b); }
NB6_DEV double dmul(double a, double b) { return __dmul_rn(a, b); }
NB6_DEV double dsub(double a, double b) { return __dsub_rn(a, b); }
NB6_DEV double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// Constants of the reference's integrator (zero.f:113-116), multiplied as
// the Fortran multiplies them, and its REAL*4 literals (it is compiled
// without -fdefault-real-8, so 0.6 enters a REAL*8 product as 0.6f).
constexpr double ONE3 = 1.0 / 3.0, ONE6 = 1.0 / 6.0, ONE12 = 1.0 / 12.0;
#define R4(c) ((double)(c##f))

// tstep.f: sqrt(eta (|F||F2| + |F1|^2) / (|F1||F3| + |F2|^2))
NB6_DEV double tstep_dev(const double *f, const double *f1, const double *f2, const double *f3, double eta) {
    double F2 = 0, F12 = 0, F22 = 0, F32 = 0;
    for (int k = 0; k < 3; ++k) {
        F2 = dadd(F2, dmul(f[k], f[k]));
        F12 = dadd(F12, dmul(f1[k], f1[k]));
        F22 = dadd(F22, dmul(f2[k], f2[k]));
        F32 = dadd(F32, dmul(f3[k], f3[k]));
    }
    const double num = dadd(__dsqrt_rn(dmul(F2, F22)), F12);
    const double den = dadd(__dsqrt_rn(dmul(F12, F32)), F22);
    if (!(den > 0)) return 1e30;
    return __dsqrt_rn(ddiv(dmul(eta, num), den));
}

// Second launch of a corrector call, one thread per active body: the forces
// of every active body come from irr_kernel first (all neighbours seen as
// predicted from their old state, as on the host), then each body is
// corrected.  out row k (24 doubles): x0[3], v0[3], fi[3], fidot[3], F[3],
// FDOT[3], step, regular-due flag, nnbid, 0, 0, 0.
// The corrector of one body at `time` from its force row fk: its record r
// and corrector state x are updated in place and its out row o (24 doubles)
// written.  Returns the regular-due flag.
NB6_DEV bool correct_state(Rec &r, Aux &x, double time, const double *__restrict__ fk, const HermiteParams &hp,
                           double *__restrict__ o) {
    const double a[3] = {fk[0], fk[1], fk[2]}, jd[3] = {fk[3], fk[4], fk[5]};
    const int id = (int)fk[6];
    const double s = dsub(time, r.t0), s1 = dmul(1.5, s), s2 = dmul(2.0, s);
    double xi[3], vi[3];
    for (int c = 0; c < 3; ++c) {
        xi[c] = dadd(dmul(dadd(dmul(dadd(dmul(r.fd[c], s), r.f[c]), s), r.v[c]), s), r.x[c]);
        vi[c] = dadd(dmul(dadd(dmul(r.fd[c], s1), r.f[c]), s2), r.v[c]);
    }
    const double dt = s, dtsq = dmul(dt, dt), dt6 = ddiv(6.0, dmul(dt, dtsq)), dt2 = ddiv(2.0, dtsq);
    const double dtsq12 = dmul(ONE12, dtsq), dt13 = dmul(ONE3, dt);
    double ftot[3], d2[3], d3[3];
    for (int c = 0; c < 3; ++c) {  // nbint_cor.f:130-150
        const double df = dsub(x.fi[c], a[c]);
        const double fid = x.fid[c];
        const double sum = dadd(fid, jd[c]);
        const double at3 = dadd(dmul(2.0, df), dmul(dt, sum));
        const double bt2 = dsub(dmul(-3.0, df), dmul(dt, dadd(sum, fid)));
        r.x[c] = dadd(xi[c], dmul(dadd(dmul(R4(0.6), at3), bt2), dtsq12));
        r.v[c] = dadd(vi[c], dmul(dadd(dmul(0.75, at3), bt2), dt13));
        x.fi[c] = a[c];
        x.fid[c] = jd[c];
        ftot[c] = dadd(x.fi[c], x.fr[c]);
        d2[c] = dmul(dadd(dmul(3.0, at3), bt2), dt2);
        d3[c] = dmul(at3, dt6);
    }
    // irregular step (nbint_cor.f:146,215-236)
    double ttmp = tstep_dev(ftot, x.fid, d2, d3, hp.eta_i);
    const double dt0 = ttmp;
    if (ttmp > dmul(2.0, x.step)) {
        const double two = dmul(2.0, x.step);
        ttmp = (fmod(time, two) == 0.0) ? (hp.smax < two ? hp.smax : two) : x.step;
    } else if (ttmp < x.step) {
        ttmp = dmul(0.5, x.step);
        if (ttmp > dt0) ttmp = dmul(ttmp, 0.5);
    } else {
        ttmp = x.step;
    }
    x.step = ttmp < hp.dtmin ? hp.dtmin : ttmp;
    r.t0 = time;
    const bool regdue = dadd(x.t0r, x.stepr) <= time;
    if (!regdue) {
        const double dtr = dsub(time, x.t0r);
        for (int c = 0; c < 3; ++c) {
            r.f[c] = dmul(0.5, dadd(dadd(dmul(x.frd[c], dtr), x.fr[c]), x.fi[c]));
            r.fd[c] = dmul(ONE6, dadd(x.frd[c], x.fid[c]));
        }
        // keep the irregular step inside the regular interval
        while (dadd(r.t0, x.step) > dadd(x.t0r, x.stepr) && x.step > hp.dtmin) x.step = dmul(x.step, 0.5);
    }
    for (int c = 0; c < 3; ++c) {
        o[c] = r.x[c];
        o[3 + c] = r.v[c];
        o[6 + c] = x.fi[c];
        o[9 + c] = x.fid[c];
        o[12 + c] = r.f[c];
        o[15 + c] = r.fd[c];
    }
    o[18] = x.step;
    o[19] = regdue ? 1.0 : 0.0;
    o[20] = (double)id;
    o[21] = o[22] = o[23] = 0.0;
    return regdue;
}

// The corrector of body i (0-based) in place, with out row o; tn[i] = t0 +
// step, the body's next block time, is kept for the device block clock.
NB6_DEV bool correct_irr_body(int i, double time, const double *__restrict__ fk, Rec *__restrict__ rec,
                              Aux *__restrict__ aux, const HermiteParams &hp, double *__restrict__ o,
                              double *__restrict__ tn) {
    Rec r = rec[i];
    Aux x = aux[i];
    const bool regdue = correct_state(r, x, time, fk, hp, o);
    rec[i] = r;
    aux[i] = x;
    tn[i] = dadd(r.t0, x.step);
    return regdue;
}

__global__ void irr_apply_corrector(int ni, const int *__restrict__ addr, double time,
                                    const double *__restrict__ force, Rec *__restrict__ rec,
                                    Aux *__restrict__ aux, HermiteParams hp, double *__restrict__ out,
                                    double *__restrict__ tn) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ni) return;
    correct_irr_body(addr[k] - 1, time, force + (size_t)k * 8, rec, aux, hp, out + (size_t)k * 24, tn);
}

// ----------------------------------------------------------------------------
// Device-resident regular corrector (nb6_regf_correct_): the host's
// Bodies::reg_correct (regcor_gpu.F:131-196 radius update, :284-444
// neighbour gain/loss force moves, :442-537 corrector, :593-737 new regular
// step) for every body of a segmented regular-force call whose list did not
// overflow, one thread per body, every operation rounded as on the host.
// Neighbours are taken from the predicted j set of the call (the state of
// every body at the block time before any regular correction -- the host's
// snapshot), the old list from the resident list rows, the new one from the
// call's output rows.
// ----------------------------------------------------------------------------
struct RegCorrParams {
    double eta_r, smax, dtmin, rsfac;
    int nnbopt, nnbmax, cap, mlp_mode;
    int nb_flag, m_flag;
    // radius-rule quantities per cluster (nb6_hermite_adjust_): cluster c
    // holds bodies [acl_a0[c], acl_a0[c+1]) (0-based), acpar[8c..] = RDENS[3],
    // RSCALE, RC2, RSFAC, BODYM; nacl = 0: none set
    int nacl;
    const int *acl_a0;
    const double *acpar;
};

// Radius-rule quantities of one cluster (as Bodies::adjust sets them).
struct ACParDev {
    double rdens[3], rscale, rc2, rsfac, bodym;
};

// Ahmad-Cohen radius update of one body at its regular step
// (regcor_gpu.F:19-238), the host's ac_radius (driver/hermite.h) operation
// for operation: REAL*4 terms of the reference (FLOAT(), literals) in float,
// the rest in double, every operation rounded separately.  xnb/vnb: the
// first min(nnb, 3) new neighbours at TIME.  dfirr/dfd: the irregular force
// change the neighbour moves start from (the small central mass, nnb = 0).
NB6_DEV double ac_radius_dev(int nb_flag, int m_flag, int nnbopt, int nnbmax, const ACParDev &a, int nnb,
                             int nnb0, double dtr, const double *xi, const double *vi, const double *xnb,
                             const double *vnb, double rs, double *dfirr, double *dfd) {
    const float zs = __fmul_rn(0.01f, (float)nnbmax);
    const double znbmin = (double)(zs > 1.0f ? zs : 1.0f);
    for (int k = 0; k < 3; ++k) dfirr[k] = dfd[k] = 0.0;
    double ri2, rh2;
    if (nb_flag) {
        const double e0 = dsub(xi[0], a.rdens[0]), e1 = dsub(xi[1], a.rdens[1]), e2 = dsub(xi[2], a.rdens[2]);
        ri2 = dadd(dadd(dmul(e0, e0), dmul(e1, e1)), dmul(e2, e2));
        rh2 = dmul(a.rscale, a.rscale);
    } else {
        ri2 = dadd(dadd(dmul(xi[0], xi[0]), dmul(xi[1], xi[1])), dmul(xi[2], xi[2]));
        rh2 = dmul(R4(9.0), dmul(a.rscale, a.rscale));
    }
    if (nnb == 0) {
        const double r2 = dadd(dadd(dmul(xi[0], xi[0]), dmul(xi[1], xi[1])), dmul(xi[2], xi[2]));
        const double fij = ddiv(dmul(R4(0.01), a.bodym), dmul(r2, __dsqrt_rn(r2)));
        const double rdot =
            ddiv(dmul(3.0, dadd(dadd(dmul(xi[0], vi[0]), dmul(xi[1], vi[1])), dmul(xi[2], vi[2]))), r2);
        for (int k = 0; k < 3; ++k) {
            dfirr[k] = dmul(-fij, xi[k]);
            dfd[k] = dmul(-dsub(vi[k], dmul(rdot, xi[k])), fij);
        }
        if (rdot > 0.0) {
            const double u = dmul(R4(0.75), rs), w = dmul(R4(0.1), a.rscale);
            return u > w ? u : w;
        }
        return dmul(R4(1.1), rs);
    }
    const float fac_s =
        __fadd_rn(1.0f, __fdiv_rn(__fmul_rn(0.1f, __fsub_rn((float)nnbopt, (float)nnb)), (float)nnb));
    double a3 = dmul((double)(float)nnb, (double)fac_s);
    const int zi = (int)znbmin;
    const int nbave = min(nnbopt + 150, max(nnbmax - 50, zi));
    const double cap = (double)__fmul_rn(0.9f, (float)nbave);
    a3 = a3 < cap ? a3 : cap;
    const int nbp = (int)a3;
    if (ri2 > rh2 && nb_flag) {
        const double f = ddiv(a.rscale, __dsqrt_rn(ri2));
        a3 = dmul(a3, f > R4(0.1) ? f : R4(0.1));
    } else {
        a3 = a3 > znbmin ? a3 : znbmin;
    }
    double a4 = ddiv(a3, (double)(float)nnb);
    if (dmul(dsub(a3, (double)(float)nnb0), dsub(a3, (double)(float)nnb)) < 0.0) a4 = __dsqrt_rn(a4);
    const double ridot = dadd(dadd(dmul(dsub(xi[0], a.rdens[0]), vi[0]), dmul(dsub(xi[1], a.rdens[1]), vi[1])),
                              dmul(dsub(xi[2], a.rdens[2]), vi[2]));
    if (ri2 > a.rc2 && nb_flag && ri2 < dmul(R4(100.0), rh2)) a4 = dmul(a4, dadd(1.0, ddiv(dmul(ridot, dtr), ri2)));
    double a5 = dmul(a.rsfac, dtr);
    a5 = a5 < 0.25 ? a5 : 0.25;
    a4 = dsub(a4, 1.0);
    if (a4 > a5) a4 = a5;
    else a4 = a4 > -a5 ? a4 : -a5;
    const double a3b = dmul(ONE3, a4);
    double a1 = dsub(dadd(1.0, a3b), dmul(a3b, a3b));
    if (nnb < znbmin && nbp > znbmin && a1 < 1.0) a1 = R4(1.05);
    if (fabs(dsub(a1, 1.0)) > R4(0.003)) {
        const double rs2 = dmul(rs, rs);
        if (rs2 > ri2 && rs2 < dmul(2.0, ri2) && nnb > 5) a1 = __dsqrt_rn(a1);
        rs = dmul(a1, rs);
    }
    if (nnb > nbave && ridot < 0.0) {
        const float drs = __fdiv_rn(__fsub_rn((float)nnb, (float)nbave), __fmul_rn(3.0f, (float)nnb));
        rs = dmul(rs, dsub(1.0, (double)drs));
    }
    if (!m_flag && nnb <= 3 && ri2 < dmul(R4(100.0), rh2)) {
        double b1 = dmul(2.0, rs);
        for (int l = 0; l < nnb; ++l) {
            const double *xj = xnb + 3 * l, *vj = vnb + 3 * l;
            const double e0 = dsub(xi[0], xj[0]), e1 = dsub(xi[1], xj[1]), e2 = dsub(xi[2], xj[2]);
            const double rij = __dsqrt_rn(dadd(dadd(dmul(e0, e0), dmul(e1, e1)), dmul(e2, e2)));
            const double rsdot = ddiv(dadd(dadd(dmul(e0, dsub(vi[0], vj[0])), dmul(e1, dsub(vi[1], vj[1]))),
                                           dmul(e2, dsub(vi[2], vj[2]))),
                                      rij);
            const double t = dadd(rij, dmul(rsdot, dtr));
            b1 = b1 < t ? b1 : t;
        }
        const double g = dmul(R4(1.1), rs);
        rs = b1 > g ? b1 : g;
    }
    return rs;
}

// host Bodies::pair_force: FP64 force and jerk of j (at xj, vj, mass mj) on i
NB6_DEV void pair_force_dev(const double *xi, const double *vi, const double *xj, const double *vj, double mj,
                            double *a, double *jd) {
    const double dx = dsub(xj[0], xi[0]), dy = dsub(xj[1], xi[1]), dz = dsub(xj[2], xi[2]);
    const double dvx = dsub(vj[0], vi[0]), dvy = dsub(vj[1], vi[1]), dvz = dsub(vj[2], vi[2]);
    const double r2 = dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz));
    const double dr2i = ddiv(1.0, r2), dr3i = dmul(dmul(mj, dr2i), __dsqrt_rn(dr2i));
    const double drdp = dmul(dmul(3.0, dadd(dadd(dmul(dx, dvx), dmul(dy, dvy)), dmul(dz, dvz))), dr2i);
    a[0] = dmul(dx, dr3i);
    a[1] = dmul(dy, dr3i);
    a[2] = dmul(dz, dr3i);
    jd[0] = dmul(dsub(dvx, dmul(dx, drdp)), dr3i);
    jd[1] = dmul(dsub(dvy, dmul(dy, drdp)), dr3i);
    jd[2] = dmul(dsub(dvz, dmul(dz, drdp)), dr3i);
}

// out row k (32 doubles): x0[3], v0[3], fi[3], fidot[3], fr[3], frdot[3],
// F[3], FDOT[3], step, stepr, rs, nnb (self removed), overflow (-nnb of an
// overflowed row, else 0), learned-radius outcome (0 off, 1 taken, 2
// fallback), 0, 0.
__global__ void reg_corrector_kernel(int ni, const int *__restrict__ addr, const int *__restrict__ iseg,
                                     const int *__restrict__ seg_j0, const int *__restrict__ seg_a0, double time,
                                     RegDeviceOut ro, Rec *__restrict__ rec, Aux *__restrict__ aux,
                                     int *__restrict__ lists, int ls, const double *__restrict__ rs_in,
                                     RegCorrParams p, double *__restrict__ out, int *status,
                                     double *__restrict__ tn) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ni) return;
    const int i = addr[k] - 1, sg = iseg[k];
    const double *of = ro.outf + (size_t)k * 8;
    const int *ol = ro.outl + (size_t)k * ro.W;
    double *o = out + (size_t)k * 32;
    for (int c = 0; c < 32; ++c) o[c] = 0.0;
    const int raw = ol[0];
    if (raw < 0 || raw > p.cap) {  // overflow: the host shrinks RS and asks again
        o[28] = (double)(raw < 0 ? raw : -raw);
        return;
    }
    const int base = seg_a0[sg], jb = seg_j0[sg], nj = seg_j0[sg + 1] - jb;
    Rec r = rec[i];
    Aux x = aux[i];
    int *orow = lists + (size_t)i * ls;
    const int nnb0 = min(max(orow[0], 0), ls - 1);
    int self_in = 0;  // i itself is in the call's list when it belongs to the segment
    for (int l = 1; l <= raw; ++l)
        if (base + ol[l] == i) self_in = 1;
    const int nnb = raw - self_in;
    const double dtr = dsub(time, x.t0r);
    const double xi[3] = {r.x[0], r.x[1], r.x[2]}, vi[3] = {r.v[0], r.v[1], r.v[2]};
    double rs = rs_in[k];  // the radius the call's h2 was formed from
    const double rs_used = rs;
    // the body's cluster and its radius-rule quantities
    ACParDev ap;
    if (p.nacl > 0) {
        int lo = 0, hi = p.nacl - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (p.acl_a0[mid] <= i) lo = mid;
            else hi = mid - 1;
        }
        const double *q = p.acpar + 8 * (size_t)lo;
        ap = {{q[0], q[1], q[2]}, q[3], q[4], q[5], q[6]};
    } else {
        ap = {{0.0, 0.0, 0.0}, 1.0, 1.0, p.rsfac, ddiv(1.0, (double)nj)};
    }
    // Ahmad-Cohen radius update (regcor_gpu.F:19-238) from the first
    // min(nnb, 3) new neighbours of the call's j set
    double xnb[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, vnb[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    {
        int l3 = 0;
        for (int l = 1; l <= raw && l3 < 3; ++l) {
            if (base + ol[l] == i) continue;
            const size_t q = (size_t)(jb + ol[l]);
            for (int c = 0; c < 3; ++c) {
                xnb[3 * l3 + c] = ro.jx[3 * q + c];
                vnb[3 * l3 + c] = ro.jv[3 * q + c];
            }
            ++l3;
        }
    }
    double dfirr[3], dfd[3];
    rs = ac_radius_dev(p.nb_flag, p.m_flag, p.nnbopt, p.nnbmax, ap, nnb, nnb0, dtr, xi, vi, xnb, vnb, rs, dfirr,
                       dfd);
    // neighbour gains and losses (regcor_gpu.F:284-444); ids are 0-based
    // global addresses, the new list's are relative to the segment
    int a = 1, b = 1;
    auto next_new = [&](int &bb) {  // skip self in the new list
        while (bb <= raw && base + ol[bb] == i) ++bb;
    };
    next_new(b);
    while (a <= nnb0 || b <= raw) {
        const int jo = a <= nnb0 ? orow[a] : 0x7fffffff;
        const int jn = b <= raw ? base + ol[b] : 0x7fffffff;
        if (jo == jn) {
            ++a;
            ++b;
            next_new(b);
            continue;
        }
        const int j = jo < jn ? jo : jn;
        if (j < base || j - base >= nj) {  // a neighbour outside the body's segment
            set_status(status, NB6_ERR_BAD_ARG);
            return;
        }
        const size_t q = (size_t)(jb + (j - base));
        const double xj[3] = {ro.jx[3 * q], ro.jx[3 * q + 1], ro.jx[3 * q + 2]};
        const double vj[3] = {ro.jv[3 * q], ro.jv[3 * q + 1], ro.jv[3 * q + 2]};
        double fa[3], fj[3];
        pair_force_dev(xi, vi, xj, vj, ro.jm[q], fa, fj);
        if (jo < jn) {  // lost
            for (int c = 0; c < 3; ++c) {
                dfirr[c] = dsub(dfirr[c], fa[c]);
                dfd[c] = dsub(dfd[c], fj[c]);
            }
            ++a;
        } else {  // gained
            for (int c = 0; c < 3; ++c) {
                dfirr[c] = dadd(dfirr[c], fa[c]);
                dfd[c] = dadd(dfd[c], fj[c]);
            }
            ++b;
            next_new(b);
        }
    }
    // regular corrector (regcor_gpu.F:442-537)
    const double dtsq = dmul(dtr, dtr), dt6 = ddiv(6.0, dmul(dtr, dtsq)), dt2 = ddiv(2.0, dtsq);
    const double dtsq12 = dmul(ONE12, dtsq), dtr13 = dmul(ONE3, dtr);
    double d2r[3], d3r[3];
    for (int c = 0; c < 3; ++c) {
        const double dfr = dsub(dsub(x.fr[c], of[c]), dfirr[c]);
        const double fdr0 = dadd(of[3 + c], dfd[c]);
        const double frd = x.frd[c];
        const double sum = dadd(frd, fdr0);
        const double at3 = dadd(dmul(2.0, dfr), dmul(dtr, sum));
        const double bt2 = dsub(dmul(-3.0, dfr), dmul(dtr, dadd(sum, frd)));
        r.x[c] = dadd(r.x[c], dmul(dadd(dmul(R4(0.6), at3), bt2), dtsq12));
        r.v[c] = dadd(r.v[c], dmul(dadd(dmul(0.75, at3), bt2), dtr13));
        x.fi[c] = dadd(x.fi[c], dfirr[c]);
        x.fr[c] = of[c];
        x.fid[c] = dadd(x.fid[c], dfd[c]);
        x.frd[c] = of[3 + c];
        d3r[c] = dmul(at3, dt6);
        d2r[c] = dmul(dadd(dmul(3.0, at3), bt2), dt2);
    }
    // the new list into the resident rows (after the merge has read the old)
    int w = 1;
    for (int l = 1; l <= raw; ++l)
        if (base + ol[l] != i) orow[w++] = base + ol[l];
    orow[0] = nnb;
    // new regular step (regcor_gpu.F:593-737)
    double ttmp = tstep_dev(x.fr, x.frd, d2r, d3r, p.eta_r);
    const double dt0 = ttmp;
    if (ttmp > dmul(2.0, x.stepr)) {
        const double two = dmul(2.0, dtr);
        ttmp = (fmod(time, two) == 0.0) ? (p.smax < two ? p.smax : two) : x.stepr;
    } else if (ttmp < dtr) {
        ttmp = dmul(0.5, dtr);
        if (ttmp > dt0) ttmp = dmul(ttmp, 0.5);
    } else {
        ttmp = x.stepr;
    }
    ttmp = (p.smax < ttmp) ? p.smax : ttmp;
    ttmp = (ttmp < p.dtmin) ? p.dtmin : ttmp;
    x.stepr = ttmp;
    x.t0r = time;
    for (int c = 0; c < 3; ++c) {
        r.f[c] = dmul(0.5, dadd(x.fi[c], x.fr[c]));
        r.fd[c] = dmul(ONE6, dadd(x.fid[c], x.frd[c]));
    }
    if (x.step > x.stepr) x.step = x.stepr;
    // learned radius (Bodies::learn_apply): take RS_used exp(dlog) when the
    // count it implies stays in [NNBOPT/2, NNBMAX]
    double outcome = 0.0;
    if (p.mlp_mode == 2) {
        const double lim = 0.69314718055994531;
        double dl = of[7];
        dl = dl > lim ? lim : (dl < -lim ? -lim : dl);
        const double expect = dmul((double)nnb, exp(dmul(3.0, dl)));
        if (nnb > 0 && dl == dl && expect >= dmul(0.5, (double)p.nnbopt) && expect <= (double)p.nnbmax) {
            rs = dmul(rs_used, exp(dl));
            outcome = 1.0;
        } else {
            outcome = 2.0;
        }
    }
    x.rs = rs;
    rec[i] = r;
    aux[i] = x;
    tn[i] = dadd(r.t0, x.step);
    for (int c = 0; c < 3; ++c) {
        o[c] = r.x[c];
        o[3 + c] = r.v[c];
        o[6 + c] = x.fi[c];
        o[9 + c] = x.fid[c];
        o[12 + c] = x.fr[c];
        o[15 + c] = x.frd[c];
        o[18 + c] = r.f[c];
        o[21 + c] = r.fd[c];
    }
    o[24] = x.step;
    o[25] = x.stepr;
    o[26] = rs;
    o[27] = (double)nnb;
    o[29] = outcome;
}

// ----------------------------------------------------------------------------
// Device block clock (nb6_blocks_run_): blocks of irregular steps run back to
// back on the device, each as two launches of one CUDA graph --
//   blk_collect  first the new records of the block before (see blk_step),
//                then the active set {i : tn_i == block time} (next_tlist.f
//                picks the same set from its level lists), or a stop when the
//                block time passes the caller's limit; also the earliest tn
//                of the other bodies, which this block leaves as they are;
//   blk_step     one warp per active body: its neighbour force
//                (irr_force_warp), then on lane 0 its irregular corrector
//                (correct_state, as nb6_irr_correct_ does), with the body's
//                new aux and tn written in place and its new record kept in
//                its corrector row until the next blk_collect -- other warps
//                of this block still read the old record of i as a
//                neighbour, predicted from its old state, as the host does;
//                then, in the last CTA to finish, the block's bookkeeping,
//                the next block time (the earlier of the others' earliest tn
//                and the block's new ones) and a stop when a body is due a
//                regular step (the host runs the regular part).
// The first block time of a run is the minimum over every body (blk_min,
// launched once per run); blk_flush writes the last block's records when a
// run ends.  A stopped control block turns every later launch into an early
// return, so the host enqueues many blocks and synchronises once.  No
// kernel waits on another: the ordering is the stream's, the last-CTA test
// is one atomic.
// ----------------------------------------------------------------------------
struct BlockCtl {
    unsigned long long tmin_bits[2];  // per parity: the block time, min tn (bits of a non-negative double)
    unsigned long long m2_bits[2];    // per parity: min tn over the bodies not in the block
    unsigned long long mact_bits[2];  // per parity: min of the block's new tn
    int nact[2];                      // per parity: active count
    int parity;
    int stop;                         // 0 run; 1 a regular-due block's irregular part is done; 2 block time > tlimit;
                                      // 3 the run's block limit reached
    int regdue;                       // the running block has a regular-due body
    unsigned cta_done;                // blk_step CTAs finished (last-CTA test)
    long long blocks, irr_steps;      // since the last reset by the host
    double tlimit, tblock;            // run limit; time of the last block done
    int last_nact;
    int nreg;                         // regular-due bodies of the running block (breg, bregxv)
    long long blimit;                 // blocks this run may do (stop 3 when reached)
    // persistent form (blk_persist): grid barrier, and the act[] half that
    // holds the last block's active set
    unsigned bar_count, bar_gen;
    int last_parity;
    // graph form: the block whose new records blk_collect still has to write
    // (its active count, act[] half and time; pend_na = 0: none)
    int pend_na, pend_parity;
    double pend_t;
};

constexpr int BLK_NT = 256;

// Programmatic dependent launch (the block kernels are captured with
// programmatic edges, so each may be scheduled while the one before it
// drains).  griddepcontrol.wait returns once the kernels this one depends
// on have completed and their memory is visible -- the guarantee of a
// kernel boundary -- so every block kernel calls it before its first
// access to the control block or to data an earlier kernel wrote, and then
// lets its own dependants be scheduled.  Both are no-ops for a launch
// without a programmatic dependency.
NB6_DEV void blk_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Minimum over the CTA (BLK_NT threads), valid in thread 0; every thread
// must call it.
template <int NT = BLK_NT>
NB6_DEV unsigned long long cta_min(unsigned long long m) {
    __shared__ unsigned long long wm[NT / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = min(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0)
        for (int w = 1; w < NT / 32; ++w) m = min(m, wm[w]);
    __syncthreads();
    return m;
}

__global__ void __launch_bounds__(BLK_NT) blk_min(int n, const double *__restrict__ tn, BlockCtl *c) {
    blk_enter();
    if (c->stop) return;
    const int p = c->parity;
    unsigned long long m = ~0ull;
    for (size_t i = blockIdx.x * (size_t)BLK_NT + threadIdx.x; i < (size_t)n; i += (size_t)gridDim.x * BLK_NT)
        m = min(m, (unsigned long long)__double_as_longlong(tn[i]));
    m = cta_min(m);
    if (threadIdx.x == 0) atomicMin(&c->tmin_bits[p], m);
}

// The new records of the block before (x0, v0, F, FDOT from its corrector
// rows, t0 = its time); act holds both halves.
NB6_DEV void blk_scatter_pending(const BlockCtl *c, const int *__restrict__ act, int n,
                                 const double *__restrict__ rows, Rec *__restrict__ rec) {
    const int na = c->pend_na;
    if (na <= 0) return;
    const int *ap = act + (size_t)c->pend_parity * n;
    const double t = c->pend_t;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < na; k += gridDim.x * blockDim.x) {
        const double *o = rows + (size_t)k * 24;
        Rec *r = rec + ap[k];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            r->x[d] = o[d];
            r->v[d] = o[3 + d];
            r->f[d] = o[12 + d];
            r->fd[d] = o[15 + d];
        }
        r->t0 = t;
    }
}

__global__ void __launch_bounds__(BLK_NT) blk_collect(int n, const double *__restrict__ tn, BlockCtl *c,
                                                      int *__restrict__ act, const double *__restrict__ rows,
                                                      Rec *__restrict__ rec) {
    blk_enter();
    blk_scatter_pending(c, act, n, rows, rec);
    if (c->stop) return;
    if (c->blocks >= c->blimit) {  // every thread reads the same count: all return
        if (blockIdx.x == 0 && threadIdx.x == 0) c->stop = 3;
        return;
    }
    const int p = c->parity;
    const double t = __longlong_as_double((long long)c->tmin_bits[p]);
    if (t > c->tlimit) {  // every thread reads the same t: all return
        if (blockIdx.x == 0 && threadIdx.x == 0) c->stop = 2;
        return;
    }
    const int lane = threadIdx.x & 31;
    act += (size_t)c->parity * n;   // this block's half
    unsigned long long m2 = ~0ull;  // the others' earliest time (they keep it through this block)
    // the next times are loaded U per thread at once, all in flight together
    // (one pass for up to U x grid threads bodies), then tested
    constexpr int U = 8;
    const size_t nt = (size_t)gridDim.x * BLK_NT;
    for (size_t i0 = blockIdx.x * (size_t)BLK_NT; i0 < (size_t)n; i0 += U * nt) {
        double tv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const size_t i = i0 + u * nt + threadIdx.x;
            tv[u] = i < (size_t)n ? tn[i] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const size_t i = i0 + u * nt + threadIdx.x;
            const bool on = i < (size_t)n && tv[u] == t;
            if (i < (size_t)n && !on) m2 = min(m2, (unsigned long long)__double_as_longlong(tv[u]));
            const unsigned b = __ballot_sync(0xffffffffu, on);
            if (b) {
                int base = 0;
                if (lane == 0) base = atomicAdd(&c->nact[p], __popc(b));
                base = __shfl_sync(0xffffffffu, base, 0);
                if (on) act[base + __popc(b & ((1u << lane) - 1u))] = (int)i;
            }
        }
    }
    m2 = cta_min(m2);  // one atomic per CTA (not per warp: they would queue on one address)
    if (threadIdx.x == 0) {
        atomicMin(&c->m2_bits[p], m2);
        if (blockIdx.x == 0) c->nreg = 0;  // this block's due list
    }
}

template <bool KS>
__global__ void __launch_bounds__(IRR_WARPS * 32)
    blk_step(BlockCtl *c, const int *__restrict__ act, int n, const Rec *__restrict__ rec, Aux *__restrict__ aux,
             const int *__restrict__ lists, int ls, KsArgs ks, HermiteParams hp, double *__restrict__ rows,
             double *__restrict__ tn, int *__restrict__ reg, double *__restrict__ regxv) {
    blk_enter();
    if (blockIdx.x == 0 && threadIdx.x == 0) c->pend_na = 0;   // blk_collect has written them
    if (c->stop) return;
    const int p = c->parity, na = c->nact[p];
    const double t = __longlong_as_double((long long)c->tmin_bits[p]);
    const int *ap = act + (size_t)p * n;
    const int lane = threadIdx.x & 31;
    bool due = false;
    unsigned long long mact = ~0ull;  // earliest new tn of this CTA's bodies
    for (int k = blockIdx.x * IRR_WARPS + (threadIdx.x >> 5); k < na; k += gridDim.x * IRR_WARPS) {
        const int i = ap[k];
        double fk[8];
        int id;
        irr_force_warp<KS, false, !KS>(i, lane, t, rec, lists, ls, n, ks, fk, fk + 3, id);
        if (lane == 0) {
            fk[6] = (double)id;
            fk[7] = 0.0;
            Rec r = rec[i];
            Aux x = aux[i];
            double *o = rows + (size_t)k * 24;
            if (correct_state(r, x, t, fk, hp, o)) {
                due = true;
                const int q = atomicAdd(&c->nreg, 1);  // (q < na <= n)
                reg[q] = i;
                for (int d = 0; d < 6; ++d) regxv[6 * (size_t)q + d] = o[d];  // x0, v0
            }
            aux[i] = x;
            const double tnew = dadd(r.t0, x.step);
            tn[i] = tnew;
            mact = min(mact, (unsigned long long)__double_as_longlong(tnew));
        }
    }
    mact = cta_min<IRR_WARPS * 32>(mact);
    if (threadIdx.x == 0) atomicMin(&c->mact_bits[p], mact);
    if (__syncthreads_or(due) && threadIdx.x == 0) atomicOr(&c->regdue, 1);
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&c->cta_done, 1u) == gridDim.x - 1) {  // last CTA: the block is done
            __threadfence();
            const int q = p ^ 1;
            c->cta_done = 0;
            c->blocks += 1;
            c->irr_steps += na;
            c->tblock = t;
            c->last_nact = na;
            c->last_parity = p;
            c->pend_na = na;
            c->pend_parity = p;
            c->pend_t = t;
            // the next block's time: the earliest of the bodies outside this
            // block (unchanged by it) and of this block's new times
            c->tmin_bits[q] = min(atomicAdd(&c->m2_bits[p], 0ull), atomicAdd(&c->mact_bits[p], 0ull));
            c->m2_bits[q] = ~0ull;
            c->mact_bits[q] = ~0ull;
            c->nact[q] = 0;
            c->parity = q;
            if (atomicExch(&c->regdue, 0)) c->stop = 1;
        }
    }
}

// The last block's new records, when a run ends.
__global__ void blk_flush(BlockCtl *c, const int *__restrict__ act, int n, const double *__restrict__ rows,
                          Rec *__restrict__ rec) {
    blk_scatter_pending(c, act, n, rows, rec);
}

// ----------------------------------------------------------------------------
// Persistent block clock (blk_persist): the same blocks, one cooperative
// launch for a whole run of them.  Each block is two phases separated by
// grid-wide barriers:
//   A  the previous block's new records go into rec[] (see B), then the
//      active set and the earliest tn of the others, as blk_collect;
//   B  one warp per active body: its neighbour force (irr_force_warp), then
//      on lane 0 its corrector (correct_state), with the new aux[i] and
//      tn[i] written in place and the new record kept in the body's out
//      row until phase A of the next block -- other warps of this block
//      still read the old record of i as a neighbour, predicted from its
//      old state, exactly as in the graph form's blk_step.
// The last CTA at the barrier after B does blk_step's bookkeeping.  Data
// written by other CTAs of the launch (records, tn, aux, the active set,
// out rows) is read through L2 only (ld.global.cg), after the barrier's
// fences.  The active set alternates between two halves of act[] (phase A
// reads the previous block's half while it writes the next one).
// Results are those of the graph form, bit for bit.
// ----------------------------------------------------------------------------
#ifndef PB_THREADS
#define PB_THREADS 256
#endif
constexpr int PB_NT = PB_THREADS;                         // threads per CTA, one CTA per SM
constexpr unsigned long long PB_WAIT_NS = 4000000000ull;  // barrier wait limit, 4 s

NB6_DEV unsigned atom_add_acq_rel(unsigned *p, unsigned v) {
    unsigned old;
    asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
NB6_DEV unsigned ld_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
NB6_DEV void st_release(unsigned *p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Grid-wide barrier (every CTA resident: cooperative launch).  Thread 0 of
// each CTA arrives with one acquire-release atomic (its CTA's writes, ordered
// before it by the CTA barrier, are released with it); the last to arrive
// has acquired every other CTA's writes, runs last() and opens the barrier
// with a release store of the next generation; the others poll the
// generation with acquire loads for at most PB_WAIT_NS of global time,
// after which they set the status word and report false (in every thread
// of the CTA).
template <class F>
NB6_DEV bool grid_sync(BlockCtl *c, int *status, F last) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int good = 1;
        const unsigned g = ld_acquire(&c->bar_gen);
        if (atom_add_acq_rel(&c->bar_count, 1u) == gridDim.x - 1) {
            last();
            c->bar_count = 0;
            st_release(&c->bar_gen, g + 1);
        } else {
            const unsigned long long t0 = globaltimer();
            while (ld_acquire(&c->bar_gen) == g) {
                if (globaltimer() - t0 > PB_WAIT_NS) {
                    set_status(status, NB6_ERR_WAIT_TIMEOUT);
                    good = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

NB6_DEV void ldcg_aux(const Aux *p, Aux &x) {
    const double2 *q = reinterpret_cast<const double2 *>(p);
    double *d = reinterpret_cast<double *>(&x);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const double2 v = __ldcg(q + k);
        d[2 * k] = v.x;
        d[2 * k + 1] = v.y;
    }
}

// NT threads per CTA, one CTA per SM (the corrected walk of the KS form
// needs 186 registers: 256 threads).
template <bool KS, int NT = KS ? 256 : PB_NT>
__global__ void __launch_bounds__(NT, 1)
    blk_persist(BlockCtl *c, int *__restrict__ act, int n, Rec *__restrict__ rec, Aux *__restrict__ aux,
                const int *__restrict__ lists, int ls, KsArgs ks, HermiteParams hp, double *__restrict__ rows,
                double *__restrict__ tn, int *__restrict__ reg, double *__restrict__ regxv, int *status) {
    volatile BlockCtl *cv = c;
    const int lane = threadIdx.x & 31;
    const int gw = blockIdx.x * (NT / 32) + (threadIdx.x >> 5), nw = gridDim.x * (NT / 32);
    const int gt = blockIdx.x * NT + threadIdx.x, nt = gridDim.x * NT;
    int prev_na = 0, prev_p = 0;
    double prev_t = 0.0;
    for (;;) {
        // ---- phase A
        for (int k = gt; k < prev_na; k += nt) {   // the previous block's new records
            const int i = __ldcg(act + (size_t)prev_p * n + k);
            const double *o = rows + (size_t)k * 24;
            Rec *r = rec + i;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                r->x[d] = __ldcg(o + d);
                r->v[d] = __ldcg(o + 3 + d);
                r->f[d] = __ldcg(o + 12 + d);
                r->fd[d] = __ldcg(o + 15 + d);
            }
            r->t0 = prev_t;
        }
        if (cv->stop) return;
        if (cv->blocks >= cv->blimit) {   // every thread reads the same count: all return
            if (blockIdx.x == 0 && threadIdx.x == 0) c->stop = 3;
            return;
        }
        const int p = cv->parity;
        const double t = __longlong_as_double((long long)cv->tmin_bits[p]);
        if (t > cv->tlimit) {
            if (blockIdx.x == 0 && threadIdx.x == 0) c->stop = 2;
            return;
        }
        int *ap = act + (size_t)p * n;
        unsigned long long m2 = ~0ull;
        constexpr int U = 8;   // next times loaded U at a time, all in flight together
        for (int i0 = gt; i0 - (int)threadIdx.x < n; i0 += U * nt) {
            double tv[U];
#pragma unroll
            for (int u = 0; u < U; ++u) tv[u] = i0 + u * nt < n ? __ldcg(tn + i0 + u * nt) : 0.0;
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int i = i0 + u * nt;
                const bool on = i < n && tv[u] == t;
                if (i < n && !on) m2 = min(m2, (unsigned long long)__double_as_longlong(tv[u]));
                const unsigned b = __ballot_sync(0xffffffffu, on);
                if (b) {
                    int base = 0;
                    if (lane == 0) base = atomicAdd(&c->nact[p], __popc(b));
                    base = __shfl_sync(0xffffffffu, base, 0);
                    if (on) ap[base + __popc(b & ((1u << lane) - 1u))] = i;
                }
            }
        }
        m2 = cta_min<NT>(m2);
        if (threadIdx.x == 0) atomicMin(&c->m2_bits[p], m2);
        if (blockIdx.x == 0 && threadIdx.x == 0) c->nreg = 0;
        if (!grid_sync(c, status, [] {})) return;
        // ---- phase B
        const int na = cv->nact[p];
        bool due = false;
        unsigned long long mact = ~0ull;
        for (int k = gw; k < na; k += nw) {
            const int i = __ldcg(ap + k);
            double fk[8];
            int id;
            irr_force_warp<KS, true>(i, lane, t, rec, lists, ls, n, ks, fk, fk + 3, id);
            if (lane == 0) {
                fk[6] = (double)id;
                fk[7] = 0.0;
                Rec r;
                Aux x;
                load_rec<true>(rec + i, r);
                ldcg_aux(aux + i, x);
                double *o = rows + (size_t)k * 24;
                if (correct_state(r, x, t, fk, hp, o)) {
                    due = true;
                    const int q = atomicAdd(&c->nreg, 1);  // (q < na <= n)
                    reg[q] = i;
                    for (int d = 0; d < 6; ++d) regxv[6 * (size_t)q + d] = o[d];  // x0, v0
                }
                aux[i] = x;
                const double tnew = dadd(r.t0, x.step);
                tn[i] = tnew;
                mact = min(mact, (unsigned long long)__double_as_longlong(tnew));
            }
        }
        mact = cta_min<NT>(mact);
        if (threadIdx.x == 0) atomicMin(&c->mact_bits[p], mact);
        if (__syncthreads_or(due) && threadIdx.x == 0) atomicOr(&c->regdue, 1);
        const bool go = grid_sync(c, status, [&] {
            // the block is done (blk_step's last-CTA bookkeeping)
            const int q = p ^ 1;
            c->blocks += 1;
            c->irr_steps += na;
            c->tblock = t;
            c->last_nact = na;
            c->last_parity = p;
            // (the arrival atomic acquired every CTA's minima and flags)
            c->tmin_bits[q] = min(cv->m2_bits[p], cv->mact_bits[p]);
            c->m2_bits[q] = ~0ull;
            c->mact_bits[q] = ~0ull;
            c->nact[q] = 0;
            c->parity = q;
            if (cv->regdue) {
                c->regdue = 0;
                c->stop = 1;
            }
        });
        if (!go) return;
        prev_na = na;
        prev_p = p;
        prev_t = t;
    }
}

// tn = t0 + step of every body (after host staging)
__global__ void blk_clock_sync(int n, const Rec *__restrict__ rec, const Aux *__restrict__ aux,
                               double *__restrict__ tn) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (size_t)n;
         i += (size_t)gridDim.x * blockDim.x)
        tn[i] = dadd(rec[i].t0, aux[i].step);
}

// The resident Hermite state of addresses a0 .. a0+n-1 (0-based), one row
// of 32 doubles each: x0[3], v0[3], F[3], FDOT[3], fi[3], fidot[3], fr[3],
// frdot[3], t0, step, t0r, stepr, rs, m, 0, 0.
__global__ void hermite_gather(int a0, int n, const Rec *__restrict__ rec, const Aux *__restrict__ aux,
                               double *__restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const Rec r = rec[a0 + k];
    const Aux x = aux[a0 + k];
    double *o = out + (size_t)k * 32;
    for (int c = 0; c < 3; ++c) {
        o[c] = r.x[c];
        o[3 + c] = r.v[c];
        o[6 + c] = r.f[c];
        o[9 + c] = r.fd[c];
        o[12 + c] = x.fi[c];
        o[15 + c] = x.fid[c];
        o[18 + c] = x.fr[c];
        o[21 + c] = x.frd[c];
    }
    o[24] = r.t0;
    o[25] = x.step;
    o[26] = x.t0r;
    o[27] = x.stepr;
    o[28] = x.rs;
    o[29] = r.m;
    o[30] = o[31] = 0.0;
}

// Scatter staged Aux records: slot s goes to particle saddr[s].
__global__ void irr_scatter_aux(int n, const int *__restrict__ saddr, const Aux *__restrict__ src,
                                Aux *__restrict__ aux) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) aux[saddr[s]] = src[s];
}

// Scatter everything staged since the last flush, in one launch: blocks
// [0, nbr) move record slot s to particle saddr[s] (one thread per record);
// the remaining blocks move list entry e (one warp per entry), which starts
// at off[e] in `words` as [addr, nnb, ids...].
constexpr int SCATTER_NT = 256;
__global__ void __launch_bounds__(SCATTER_NT)
    irr_scatter(int njp, int nbr, const int *__restrict__ saddr, const Rec *__restrict__ src,
                Rec *__restrict__ rec, int ne, const int *__restrict__ off, const int *__restrict__ words,
                int *__restrict__ lists, int ls) {
    if ((int)blockIdx.x < nbr) {
        const int s = blockIdx.x * SCATTER_NT + threadIdx.x;
        if (s < njp) rec[saddr[s]] = src[s];
        return;
    }
    const int warp = ((blockIdx.x - nbr) * SCATTER_NT + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= ne) return;
    const int *e = words + off[warp];
    const int a = e[0], nnb = e[1];
    int *row = lists + (size_t)a * ls;
    if (lane == 0) row[0] = nnb;
    for (int l = lane; l < nnb; l += 32) row[1 + l] = e[2 + l];
}

// Predict resident records to time t and write them as the regular-force j
// set: output body q lies in segment s with segoff[s] <= q < segoff[s+1] and
// is record addr0[s] + (q - segoff[s]).  The predictor is xbpredall.F:50-59
// with every operation rounded separately (no FMA contraction), so the
// values equal a host FP64 prediction of the same state bit for bit.
__global__ void irr_predict_pack(int n, double t, int nseg, const int *__restrict__ segoff,
                                 const int *__restrict__ addr0, const Rec *__restrict__ rec,
                                 double *__restrict__ jm, double *__restrict__ jx,
                                 double *__restrict__ jv, JSetOut o, int *status) {
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < o.npad;
         q += (size_t)gridDim.x * blockDim.x) {
        if (q >= (size_t)n) {
            write_j(o, q, false, 0, 0, 0, 0, 0, 0, 0);
            continue;
        }
        int lo = 0, hi = nseg - 1;  // last segment with segoff <= q
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (segoff[mid] <= (int)q) lo = mid;
            else hi = mid - 1;
        }
        Rec r;
        load_rec(rec + addr0[lo] + ((int)q - segoff[lo]), r);
        const double s = __dsub_rn(t, r.t0);
        const double s1 = __dmul_rn(1.5, s), s2 = __dmul_rn(2.0, s);
        double x[3], v[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            x[k] = __dadd_rn(__dmul_rn(__dadd_rn(__dmul_rn(__dadd_rn(__dmul_rn(r.fd[k], s), r.f[k]), s),
                                                 r.v[k]),
                                       s),
                             r.x[k]);
            v[k] = __dadd_rn(__dmul_rn(__dadd_rn(__dmul_rn(r.fd[k], s1), r.f[k]), s2), r.v[k]);
        }
        if (x[0] != x[0] || x[1] != x[1] || x[2] != x[2] || v[0] != v[0] || v[1] != v[1] ||
            v[2] != v[2] || r.m != r.m)
            set_status(status, NB6_ERR_NAN_INPUT);
        jm[q] = r.m;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            jx[3 * q + k] = x[k];
            jv[3 * q + k] = v[k];
        }
        write_j(o, q, true, x[0], x[1], x[2], r.m, v[0], v[1], v[2]);
    }
}

struct IrrState {
    bool open = false;
    int nmax = 0, lmax = 0;
    DevBuf<Rec> rec;
    DevBuf<int> lists;
    DevBuf<Rec> dstage_rec;
    DevBuf<int> dints;     // [jp addr | list offsets | active addr | list words]
    DevBuf<double> dout;
    DevBuf<int> dseg;      // predict-send segment tables
    HostBuf<int> hseg;
    HostBuf<Rec> hstage_rec;
    HostBuf<int> hstage_addr, hstage_list, hints;
    HostBuf<double> hout;
    std::vector<int> jp_slot, list_slot;  // staged slot per particle, -1 if none
    std::vector<int> nnb_host;            // list lengths, for the profile counters
    long long nnb_total = 0;              // their sum
    std::vector<int> flush_off;           // latest list entry per particle, per flush
    int njp = 0, nlist = 0;
    size_t list_words = 0;
    double time_grav = 0;
    unsigned long long num_inter = 0, num_fcall = 0, num_steps = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;  // irr_kernel of the last call
    cudaStream_t cst = nullptr;                // downloads of the chunks' results
    cudaEvent_t evk[IRR_CHUNKS] = {}, evc[IRR_CHUNKS] = {};   // chunk kernel / download done
    int chunks_max = IRR_CHUNKS;               // nb6_irr_tune_
    DevBuf<Pv> pv;                             // the predicted set of the running call, nmax bodies
    bool pv_zeroed = false;                    // pv cleared since open (bodies never set stay zero)
    int pv_mode = -1;                          // nb6_irr_pv_ / NB6_IRR_PV: 0 never, 1 by size, 2 always
    int addr_hi = 0;                           // 1 + the highest address set (records above are zero)
    // device-resident corrector state (nb6_hermite_open_)
    bool hermite = false;
    HermiteParams hp{};
    DevBuf<Aux> aux, dstage_aux;
    DevBuf<int> dstage_aux_addr;
    HostBuf<Aux> hstage_aux;
    HostBuf<int> hstage_aux_addr;
    std::vector<int> aux_slot;
    int naux = 0;
    // perturbed KS pairs (nb6_ks_set_): slot table over addresses, pair
    // data [xk 6P | vk 6P | mk 2P], ints [pofs P+1 | plist]
    DevBuf<int> ks_slot, ks_int;
    DevBuf<double> ks_dbl;
    HostBuf<int> ks_hint;
    HostBuf<double> ks_hdbl;
    int ks_npair = 0;
    // device block clock (nb6_blocks_run_): tn[i] = t0 + step of every
    // body, kept by the correctors; recomputed after host staging
    DevBuf<double> tn;
    bool clock_dirty = true;
    DevBuf<int> bact;                 // active set of the running block
    DevBuf<double> brows;             // its corrector rows [nmax][24]
    DevBuf<BlockCtl> bctl;
    HostBuf<BlockCtl> hctl;
    cudaGraphExec_t bgraph = nullptr;
    const void *bgraph_key[11] = {};  // buffers, size and pair table the graph was made with
    int blk_batch = 16;               // blocks per synchronisation
    int blk_unroll = 0;               // blocks per graph (NB6_BLK_UNROLL, default 4)
    bool blk_pdl = true;              // programmatic edges between the block kernels (NB6_BLK_PDL=0: off)
    int blk_persist = -1;             // 1: one persistent launch per run (NB6_BLK_PERSIST=1; default 0)
    const int *bact_last = nullptr;   // the last block's active set (a half of bact in the persistent form)
    DevBuf<int> breg;                 // regular-due bodies of the running block
    DevBuf<double> bregxv;            // their x0, v0
    DevBuf<int> bsort;                // [sorted addresses | slots in | slots out], 3 x nmax
    DevBuf<char> bsort_tmp;
    long long rc_calls = 0;           // nb6_regf_correct_ calls and their host-side phases
    double rc_t[4] = {0, 0, 0, 0};
    // radius-rule quantities per cluster (nb6_hermite_adjust_)
    int ac_nb_flag = 0, nacl = 0;
    DevBuf<int> acl_a0;
    DevBuf<double> acpar;
    // neighbour rows read back (nb6_irr_lists_get_)
    DevBuf<int> lg_dev;
    HostBuf<int> lg_host;
};
IrrState I;

// the current pair table for the force kernels (none: slot == nullptr)
KsArgs ks_args() {
    KsArgs k{};
    if (I.ks_npair <= 0) return k;
    const size_t P = (size_t)I.ks_npair;
    k.slot = I.ks_slot.ptr;
    k.xk = I.ks_dbl.ptr;
    k.vk = I.ks_dbl.ptr + 6 * P;
    k.mk = I.ks_dbl.ptr + 12 * P;
    k.pofs = I.ks_int.ptr;
    k.plist = I.ks_int.ptr + P + 1;
    return k;
}

// The predicted set for a call at ti over ni active bodies, or null when
// the record walk serves the call: with a pair table, or when the call's
// list entries (ni x the mean list length) number fewer than 4 per body
// set.  The prediction pass reads every record set so far and writes its
// 64-byte body (192 bytes per body) and saves 64 bytes per list entry; on
// a B200 (lists of 64 in a Plummer N = 262,144) the call took 7% less time
// at 4 entries per body set, 16% less at 16, the same at 2 and 9% more at
// 1.
const Pv *irr_predicted_set(int ni, double ti, cudaStream_t st) {
    if (I.pv_mode < 0) {
        const char *e = getenv("NB6_IRR_PV");
        I.pv_mode = e ? atoi(e) : 1;
    }
    const int n = I.addr_hi;
    if (I.ks_npair > 0 || I.pv_mode == 0 || n <= 0) return nullptr;
    if (I.pv_mode == 1 && (double)ni * (double)I.nnb_total < 4.0 * (double)n * (double)n) return nullptr;
    if (!I.pv_zeroed) {
        // every address the lists or the active set can name (< nmax) has a
        // body; those never set keep the zeros that predict() makes of
        // their zero records
        I.pv.reserve((size_t)I.nmax);
        NB6_CUDA_CHECK(cudaMemsetAsync(I.pv.ptr, 0, sizeof(Pv) * (size_t)I.nmax, st));
        I.pv_zeroed = true;
    }
    irr_predict_set<<<(n + PS_NT - 1) / PS_NT, PS_NT, 0, st>>>(n, ti, I.rec.ptr, I.pv.ptr);
    return I.pv.ptr;
}

// out: rows of 8 doubles; or, out null, the caller's layout in fv.  pv: the
// call's predicted set (irr_predicted_set), null for the record walk.
void launch_irr_kernel(int ni, const int *daddr, double ti, double *out, cudaStream_t st, double *fv = nullptr,
                       const Pv *pv = nullptr) {
    const KsArgs ks = ks_args();
    const dim3 grid((ni + IRR_WARPS - 1) / IRR_WARPS), block(IRR_WARPS * 32);
    const Rec *rec = I.rec.ptr;
    const int *lists = I.lists.ptr;
    if (ks.slot)
        irr_kernel<true><<<grid, block, 0, st>>>(ni, daddr, ti, rec, nullptr, lists, I.lmax, I.nmax, ks, out, fv);
    else if (pv)
        irr_kernel<false, true><<<grid, block, 0, st>>>(ni, daddr, ti, rec, pv, lists, I.lmax, I.nmax, ks, out, fv);
    else
        irr_kernel<false><<<grid, block, 0, st>>>(ni, daddr, ti, rec, nullptr, lists, I.lmax, I.nmax, ks, out, fv);
}

__global__ void ks_scatter_slots(int npair, const int *__restrict__ cm, int *__restrict__ slot) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < npair) slot[cm[p]] = p;
}

void irr_open_impl(int nmax, int lmax, int rank) {
    nb6_devinit_once(rank);
    if (I.open) {
        fprintf(stderr, "irr_simd: it is already open\n");
        return;
    }
    if (nmax <= 0 || lmax < 1) {
        nb6_fatal(NB6_ERR_BAD_ARG);
        return;
    }
    I.open = true;
    nb6_lib_opened();
    I.nmax = nmax;
    I.lmax = lmax;
    I.rec.reserve((size_t)nmax + 1);
    I.lists.reserve((size_t)nmax * lmax);
    NB6_CUDA_CHECK(cudaMemsetAsync(I.rec.ptr, 0, sizeof(Rec) * ((size_t)nmax + 1), nb6_stream()));
    NB6_CUDA_CHECK(cudaMemsetAsync(I.lists.ptr, 0, sizeof(int) * (size_t)nmax * lmax, nb6_stream()));
    I.jp_slot.assign(nmax, -1);
    I.list_slot.assign(nmax, -1);
    I.nnb_host.assign(nmax, 0);
    I.nnb_total = 0;
    I.njp = I.nlist = 0;
    I.addr_hi = 0;
    I.pv_zeroed = false;
    I.list_words = 0;
    I.time_grav = 0;
    I.num_inter = I.num_fcall = I.num_steps = 0;
    if (getenv("NB6_VERBOSE"))
        fprintf(stderr, "# Opening IRR lib. GPU ver. - rank: %d; nmax: %d, lmax: %d\n", rank, nmax, lmax);
}

void irr_profile_impl(int rank);

void irr_close_impl() {
    if (!I.open) {
        fprintf(stderr, "irr_simd: it is already close\n");
        return;
    }
    if (getenv("NB6_VERBOSE")) irr_profile_impl(0);   // the counters of the session
    I.open = false;
    I.rec.release();
    I.pv.release();
    I.lists.release();
    I.dstage_rec.release();
    I.dints.release();
    I.dout.release();
    I.dseg.release();
    I.hseg.release();
    I.aux.release();
    I.tn.release();
    I.clock_dirty = true;
    if (I.bgraph) cudaGraphExecDestroy(I.bgraph);
    I.bgraph = nullptr;
    memset(I.bgraph_key, 0, sizeof(I.bgraph_key));
    I.bact.release();
    I.bact_last = nullptr;
    I.breg.release();
    I.bregxv.release();
    I.bsort.release();
    I.bsort_tmp.release();
    I.brows.release();
    I.bctl.release();
    I.hctl.release();
    I.dstage_aux.release();
    I.dstage_aux_addr.release();
    I.hstage_aux.release();
    I.hstage_aux_addr.release();
    I.aux_slot.clear();
    I.naux = 0;
    I.hermite = false;
    I.nacl = 0;
    I.ac_nb_flag = 0;
    I.acl_a0.release();
    I.acpar.release();
    I.lg_dev.release();
    I.lg_host.release();
    I.ks_slot.release();
    I.ks_int.release();
    I.ks_dbl.release();
    I.ks_hint.release();
    I.ks_hdbl.release();
    I.ks_npair = 0;
    I.hstage_rec.release();
    I.hstage_addr.release();
    I.hstage_list.release();
    I.hints.release();
    I.hout.release();
    I.jp_slot.clear();
    I.list_slot.clear();
    nb6_lib_closed();
}

void irr_set_jp_impl(int a, const double *pos, const double *vel, const double *acc2,
                     const double *jrk6, double mass, double time) {
    if (!I.open) {
        nb6_fatal(NB6_ERR_NOT_OPEN);
        return;
    }
    if (a < 0 || a >= I.nmax) {
        fprintf(stderr, "irr_simd_set_jp: address %d outside [1, %d]\n", a + 1, I.nmax);
        nb6_fatal(NB6_ERR_BAD_ARG);
        return;
    }
    if (a + 1 > I.addr_hi) I.addr_hi = a + 1;
    int s = I.jp_slot[a];
    if (s < 0) {
        s = I.njp++;
        I.jp_slot[a] = s;
        if ((size_t)I.njp > I.hstage_rec.cap) {
            // grow pinned staging, keeping staged content
            HostBuf<Rec> nr;
            HostBuf<int> na;
            nr.reserve((size_t)I.njp * 2);
            na.reserve((size_t)I.njp * 2);
            if (I.njp > 1) {
                memcpy(nr.ptr, I.hstage_rec.ptr, sizeof(Rec) * (I.njp - 1));
                memcpy(na.ptr, I.hstage_addr.ptr, sizeof(int) * (I.njp - 1));
            }
            I.hstage_rec.release();
            I.hstage_addr.release();
            I.hstage_rec = nr;
            I.hstage_addr = na;
        }
        I.hstage_addr.ptr[s] = a;
    }
    Rec &r = I.hstage_rec.ptr[s];
    for (int k = 0; k < 3; ++k) {
        r.x[k] = pos[k];
        r.v[k] = vel[k];
        r.f[k] = acc2[k];
        r.fd[k] = jrk6[k];
    }
    r.m = mass;
    r.t0 = time;
    r.pad0 = r.pad1 = 0.0;
}

void irr_set_list_impl(int a, const int *nblist) {
    if (!I.open) {
        nb6_fatal(NB6_ERR_NOT_OPEN);
        return;
    }
    const int nnb = nblist[0];
    if (a < 0 || a >= I.nmax || nnb < 0 || nnb > I.lmax - 1) {
        fprintf(stderr, "irr_simd_set_list: address %d or nnb %d outside the opened sizes\n", a + 1, nnb);
        nb6_fatal(NB6_ERR_BAD_ARG);
        return;
    }
    for (int l = 1; l <= nnb; ++l) {
        if (nblist[l] < 1 || nblist[l] > I.nmax) {
            fprintf(stderr, "irr_simd_set_list: neighbour id %d outside [1, %d]\n", nblist[l], I.nmax);
            nb6_fatal(NB6_ERR_BAD_ARG);
            return;
        }
    }
    // Entries are appended; a re-set of the same particle before the next
    // flush supersedes the earlier entry (list_slot keeps the latest).
    const size_t need = I.list_words + 2 + nnb;
    if (need > I.hstage_list.cap) {
        HostBuf<int> nl;
        nl.reserve(std::max(need * 2, (size_t)4096));
        if (I.list_words) memcpy(nl.ptr, I.hstage_list.ptr, sizeof(int) * I.list_words);
        I.hstage_list.release();
        I.hstage_list = nl;
    }
    int *e = I.hstage_list.ptr + I.list_words;
    e[0] = a;
    e[1] = nnb;
    for (int l = 0; l < nnb; ++l) e[2 + l] = nblist[1 + l] - 1;
    I.list_slot[a] = (int)I.list_words;
    I.nnb_total += nnb - I.nnb_host[a];
    I.nnb_host[a] = nnb;
    I.list_words = need;
    I.nlist++;
}

// Small stagings are read by the kernels straight from pinned host memory
// (mapped under unified addressing), and small results written straight
// into it, which saves the copy launches that dominate a small call; large
// ones go through one bulk DMA copy each.  The limits differ by access:
//   records (ZC_REC_MAX)   read once, coalesced, by the scatter kernel;
//   integers (ZC_INTS_MAX) the active addresses among them, read one per
//                          warp at the head of each walk, so each warp
//                          waits a PCIe round trip;
//   results (ZC_OUT_MAX)   written in 8-byte pieces per body.
// Measured on a B200 (irr_simd_firr_vec_, lists of 64 in a Plummer
// N = 262,144): results written to host memory cost 0.24 ms per call at
// 16,384 bodies against 0.11 ms through a device buffer and one download,
// and the same at 256 bodies; addresses read from host memory cost 0.34 ms
// at 65,536 bodies against 0.25 ms uploaded, and won at 4,096.
// NB6_ZC_REC, NB6_ZC_INTS and NB6_ZC_OUT (bytes) override them.
constexpr size_t ZC_REC_MAX = 1 << 20, ZC_INTS_MAX = 32 << 10, ZC_OUT_MAX = 16 << 10;
size_t zc_limit(const char *name, size_t def) {
    const char *e = getenv(name);
    return nb6_uva() ? (e ? (size_t)atoll(e) : def) : 0;
}
size_t zero_copy_rec_bytes() {
    static const size_t lim = zc_limit("NB6_ZC_REC", ZC_REC_MAX);
    return lim;
}
size_t zero_copy_ints_bytes() {
    static const size_t lim = zc_limit("NB6_ZC_INTS", ZC_INTS_MAX);
    return lim;
}
size_t zero_copy_out_bytes() {
    static const size_t lim = zc_limit("NB6_ZC_OUT", ZC_OUT_MAX);
    return lim;
}

// Upload and scatter everything staged since the last flush, with the
// active addresses of a force call (active may be null): the records and
// all integers either read in place or copied once each, then one scatter
// launch.  Returns a device-readable pointer to the active addresses.
const int *irr_flush(cudaStream_t st, const int *active = nullptr, int ni = 0) {
    if (I.naux > 0) {
        I.dstage_aux.reserve(I.naux);
        I.dstage_aux_addr.reserve(I.naux);
        NB6_CUDA_CHECK(cudaMemcpyAsync(I.dstage_aux.ptr, I.hstage_aux.ptr, sizeof(Aux) * I.naux,
                                       cudaMemcpyHostToDevice, st));
        NB6_CUDA_CHECK(cudaMemcpyAsync(I.dstage_aux_addr.ptr, I.hstage_aux_addr.ptr, sizeof(int) * I.naux,
                                       cudaMemcpyHostToDevice, st));
        irr_scatter_aux<<<(I.naux + 255) / 256, 256, 0, st>>>(I.naux, I.dstage_aux_addr.ptr, I.dstage_aux.ptr,
                                                             I.aux.ptr);
        NB6_CUDA_CHECK(cudaGetLastError());
        for (int q = 0; q < I.naux; ++q) I.aux_slot[I.hstage_aux_addr.ptr[q]] = -1;
        I.naux = 0;
        I.clock_dirty = true;
    }
    // keep only the latest list entry per particle
    int ne = 0;
    std::vector<int> &offs = I.flush_off;
    offs.clear();
    if (I.nlist > 0) {
        size_t w = 0;
        while (w < I.list_words) {
            const int a = I.hstage_list.ptr[w];
            const int nnb = I.hstage_list.ptr[w + 1];
            if (I.list_slot[a] == (int)w) {
                offs.push_back((int)w);
                I.list_slot[a] = -1;
            }
            w += 2 + nnb;
        }
        ne = (int)offs.size();
    }
    const int njp = I.njp;
    const size_t nint = (size_t)njp + ne + ni + I.list_words;
    if (nint == 0) return nullptr;
    I.hints.reserve(nint);
    I.dints.reserve(nint);
    int *h = I.hints.ptr;
    if (njp) memcpy(h, I.hstage_addr.ptr, sizeof(int) * njp);
    if (ne) memcpy(h + njp, offs.data(), sizeof(int) * ne);
    if (ni) memcpy(h + njp + ne, active, sizeof(int) * ni);
    if (I.list_words) memcpy(h + njp + ne + ni, I.hstage_list.ptr, sizeof(int) * I.list_words);
    const Rec *drec = I.hstage_rec.ptr;
    if (njp && sizeof(Rec) * (size_t)njp > zero_copy_rec_bytes()) {
        I.dstage_rec.reserve(njp);
        NB6_CUDA_CHECK(cudaMemcpyAsync(I.dstage_rec.ptr, I.hstage_rec.ptr, sizeof(Rec) * njp,
                                       cudaMemcpyHostToDevice, st));
        drec = I.dstage_rec.ptr;
    }
    const int *d = h;
    if (sizeof(int) * nint > zero_copy_ints_bytes()) {
        NB6_CUDA_CHECK(cudaMemcpyAsync(I.dints.ptr, h, sizeof(int) * nint, cudaMemcpyHostToDevice, st));
        d = I.dints.ptr;
    }
    const int nbr = (njp + SCATTER_NT - 1) / SCATTER_NT;
    const int nbl = (int)(((size_t)ne * 32 + SCATTER_NT - 1) / SCATTER_NT);
    if (nbr + nbl > 0) {
        irr_scatter<<<nbr + nbl, SCATTER_NT, 0, st>>>(njp, nbr, d, drec, I.rec.ptr, ne, d + njp,
                                                      d + njp + ne + ni, I.lists.ptr, I.lmax);
        NB6_CUDA_CHECK(cudaGetLastError());
    }
    for (int q = 0; q < njp; ++q) I.jp_slot[I.hstage_addr.ptr[q]] = -1;
    if (njp) I.clock_dirty = true;
    I.njp = 0;
    I.nlist = 0;
    I.list_words = 0;
    return d + njp + ne;
}

void irr_firr_vec_impl(double ti, int ni, const int *addr, double (*acc)[3], double (*jrk)[3],
                       int *nnbid) {
    if (!I.open) {
        nb6_fatal(NB6_ERR_NOT_OPEN);
        return;
    }
    if (ni <= 0) return;
    int bad = 0;
    for (int k = 0; k < ni; ++k) bad |= (addr[k] < 1) | (addr[k] > I.nmax);
    if (bad) {
        for (int k = 0; k < ni; ++k)
            if (addr[k] < 1 || addr[k] > I.nmax) {
                fprintf(stderr, "irr_simd_firr_vec: address %d outside [1, %d]\n", addr[k], I.nmax);
                break;
            }
        nb6_fatal(NB6_ERR_BAD_ARG);
        return;
    }
    const double t0 = nb6_wtime();
    cudaStream_t st = nb6_stream();
    // the pinned staging is reused only after this call's synchronize, so
    // the uploads enqueued here read it intact
    const int *daddr = irr_flush(st, addr, ni);
    // Results in the caller's layout, per chunk of bodies [a, a+m): at
    // double offset 7a, acc[m][3] | jrk[m][3] (doubles) | nnbid[m] | nnb[m]
    // (ints) -- one chunk covering all ni is exactly the caller's three
    // arrays back to back.  Small calls write straight to pinned host
    // memory; large ones into one device buffer, each chunk downloaded on a
    // second stream as soon as its kernel ends, then copied into the
    // caller's arrays by the copy pool while later chunks run.  (With a
    // device status error and NB6_ABORT_ON_ERROR=0 the caller's arrays may
    // hold part of the results.)
    const size_t nd = 7 * (size_t)ni;   // 6 ni doubles + 2 ni ints
    const size_t bytes = sizeof(double) * nd;
    I.hout.reserve(nd);
    const bool direct = bytes <= zero_copy_out_bytes();
    double *out = I.hout.ptr;
    if (!direct) {
        I.dout.reserve(nd);
        out = I.dout.ptr;
    }
    const int nch = direct ? 1 : std::max(1, std::min(I.chunks_max, ni / IRR_CHUNK_MIN));
    if (!I.ev0) {
        NB6_CUDA_CHECK(cudaEventCreate(&I.ev0));
        NB6_CUDA_CHECK(cudaEventCreate(&I.ev1));
    }
    if (!direct && !I.cst) {
        NB6_CUDA_CHECK(cudaStreamCreateWithFlags(&I.cst, cudaStreamNonBlocking));
        for (int c = 0; c < IRR_CHUNKS; ++c) {
            NB6_CUDA_CHECK(cudaEventCreateWithFlags(&I.evk[c], cudaEventDisableTiming));
            NB6_CUDA_CHECK(cudaEventCreateWithFlags(&I.evc[c], cudaEventDisableTiming));
        }
    }
    CopyPool *pool = direct ? nullptr : &nb6_copy_pool();
    auto chunk_lo = [&](int c) { return (int)((long long)ni * c / nch); };
    NB6_CUDA_CHECK(cudaEventRecord(I.ev0, st));
    const Pv *pv = irr_predicted_set(ni, ti, st);
    for (int c = 0; c < nch; ++c) {
        const int a = chunk_lo(c), m = chunk_lo(c + 1) - a;
        launch_irr_kernel(m, daddr + a, ti, nullptr, st, out + 7 * (size_t)a, pv);
        NB6_CUDA_CHECK(cudaGetLastError());
        if (!direct) {
            NB6_CUDA_CHECK(cudaEventRecord(I.evk[c], st));
            NB6_CUDA_CHECK(cudaStreamWaitEvent(I.cst, I.evk[c], 0));
            NB6_CUDA_CHECK(cudaMemcpyAsync(I.hout.ptr + 7 * (size_t)a, out + 7 * (size_t)a,
                                           sizeof(double) * 7 * (size_t)m, cudaMemcpyDeviceToHost, I.cst));
            NB6_CUDA_CHECK(cudaEventRecord(I.evc[c], I.cst));
        }
    }
    NB6_CUDA_CHECK(cudaEventRecord(I.ev1, st));
    nb6_status_fetch(st);
    unsigned long long inter = 0;
    if (pool) pool->arm();
    if (!direct) {
        const int np = pool->parts();
        std::vector<unsigned long long> part(np);
        for (int c = 0; c < nch; ++c) {
            NB6_CUDA_CHECK(cudaEventSynchronize(I.evc[c]));
            const int a = chunk_lo(c), m = chunk_lo(c + 1) - a;
            const double *h = I.hout.ptr + 7 * (size_t)a;
            pool->run([&](int p) {
                const int lo = (int)((long long)m * p / np), hi = (int)((long long)m * (p + 1) / np);
                if (hi <= lo) return;
                memcpy(&acc[a + lo][0], h + 3 * (size_t)lo, sizeof(double) * 3 * (size_t)(hi - lo));
                memcpy(&jrk[a + lo][0], h + 3 * (size_t)m + 3 * (size_t)lo, sizeof(double) * 3 * (size_t)(hi - lo));
                const int *hi_ = reinterpret_cast<const int *>(h + 6 * (size_t)m);
                memcpy(nnbid + a + lo, hi_ + lo, sizeof(int) * (size_t)(hi - lo));
                unsigned long long s = 0;
                for (int k = lo; k < hi; ++k) s += (unsigned)hi_[m + k];
                part[p] += s;
            });
        }
        for (int p = 0; p < np; ++p) inter += part[p];
    }
    NB6_CUDA_CHECK(cudaStreamSynchronize(st));
    if (nb6_check_dev_status() != 0) return;
    if (direct) {
        const double *h = I.hout.ptr;
        memcpy(&acc[0][0], h, sizeof(double) * 3 * (size_t)ni);
        memcpy(&jrk[0][0], h + 3 * (size_t)ni, sizeof(double) * 3 * (size_t)ni);
        const int *hi = reinterpret_cast<const int *>(h + 6 * (size_t)ni);
        memcpy(nnbid, hi, sizeof(int) * (size_t)ni);
        for (int k = 0; k < ni; ++k) inter += (unsigned)hi[ni + k];
    }
    I.num_inter += inter;
    I.time_grav += nb6_wtime() - t0;
    I.num_fcall++;
    I.num_steps += ni;
}

void hermite_open_impl(double eta_i, double smax, double dtmin) {
    if (!I.open) {
        nb6_fatal(NB6_ERR_NOT_OPEN);
        return;
    }
    I.aux.reserve((size_t)I.nmax + 1);
    NB6_CUDA_CHECK(cudaMemsetAsync(I.aux.ptr, 0, sizeof(Aux) * ((size_t)I.nmax + 1), nb6_stream()));
    I.tn.reserve((size_t)I.nmax + 1);
    I.clock_dirty = true;
    I.aux_slot.assign(I.nmax, -1);
    I.naux = 0;
    I.hp.eta_i = eta_i;
    I.hp.smax = smax;
    I.hp.dtmin = dtmin;
    I.hermite = true;
}

void hermite_set_impl(int a, const double *fi, const double *fid, const double *fr, const double *frd,
                      double step, double t0r, double stepr, double rs) {
    if (!I.hermite) {
        nb6_fatal(NB6_ERR_NOT_OPEN);
        return;
    }
    if (a < 0 || a >= I.nmax) {
        fprintf(stderr, "nb6_hermite_set: address %d outside [1, %d]\n", a + 1, I.nmax);
        nb6_fatal(NB6_ERR_BAD_ARG);
        return;
    }
    int slot = I.aux_slot[a];
    if (slot < 0) {
        slot = I.naux++;
        I.aux_slot[a] = slot;
        if ((size_t)I.naux > I.hstage_aux.cap) {
            HostBuf<Aux> na;
            HostBuf<int> nd;
            na.reserve((size_t)I.naux * 2);
            nd.reserve((size_t)I.naux * 2);
            if (I.naux > 1) {
                memcpy(na.ptr, I.hstage_aux.ptr, sizeof(Aux) * (I.naux - 1));
                memcpy(nd.ptr, I.hstage_aux_addr.ptr, sizeof(int) * (I.naux - 1));
            }
            I.hstage_aux.release();
            I.hstage_aux_addr.release();
            I.hstage_aux = na;
            I.hstage_aux_addr = nd;
        }
        I.hstage_aux_addr.ptr[slot] = a;
    }
    Aux &x = I.hstage_aux.ptr[slot];
    for (int k = 0; k < 3; ++k) {
        x.fi[k] = fi[k];
        x.fid[k] = fid[k];
        x.fr[k] = fr[k];
        x.frd[k] = frd[k];
    }
    x.step = step;
    x.t0r = t0r;
    x.stepr = stepr;
    x.rs = rs;
}

void irr_correct_impl(double time, int ni, const int *addr, double *out) {
    if (!I.open || !I.hermite) {
        nb6_fatal(NB6_ERR_NOT_OPEN);
        return;
    }
    if (ni <= 0) return;
    for (int k = 0; k < ni; ++k) {
        if (addr[k] < 1 || addr[k] > I.nmax) {
            fprintf(stderr, "nb6_irr_correct: address %d outside [1, %d]\n", addr[k], I.nmax);
            nb6_fatal(NB6_ERR_BAD_ARG);
            return;
        }
    }
    const double t0 = nb6_wtime();
    cudaStream_t st = nb6_stream();
    const int *daddr = irr_flush(st, addr, ni);
    const size_t rowd = 24;
    I.hout.reserve((size_t)ni * rowd);
    const bool direct = sizeof(double) * rowd * (size_t)ni <= zero_copy_out_bytes();
    // forces of all active bodies into a device buffer, then the corrector
    I.dout.reserve((size_t)ni * (8 + (direct ? 0 : rowd)));
    double *force = I.dout.ptr;
    double *o = direct ? I.hout.ptr : I.dout.ptr + (size_t)ni * 8;
    if (!I.ev0) {
        NB6_CUDA_CHECK(cudaEventCreate(&I.ev0));
        NB6_CUDA_CHECK(cudaEventCreate(&I.ev1));
    }
    NB6_CUDA_CHECK(cudaEventRecord(I.ev0, st));
    launch_irr_kernel(ni, daddr, time, force, st, nullptr, irr_predicted_set(ni, time, st));
    NB6_CUDA_CHECK(cudaGetLastError());
    NB6_CUDA_CHECK(cudaEventRecord(I.ev1, st));
    irr_apply_corrector<<<(ni + 127) / 128, 128, 0, st>>>(ni, daddr, time, force, I.rec.ptr, I.aux.ptr, I.hp, o,
                                                          I.tn.ptr);
    NB6_CUDA_CHECK(cudaGetLastError());
    if (!direct)
        NB6_CUDA_CHECK(cudaMemcpyAsync(I.hout.ptr, o, sizeof(double) * rowd * ni, cudaMemcpyDeviceToHost, st));
    nb6_status_fetch(st);
    NB6_CUDA_CHECK(cudaStreamSynchronize(st));
    if (nb6_check_dev_status() != 0) return;
    memcpy(out, I.hout.ptr, sizeof(double) * rowd * ni);
    unsigned long long inter = 0;
    for (int k = 0; k < ni; ++k) inter += (unsigned long long)I.nnb_host[addr[k] - 1];
    I.num_inter += inter;
    I.time_grav += nb6_wtime() - t0;
    I.num_fcall++;
    I.num_steps += ni;
}

void ks_set_impl(int npair, const int *cm, const double *xk, const double *vk, const double *mk, const int *pofs,
                 const int *plist) {
    if (!I.open) {
        nb6_fatal(NB6_ERR_NOT_OPEN);
        return;
    }
    if (npair < 0) {
        nb6_fatal(NB6_ERR_BAD_ARG);
        return;
    }
    cudaStream_t st = nb6_stream();
    if (npair == 0) {  // no perturbed pairs: the forces go uncorrected
        I.ks_npair = 0;
        return;
    }
    bool bad = pofs[0] != 0;
    std::vector<char> seen(I.nmax, 0);
    for (int p = 0; p < npair && !bad; ++p) {
        bad = cm[p] < 1 || cm[p] > I.nmax || seen[cm[p] - 1] || pofs[p + 1] < pofs[p];
        if (!bad) seen[cm[p] - 1] = 1;
    }
    const int nl = bad ? 0 : pofs[npair];
    for (int l = 0; l < nl && !bad; ++l) bad = plist[l] < 1 || plist[l] > I.nmax;
    if (bad) {
        fprintf(stderr, "nb6_ks_set: pair address, perturber id or list offsets outside [1, %d]\n", I.nmax);
        nb6_fatal(NB6_ERR_BAD_ARG);
        return;
    }
    for (size_t k = 0; k < 6 * (size_t)npair; ++k)
        if (xk[k] != xk[k] || vk[k] != vk[k]) {
            fprintf(stderr, "nb6_ks_set: NaN in a pair's components\n");
            nb6_fatal(NB6_ERR_NAN_INPUT);
            return;
        }
    const size_t P = (size_t)npair;
    const size_t nd = 14 * P, ni = P + (P + 1) + (size_t)nl;
    I.ks_hdbl.reserve(nd);
    I.ks_hint.reserve(ni);
    I.ks_dbl.reserve(nd);
    I.ks_int.reserve(ni);
    I.ks_slot.reserve(I.nmax);
    memcpy(I.ks_hdbl.ptr, xk, sizeof(double) * 6 * P);
    memcpy(I.ks_hdbl.ptr + 6 * P, vk, sizeof(double) * 6 * P);
    memcpy(I.ks_hdbl.ptr + 12 * P, mk, sizeof(double) * 2 * P);
    // ints on the device: [pofs | plist - 1 | cm - 1]
    int *h = I.ks_hint.ptr;
    memcpy(h, pofs, sizeof(int) * (P + 1));
    for (int l = 0; l < nl; ++l) h[P + 1 + l] = plist[l] - 1;
    for (size_t p = 0; p < P; ++p) h[P + 1 + nl + p] = cm[p] - 1;
    NB6_CUDA_CHECK(cudaMemcpyAsync(I.ks_dbl.ptr, I.ks_hdbl.ptr, sizeof(double) * nd, cudaMemcpyHostToDevice, st));
    NB6_CUDA_CHECK(cudaMemcpyAsync(I.ks_int.ptr, h, sizeof(int) * ni, cudaMemcpyHostToDevice, st));
    NB6_CUDA_CHECK(cudaMemsetAsync(I.ks_slot.ptr, 0xff, sizeof(int) * (size_t)I.nmax, st));
    ks_scatter_slots<<<(npair + 255) / 256, 256, 0, st>>>(npair, I.ks_int.ptr + P + 1 + nl, I.ks_slot.ptr);
    NB6_CUDA_CHECK(cudaGetLastError());
    // the pinned staging is rewritten by the next call
    NB6_CUDA_CHECK(cudaStreamSynchronize(st));
    I.ks_npair = npair;
}

// Capture the four launches of one block as a graph (rebuilt when a buffer
// moved or the pair table came or went).
// One cooperative launch of blk_persist for the whole run; false when the
// device cannot hold the grid (then the graph form runs).  On return h holds
// the control block.
bool blocks_persist(cudaStream_t st, int max_blocks, BlockCtl &h) {
    (void)max_blocks;   // in the control block (blimit)
    const KsArgs ks = ks_args();
    const void *fn = ks.slot ? (const void *)blk_persist<true> : (const void *)blk_persist<false>;
    const int nt = ks.slot ? 256 : PB_NT;
    static int coop = -1;
    if (coop < 0) {
        int dev = 0, v = 0;
        NB6_CUDA_CHECK(cudaGetDevice(&dev));
        coop = (cudaDeviceGetAttribute(&v, cudaDevAttrCooperativeLaunch, dev) == cudaSuccess && v) ? 1 : 0;
    }
    int occ = 0;
    if (!coop || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, nt, 0) != cudaSuccess || occ < 1) {
        cudaGetLastError();
        return false;
    }
    const int grid = nb6_num_sms();
    BlockCtl *cp = I.bctl.ptr;
    int *ap = I.bact.ptr;
    int n = I.nmax, ls = I.lmax;
    Rec *rp = I.rec.ptr;
    Aux *xp = I.aux.ptr;
    const int *lp = I.lists.ptr;
    KsArgs ka = ks;
    HermiteParams hp = I.hp;
    double *rows = I.brows.ptr, *tn = I.tn.ptr, *rxv = I.bregxv.ptr;
    int *reg = I.breg.ptr, *status = nb6_dev_status();
    void *args[] = {&cp, &ap, &n, &rp, &xp, &lp, &ls, &ka, &hp, &rows, &tn, &reg, &rxv, &status};
    NB6_CUDA_CHECK(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(nt), args, 0, st));
    NB6_CUDA_CHECK(cudaMemcpyAsync(&h, I.bctl.ptr, sizeof(BlockCtl), cudaMemcpyDeviceToHost, st));
    nb6_status_fetch(st);
    NB6_CUDA_CHECK(cudaStreamSynchronize(st));
    nb6_check_dev_status();
    return true;
}

bool blocks_graph(cudaStream_t st) {
    const KsArgs ks = ks_args();
    const void *key[11] = {I.bact.ptr, I.brows.ptr, I.bctl.ptr, I.tn.ptr, I.breg.ptr, I.bregxv.ptr, I.rec.ptr,
                           I.aux.ptr, I.lists.ptr, ks.slot ? (const void *)I.ks_slot.ptr : nullptr,
                           reinterpret_cast<const void *>((size_t)I.nmax)};
    // (a pair table's layout depends on its size: with one set, capture anew)
    if (I.bgraph && memcmp(key, I.bgraph_key, sizeof(key)) == 0 && !ks.slot) return true;
    if (I.bgraph) {
        cudaGraphExecDestroy(I.bgraph);
        I.bgraph = nullptr;
    }
    const int sms = nb6_num_sms();
    // blk_step: one resident wave of CTAs (they stride over the active set)
    int step_occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &step_occ, ks.slot ? (const void *)blk_step<true> : (const void *)blk_step<false>, IRR_WARPS * 32,
            0) != cudaSuccess ||
        step_occ < 1)
        step_occ = 4;
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return false;
    // blk_unroll blocks back to back; with blk_pdl every kernel after the
    // first is captured with a programmatic edge to the one before it
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    auto cfg = [&](int grid, int threads, bool first) {
        cudaLaunchConfig_t c = {};
        c.gridDim = dim3(grid);
        c.blockDim = dim3(threads);
        c.dynamicSmemBytes = 0;
        c.stream = st;
        c.attrs = at;
        c.numAttrs = (I.blk_pdl && !first) ? 1 : 0;
        return c;
    };
    bool ok = true;
    for (int u = 0; u < I.blk_unroll && ok; ++u) {
        cudaLaunchConfig_t c0 = cfg(sms * 4, BLK_NT, u == 0);
        ok = cudaLaunchKernelEx(&c0, blk_collect, I.nmax, (const double *)I.tn.ptr, I.bctl.ptr, I.bact.ptr,
                                (const double *)I.brows.ptr, I.rec.ptr) == cudaSuccess;
        cudaLaunchConfig_t c1 = cfg(sms * step_occ, IRR_WARPS * 32, false);
        const int *ca = I.bact.ptr, *cl = I.lists.ptr;
        const Rec *cr = I.rec.ptr;
        if (ok && ks.slot)
            ok = cudaLaunchKernelEx(&c1, blk_step<true>, I.bctl.ptr, ca, I.nmax, cr, I.aux.ptr, cl, I.lmax, ks, I.hp,
                                    I.brows.ptr, I.tn.ptr, I.breg.ptr, I.bregxv.ptr) == cudaSuccess;
        else if (ok)
            ok = cudaLaunchKernelEx(&c1, blk_step<false>, I.bctl.ptr, ca, I.nmax, cr, I.aux.ptr, cl, I.lmax, ks,
                                    I.hp, I.brows.ptr, I.tn.ptr, I.breg.ptr, I.bregxv.ptr) == cudaSuccess;
    }
    if (cudaStreamEndCapture(st, &g) != cudaSuccess || !g || !ok) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        if (I.blk_pdl) {  // a runtime without programmatic edges in capture: plain edges
            I.blk_pdl = false;
            return blocks_graph(st);
        }
        return false;
    }
    ok = cudaGraphInstantiate(&I.bgraph, g, 0) == cudaSuccess;
    cudaGraphDestroy(g);
    if (!ok) {
        I.bgraph = nullptr;
        return false;
    }
    memcpy(I.bgraph_key, key, sizeof(key));
    return true;
}

void blocks_run_impl(double tlimit, int max_blocks, int *reason, long long *nblocks, long long *nirr,
                     double *tblock, int *nact) {
    *reason = 0;
    *nblocks = *nirr = 0;
    *nact = 0;
    if (!I.open || !I.hermite) {
        nb6_fatal(NB6_ERR_NOT_OPEN);
        return;
    }
    if (max_blocks < 1 || tlimit != tlimit) {
        nb6_fatal(NB6_ERR_BAD_ARG);
        return;
    }
    const double t0 = nb6_wtime();
    cudaStream_t st = nb6_stream();
    irr_flush(st);
    I.bact.reserve((size_t)I.nmax * 2);
    I.brows.reserve((size_t)I.nmax * 24);
    I.breg.reserve((size_t)I.nmax);
    I.bregxv.reserve((size_t)I.nmax * 6);
    I.bctl.reserve(1);
    I.hctl.reserve(1);
    if (I.clock_dirty) {
        blk_clock_sync<<<nb6_num_sms() * 8, 256, 0, st>>>(I.nmax, I.rec.ptr, I.aux.ptr, I.tn.ptr);
        NB6_CUDA_CHECK(cudaGetLastError());
        I.clock_dirty = false;
    }
    BlockCtl &h = *I.hctl.ptr;
    memset(&h, 0, sizeof(h));
    for (int q = 0; q < 2; ++q) h.tmin_bits[q] = h.m2_bits[q] = h.mact_bits[q] = ~0ull;
    h.tlimit = tlimit;
    h.blimit = max_blocks;
    if (I.blk_unroll == 0) {
        const char *e = getenv("NB6_BLK_UNROLL");
        I.blk_unroll = std::max(1, std::min(32, e ? atoi(e) : 4));
        const char *q = getenv("NB6_BLK_PDL");
        I.blk_pdl = !(q && q[0] == '0');
    }
    if (I.blk_persist < 0) {
        const char *e = getenv("NB6_BLK_PERSIST");
        I.blk_persist = (e && e[0] == '1') ? 1 : 0;
    }
    NB6_CUDA_CHECK(cudaMemcpyAsync(I.bctl.ptr, &h, sizeof(BlockCtl), cudaMemcpyHostToDevice, st));
    // the first block's time from every body; each later one comes from the
    // block before it (blk_collect and blk_step)
    blk_min<<<nb6_num_sms() * 4, BLK_NT, 0, st>>>(I.nmax, I.tn.ptr, I.bctl.ptr);
    NB6_CUDA_CHECK(cudaGetLastError());
    if (I.blk_persist && blocks_persist(st, max_blocks, h)) {
        I.bact_last = I.bact.ptr + (size_t)h.last_parity * I.nmax;
        *reason = h.stop == 3 ? 0 : h.stop;
        *nblocks = h.blocks;
        *nirr = h.irr_steps;
        *tblock = h.tblock;
        *nact = h.last_nact;
        I.time_grav += nb6_wtime() - t0;
        I.num_fcall += (unsigned long long)h.blocks;
        I.num_steps += (unsigned long long)h.irr_steps;
        return;
    }
    if (!blocks_graph(st)) {
        fprintf(stderr, "nb6_blocks_run: the block graph could not be built\n");
        nb6_fatal(NB6_ERR_CUDA);
        return;
    }
    long long done = 0;
    int batch = I.blk_batch;
    for (;;) {
        // blocks past the run's limit or a stop return at once (blimit)
        const int k = (int)std::min<long long>(batch, (long long)max_blocks - done);
        for (int b = 0; b < k; b += I.blk_unroll) NB6_CUDA_CHECK(cudaGraphLaunch(I.bgraph, st));
        NB6_CUDA_CHECK(cudaMemcpyAsync(&h, I.bctl.ptr, sizeof(BlockCtl), cudaMemcpyDeviceToHost, st));
        nb6_status_fetch(st);
        NB6_CUDA_CHECK(cudaStreamSynchronize(st));
        if (nb6_check_dev_status() != 0) return;
        done = h.blocks;
        if (h.stop || done >= max_blocks) break;
        batch = std::min(batch * 2, 256);
    }
    // the last block's new records (the next run starts from a fresh
    // control block)
    if (h.pend_na > 0) {
        blk_flush<<<std::min((h.pend_na + 255) / 256, nb6_num_sms() * 4), 256, 0, st>>>(
            I.bctl.ptr, I.bact.ptr, I.nmax, (const double *)I.brows.ptr, I.rec.ptr);
        NB6_CUDA_CHECK(cudaGetLastError());
        NB6_CUDA_CHECK(cudaStreamSynchronize(st));
    }
    I.bact_last = I.bact.ptr + (size_t)h.last_parity * I.nmax;
    // next run's first batch: about twice this run's length
    I.blk_batch = (int)std::max<long long>(2, std::min<long long>(128, 2 * done));
    *reason = h.stop == 3 ? 0 : h.stop;
    *nblocks = h.blocks;
    *nirr = h.irr_steps;
    *tblock = h.tblock;
    *nact = h.last_nact;
    I.time_grav += nb6_wtime() - t0;
    I.num_fcall += (unsigned long long)h.blocks;
    I.num_steps += (unsigned long long)h.irr_steps;
}

void blocks_active_impl(int *nact, int *addr, double *rows) {
    if (!I.open || !I.hermite || !I.hctl.ptr) {
        nb6_fatal(NB6_ERR_NOT_OPEN);
        return;
    }
    const int na = I.hctl.ptr->last_nact;
    *nact = na;
    if (na <= 0) return;
    cudaStream_t st = nb6_stream();
    NB6_CUDA_CHECK(cudaMemcpyAsync(addr, I.bact_last ? I.bact_last : I.bact.ptr, sizeof(int) * na,
                                   cudaMemcpyDeviceToHost, st));
    NB6_CUDA_CHECK(cudaMemcpyAsync(rows, I.brows.ptr, sizeof(double) * 24 * (size_t)na, cudaMemcpyDeviceToHost, st));
    NB6_CUDA_CHECK(cudaStreamSynchronize(st));
    for (int k = 0; k < na; ++k) addr[k] += 1;
}

__global__ void iota_kernel(int n, int *v) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) v[k] = k;
}

// The due list in address order: 1-based addresses and the x0, v0 rows
// permuted to match.
// keys: sorted 0-based addresses, slot: their append slots; out: 1-based
// addresses and each body's x0, v0 in that order
__global__ void due_gather(int n, const int *__restrict__ keys, const int *__restrict__ slot,
                           const double *__restrict__ xv, int *__restrict__ addr, double *__restrict__ out) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        addr[k] = keys[k] + 1;
        const double *src = xv + 6 * (size_t)slot[k];
        for (int d = 0; d < 6; ++d) out[6 * (size_t)k + d] = src[d];
    }
}

// The same for a short due list in one launch: one CTA holds the n keys in
// shared memory and each key's place is the number of keys before it in
// (key, slot) order, so the result is the sort's.
constexpr int DUE_RANK_MAX = 2048, DUE_RANK_NT = 1024;
__global__ void __launch_bounds__(DUE_RANK_NT) due_rank(int n, const int *__restrict__ keys,
                                                        const double *__restrict__ xv, int *__restrict__ addr,
                                                        double *__restrict__ out) {
    __shared__ int sk[DUE_RANK_MAX];
    for (int q = threadIdx.x; q < n; q += DUE_RANK_NT) sk[q] = keys[q];
    __syncthreads();
    for (int q = threadIdx.x; q < n; q += DUE_RANK_NT) {
        const int k = sk[q];
        int r = 0;
        for (int p = 0; p < n; ++p) {
            const int kp = sk[p];
            r += (kp < k) | ((kp == k) & (p < q));
        }
        addr[r] = k + 1;
        const double *src = xv + 6 * (size_t)q;
        for (int d = 0; d < 6; ++d) out[6 * (size_t)r + d] = src[d];
    }
}

void blocks_regular_impl(int *nreg, int *addr, double *xv) {
    if (!I.open || !I.hermite || !I.hctl.ptr) {
        nb6_fatal(NB6_ERR_NOT_OPEN);
        return;
    }
    const int nr = I.hctl.ptr->nreg;
    *nreg = nr;
    if (nr <= 0) return;
    cudaStream_t st = nb6_stream();
    // ascending addresses (the device appends in no particular order), then
    // [x0, v0 of each | 1-based addresses] in one device block, one
    // download into pinned staging and two copies into the caller's arrays.
    // Up to NB6_DUE_SORT_MIN bodies (default 2,048) one launch ranks the
    // keys; longer lists take a radix sort of (address, slot).
    const size_t nd = 6 * (size_t)nr + ((size_t)nr + 1) / 2;
    I.dout.reserve(nd);
    I.hout.reserve(nd);
    double *dxv = I.dout.ptr;
    int *daddr = reinterpret_cast<int *>(I.dout.ptr + 6 * (size_t)nr);
    const char *e = getenv("NB6_DUE_SORT_MIN");
    const int rank_max = std::min(DUE_RANK_MAX, e ? atoi(e) : DUE_RANK_MAX);
    if (nr <= rank_max) {
        due_rank<<<1, DUE_RANK_NT, 0, st>>>(nr, I.breg.ptr, I.bregxv.ptr, daddr, dxv);
    } else {
        I.bsort.reserve(3 * (size_t)nr);
        int *keys_out = I.bsort.ptr, *vals_in = I.bsort.ptr + nr, *vals_out = I.bsort.ptr + 2 * (size_t)nr;
        const int g = std::min((nr + 255) / 256, nb6_num_sms() * 4);
        iota_kernel<<<g, 256, 0, st>>>(nr, vals_in);
        int bits = 1;
        while (bits < 31 && (1 << bits) < I.nmax) ++bits;
        size_t tmp = 0;
        NB6_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, tmp, I.breg.ptr, keys_out, vals_in, vals_out, nr, 0,
                                                       bits, st));
        I.bsort_tmp.reserve(tmp + 16);
        NB6_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(I.bsort_tmp.ptr, tmp, I.breg.ptr, keys_out, vals_in, vals_out,
                                                       nr, 0, bits, st));
        due_gather<<<g, 256, 0, st>>>(nr, keys_out, vals_out, I.bregxv.ptr, daddr, dxv);
    }
    NB6_CUDA_CHECK(cudaGetLastError());
    NB6_CUDA_CHECK(cudaMemcpyAsync(I.hout.ptr, I.dout.ptr, sizeof(double) * nd, cudaMemcpyDeviceToHost, st));
    NB6_CUDA_CHECK(cudaStreamSynchronize(st));
    memcpy(xv, I.hout.ptr, sizeof(double) * 6 * (size_t)nr);
    memcpy(addr, I.hout.ptr + 6 * (size_t)nr, sizeof(int) * (size_t)nr);
}

void hermite_get_impl(int a0, int n, double *out) {
    if (!I.open || !I.hermite) {
        nb6_fatal(NB6_ERR_NOT_OPEN);
        return;
    }
    if (n <= 0) return;
    if (a0 < 1 || (long long)a0 - 1 + n > I.nmax) {
        fprintf(stderr, "nb6_hermite_get: range outside [1, %d]\n", I.nmax);
        nb6_fatal(NB6_ERR_BAD_ARG);
        return;
    }
    cudaStream_t st = nb6_stream();
    irr_flush(st);
    I.dout.reserve((size_t)n * 32);
    hermite_gather<<<(n + 127) / 128, 128, 0, st>>>(a0 - 1, n, I.rec.ptr, I.aux.ptr, I.dout.ptr);
    NB6_CUDA_CHECK(cudaGetLastError());
    NB6_CUDA_CHECK(cudaMemcpyAsync(out, I.dout.ptr, sizeof(double) * 32 * (size_t)n, cudaMemcpyDeviceToHost, st));
    NB6_CUDA_CHECK(cudaStreamSynchronize(st));
}

void regf_correct_impl(double time, int ni, const int *addr, int *iseg, int nseg, int *seg_j0, const int *seg_a0,
                       double *h2, double *dtr, const double *rs, double (*xi)[3], double (*vi)[3], int lmax,
                       int nnbmax, int mflag, const double *prm, double *out) {
    if (!I.open || !I.hermite) {
        nb6_fatal(NB6_ERR_NOT_OPEN);
        return;
    }
    if (ni <= 0) return;
    bool bad = lmax > I.lmax || nseg <= 0;
    for (int k = 0; k < ni && !bad; ++k) bad = addr[k] < 1 || addr[k] > I.nmax;
    for (int c = 0; c < nseg && !bad; ++c) bad = seg_a0[c] < 1 || seg_a0[c] > I.nmax;
    if (bad) {
        fprintf(stderr, "nb6_regf_correct: bad address, segment or lmax (> %d)\n", I.lmax);
        nb6_fatal(NB6_ERR_BAD_ARG);
        return;
    }
    const double t0 = nb6_wtime();
    cudaStream_t st = nb6_stream();
    irr_flush(st);  // state staged by the host first
    RegDeviceOut ro;
    if (!regular_seg_on_device(ni, iseg, h2, dtr, xi, vi, lmax, nnbmax, mflag, nseg, seg_j0, &ro)) return;
    const double t1 = nb6_wtime();
    // [addr | iseg | seg_j0 (nseg+1) | seg_a0 - 1 (nseg) | pad | rs (ni doubles)]
    const size_t nint = 2 * (size_t)ni + 2 * (size_t)nseg + 1, nint2 = (nint + 1) & ~(size_t)1;
    I.hseg.reserve(nint2 + 2 * (size_t)ni);
    I.dseg.reserve(nint2 + 2 * (size_t)ni);
    int *h = I.hseg.ptr;
    memcpy(h + nint2, rs, sizeof(double) * ni);
    memcpy(h, addr, sizeof(int) * ni);
    memcpy(h + ni, iseg, sizeof(int) * ni);
    memcpy(h + 2 * (size_t)ni, seg_j0, sizeof(int) * (nseg + 1));
    for (int c = 0; c < nseg; ++c) h[2 * (size_t)ni + nseg + 1 + c] = seg_a0[c] - 1;
    NB6_CUDA_CHECK(cudaMemcpyAsync(I.dseg.ptr, h, sizeof(int) * (nint2 + 2 * (size_t)ni), cudaMemcpyHostToDevice,
                                   st));
    const int *d = I.dseg.ptr;
    const double *drs = reinterpret_cast<const double *>(I.dseg.ptr + nint2);
    RegCorrParams p;
    p.eta_r = prm[0];
    p.smax = prm[1];
    p.dtmin = prm[2];
    p.rsfac = prm[3];
    p.nnbopt = (int)prm[4];
    p.nnbmax = nnbmax;
    p.cap = std::max(0, std::min(nnbmax, lmax - 1));
    p.mlp_mode = (int)prm[5];
    p.nb_flag = I.ac_nb_flag;
    p.m_flag = mflag ? 1 : 0;
    p.nacl = I.nacl;
    p.acl_a0 = I.acl_a0.ptr;
    p.acpar = I.acpar.ptr;
    const size_t rowd = 32;
    I.hout.reserve((size_t)ni * rowd);
    const bool direct = sizeof(double) * rowd * (size_t)ni <= zero_copy_out_bytes();
    double *o = I.hout.ptr;
    if (!direct) {
        I.dout.reserve((size_t)ni * rowd);
        o = I.dout.ptr;
    }
    reg_corrector_kernel<<<(ni + 127) / 128, 128, 0, st>>>(ni, d, d + ni, d + 2 * (size_t)ni,
                                                         d + 2 * (size_t)ni + nseg + 1, time, ro, I.rec.ptr, I.aux.ptr,
                                                         I.lists.ptr, I.lmax, drs, p, o, nb6_dev_status(),
                                                         I.tn.ptr);
    NB6_CUDA_CHECK(cudaGetLastError());
    if (!direct)
        NB6_CUDA_CHECK(cudaMemcpyAsync(I.hout.ptr, o, sizeof(double) * rowd * ni, cudaMemcpyDeviceToHost, st));
    nb6_status_fetch(st);
    const double t2 = nb6_wtime();
    NB6_CUDA_CHECK(cudaStreamSynchronize(st));
    const double t3 = nb6_wtime();
    if (nb6_check_dev_status() != 0) return;
    memcpy(out, I.hout.ptr, sizeof(double) * rowd * ni);
    for (int k = 0; k < ni; ++k)
        if (out[rowd * k + 28] == 0.0) {
            const int nn = (int)out[rowd * k + 27];
            I.nnb_total += nn - I.nnb_host[addr[k] - 1];
            I.nnb_host[addr[k] - 1] = nn;
        }
    const double t4 = nb6_wtime();
    I.time_grav += t4 - t0;
    I.rc_calls++;
    I.rc_t[0] += t1 - t0;  // regular force enqueued (host preparation)
    I.rc_t[1] += t2 - t1;  // corrector enqueued
    I.rc_t[2] += t3 - t2;  // waiting for the device
    I.rc_t[3] += t4 - t3;  // results out
}

// The regular-force j set from the resident records: segments of
// consecutive addresses, predicted to t on the device (see irr_predict_pack).
void irr_predict_send_impl(double t, int nseg, const int *addr0, const int *count) {
    if (!I.open) {
        nb6_fatal(NB6_ERR_NOT_OPEN);
        return;
    }
    long long n = 0;
    bool bad = nseg <= 0;
    for (int s = 0; s < nseg && !bad; ++s) {
        bad = count[s] < 0 || addr0[s] < 1 || (long long)addr0[s] - 1 + count[s] > I.nmax;
        n += count[s];
    }
    if (bad || n > INT_MAX / 4) {
        fprintf(stderr, "nb6_irr_predict_send: segment outside [1, %d]\n", I.nmax);
        nb6_fatal(NB6_ERR_BAD_ARG);
        return;
    }
    cudaStream_t st = nb6_stream();
    irr_flush(st);  // records staged by set_jp must be on the device first
    double *jm, *jx, *jv;
    JSetOut o;
    if (!regular_bind_j((int)n, &jm, &jx, &jv, &o)) return;
    // [segoff (nseg+1) | addr0 - 1 (nseg)]
    I.hseg.reserve(2 * (size_t)nseg + 1);
    I.dseg.reserve(2 * (size_t)nseg + 1);
    int *h = I.hseg.ptr;
    h[0] = 0;
    for (int s = 0; s < nseg; ++s) {
        h[s + 1] = h[s] + count[s];
        h[nseg + 1 + s] = addr0[s] - 1;
    }
    NB6_CUDA_CHECK(cudaMemcpyAsync(I.dseg.ptr, h, sizeof(int) * (2 * (size_t)nseg + 1),
                                   cudaMemcpyHostToDevice, st));
    const int blocks = (int)std::min<size_t>((o.npad + 255) / 256, (size_t)nb6_num_sms() * 8);
    irr_predict_pack<<<blocks, 256, 0, st>>>((int)n, t, nseg, I.dseg.ptr, I.dseg.ptr + nseg + 1, I.rec.ptr,
                                             jm, jx, jv, o, nb6_dev_status());
    NB6_CUDA_CHECK(cudaGetLastError());
    // the host table may be rewritten by the next call: wait for the copy
    NB6_CUDA_CHECK(cudaStreamSynchronize(st));
}

void irr_profile_impl(int rank) {
    if (I.open && I.rc_calls && getenv("NB6_VERBOSE"))
        fprintf(stderr,
                "[R.%d GPU Reg.C ] Ncall: %lld prepare+force %.3f s, corrector %.3f s, wait %.3f s, out %.3f s\n",
                rank, I.rc_calls, I.rc_t[0], I.rc_t[1], I.rc_t[2], I.rc_t[3]);
    I.rc_calls = 0;
    I.rc_t[0] = I.rc_t[1] = I.rc_t[2] = I.rc_t[3] = 0;
    if (I.open && I.num_fcall) {
        const double gf = I.time_grav > 0 ? 60.0 * (double)I.num_inter * 1e-9 / I.time_grav : 0.0;
        fprintf(stderr, "[R.%d GPU Irr.F ] Ncall: %llu <NI>: %d grav: %f s, %f Gflops, %f usec\n", rank,
                I.num_fcall, (int)(I.num_steps / I.num_fcall), I.time_grav, gf,
                1e6 * I.time_grav / (double)I.num_fcall);
    }
    I.time_grav = 0;
    I.num_inter = I.num_fcall = I.num_steps = 0;
}

}  // namespace

// Radius-rule quantities per cluster for the device regular corrector.
void hermite_adjust_impl(int nb_flag, int ncl, const int *a0, const double *par) {
    if (!I.open) {
        nb6_fatal(NB6_ERR_NOT_OPEN);
        return;
    }
    bool bad = ncl < 0 || (ncl > 0 && (a0[0] < 1 || a0[ncl] > I.nmax + 1));
    for (int c = 0; c < ncl && !bad; ++c) bad = a0[c + 1] < a0[c];
    for (int c = 0; c < 8 * ncl && !bad; ++c) bad = par[c] != par[c];
    if (bad) {
        fprintf(stderr, "nb6_hermite_adjust: bad cluster table\n");
        nb6_fatal(NB6_ERR_BAD_ARG);
        return;
    }
    I.ac_nb_flag = nb_flag ? 1 : 0;
    I.nacl = ncl;
    if (ncl == 0) return;
    cudaStream_t st = nb6_stream();
    std::vector<int> h(ncl + 1);
    for (int c = 0; c <= ncl; ++c) h[c] = a0[c] - 1;
    I.acl_a0.reserve((size_t)ncl + 1);
    I.acpar.reserve(8 * (size_t)ncl);
    NB6_CUDA_CHECK(cudaMemcpyAsync(I.acl_a0.ptr, h.data(), sizeof(int) * (ncl + 1), cudaMemcpyHostToDevice, st));
    NB6_CUDA_CHECK(cudaMemcpyAsync(I.acpar.ptr, par, sizeof(double) * 8 * ncl, cudaMemcpyHostToDevice, st));
    NB6_CUDA_CHECK(cudaStreamSynchronize(st));
}

// Row lengths of the bodies addr[0 .. n) (0-based), capped at cap ids.
__global__ void lists_count(int n, const int *__restrict__ addr, const int *__restrict__ lists, int ls, int cap,
                            int *__restrict__ cnt) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int c = lists[(size_t)addr[k] * ls];
    cnt[k] = min(max(c, 0), cap);
}

// One warp per body: its row [nnb, ids] packed at offs[k], ids 1-based.
__global__ void lists_pack(int n, const int *__restrict__ addr, const int *__restrict__ lists, int ls,
                           const int *__restrict__ cnt, const long long *__restrict__ offs, int *__restrict__ packed) {
    const int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (k >= n) return;
    const int *row = lists + (size_t)addr[k] * ls;
    int *o = packed + offs[k];
    const int c = cnt[k];
    if (lane == 0) o[0] = c;
    for (int l = lane; l < c; l += 32) o[1 + l] = row[1 + l] + 1;
}

void lists_get_impl(int n, const int *addr, int ls, int *out) {
    if (!I.open) {
        nb6_fatal(NB6_ERR_NOT_OPEN);
        return;
    }
    if (n <= 0) return;
    bool bad = ls < 1;
    for (int k = 0; k < n && !bad; ++k) bad = addr[k] < 1 || addr[k] > I.nmax;
    if (bad) {
        fprintf(stderr, "nb6_irr_lists_get: address outside [1, %d] or ls < 1\n", I.nmax);
        nb6_fatal(NB6_ERR_BAD_ARG);
        return;
    }
    cudaStream_t st = nb6_stream();
    irr_flush(st);
    const int cap = std::min(I.lmax, ls) - 1;
    const size_t nn = (size_t)n;
    // [counts n | pad | offsets n (long long) | addresses n, 0-based] on the
    // device; [counts | pad | offsets] on the host; then the packed rows
    const size_t noff = (nn + 1) & ~(size_t)1;
    I.lg_dev.reserve(noff + 3 * nn + 2);
    I.lg_host.reserve(noff + 3 * nn + 2);
    int *dcnt = I.lg_dev.ptr;
    int *daddr = I.lg_dev.ptr + noff + 2 * nn;
    int *haddr = I.lg_host.ptr + noff + 2 * nn;
    for (size_t k = 0; k < nn; ++k) haddr[k] = addr[k] - 1;
    NB6_CUDA_CHECK(cudaMemcpyAsync(daddr, haddr, sizeof(int) * nn, cudaMemcpyHostToDevice, st));
    lists_count<<<(n + 255) / 256, 256, 0, st>>>(n, daddr, I.lists.ptr, I.lmax, cap, dcnt);
    NB6_CUDA_CHECK(cudaGetLastError());
    NB6_CUDA_CHECK(cudaMemcpyAsync(I.lg_host.ptr, dcnt, sizeof(int) * nn, cudaMemcpyDeviceToHost, st));
    NB6_CUDA_CHECK(cudaStreamSynchronize(st));
    long long *hoff = reinterpret_cast<long long *>(I.lg_host.ptr + noff);
    long long tot = 0;
    for (size_t k = 0; k < nn; ++k) {
        hoff[k] = tot;
        tot += 1 + I.lg_host.ptr[k];
    }
    long long *doff = reinterpret_cast<long long *>(I.lg_dev.ptr + noff);
    NB6_CUDA_CHECK(cudaMemcpyAsync(doff, hoff, sizeof(long long) * nn, cudaMemcpyHostToDevice, st));
    DevBuf<int> dpk;
    HostBuf<int> hpk;
    dpk.reserve((size_t)tot);
    hpk.reserve((size_t)tot);
    lists_pack<<<(unsigned)((nn * 32 + 255) / 256), 256, 0, st>>>(n, daddr, I.lists.ptr, I.lmax, dcnt, doff, dpk.ptr);
    NB6_CUDA_CHECK(cudaGetLastError());
    NB6_CUDA_CHECK(cudaMemcpyAsync(hpk.ptr, dpk.ptr, sizeof(int) * tot, cudaMemcpyDeviceToHost, st));
    NB6_CUDA_CHECK(cudaStreamSynchronize(st));
    for (size_t k = 0; k < nn; ++k) {
        const int *src = hpk.ptr + hoff[k];
        int *row = out + k * (size_t)ls;
        const int c = src[0];
        memcpy(row, src, sizeof(int) * (size_t)(1 + c));
        for (int l = 1 + c; l < std::min(ls, 1 + c + 8); ++l) row[l] = 0;
    }
    dpk.release();
    hpk.release();
}

extern "C" {

void irr_simd_open_(int *nmax, int *lmax, int *rank) { irr_open_impl(*nmax, *lmax, *rank); }
void irr_simd_close_(int *rank) { (void)rank; irr_close_impl(); }
void irr_simd_profile_(int *rank) { irr_profile_impl(*rank); }
void irr_simd_set_jp_(int *addr, double pos[3], double vel[3], double acc2[3], double jrk6[3],
                      double *mass, double *time) {
    irr_set_jp_impl(*addr - 1, pos, vel, acc2, jrk6, *mass, *time);
}
void irr_simd_set_list_(int *addr, int *nblist) { irr_set_list_impl(*addr - 1, nblist); }
void irr_simd_firr_vec_(double *ti, int *ni, int addr[], double acc[][3], double jrk[][3],
                        int nnbid[]) {
    irr_firr_vec_impl(*ti, *ni, addr, acc, jrk, nnbid);
}

// NBODY6/GPU names (fpoly0.F:42,70,202,383, intgrt.F:1329 -- commented out
// in the reference): same arguments, rank 0.
void gpuirr_open_(int *nmax, int *lmax) { irr_open_impl(*nmax, *lmax, 0); }
void gpuirr_close_() { irr_close_impl(); }
void gpuirr_set_jp_(int *addr, double pos[3], double vel[3], double acc2[3], double jrk6[3],
                    double *mass, double *time) {
    irr_set_jp_impl(*addr - 1, pos, vel, acc2, jrk6, *mass, *time);
}
void gpuirr_set_list_(int *addr, int *nblist) { irr_set_list_impl(*addr - 1, nblist); }

// Extensions (no reference counterpart): the irregular corrector on the
// device (the host's NBINT_COR / intgrt.F:533-581 work for each active body).
// nb6_hermite_open_ allocates the per-body corrector state beside the records
// (after irr_simd_open_); nb6_hermite_set_ stages a body's FI, FIDOT, FR,
// FRDOT (irregular and regular force and derivative), STEP, T0R, STEPR, the
// way irr_simd_set_jp_ stages its position record.  nb6_irr_correct_ then
// does, for the active bodies at *time: neighbour force, Hermite corrector,
// new irregular step, the regular-due test and, when no regular step is due,
// the F/FDOT extrapolation -- updating the device state and returning per body
// out[k][24] = x0[3], v0[3], fi[3], fidot[3], F[3], FDOT[3], step,
// regular-due (0/1), nnbid, 0, 0, 0.
void nb6_hermite_open_(double *eta_i, double *smax, double *dtmin) { hermite_open_impl(*eta_i, *smax, *dtmin); }
void nb6_hermite_set_(int *addr, double fi[3], double fidot[3], double fr[3], double frdot[3], double *step,
                      double *t0r, double *stepr, double *rs) {
    hermite_set_impl(*addr - 1, fi, fidot, fr, frdot, *step, *t0r, *stepr, *rs);
}
void nb6_irr_correct_(double *time, int *ni, int *addr, double *out) { irr_correct_impl(*time, *ni, addr, out); }

// KS pairs whose components the irregular force resolves, replacing the
// table of the previous call (npair = 0 clears it).  Pair p: the c.m. body
// cm[p] (1-based address), its components' positions xk[p][2][3] and
// velocities vk[p][2][3] at the time of the coming irregular calls, their
// masses mk[p][2], and the perturber list (LIST(2..,I1) of the first
// component) plist[pofs[p] .. pofs[p+1]) (1-based, pofs[0] = 0).  Every
// following irr_simd_firr_vec_ / nb6_irr_correct_ returns FIRR and FD with
// the corrections NBINT_COR adds on the host (cmfirr_cor.f,
// cmfirr_ucor.f; nbint_cor.f:37-65), so a caller skips its own CMFIRR_COR
// and CMFIRR_UCOR.  Only perturbed pairs are listed: an unperturbed pair
// acts as its c.m. point mass, as in the reference.
void nb6_ks_set_(int *npair, int *cm, double *xk, double *vk, double *mk, int *pofs, int *plist) {
    ks_set_impl(*npair, cm, xk, vk, mk, pofs, plist);
}

// Device block clock: run blocks of irregular steps on the device (each
// block: the earliest t0 + STEP over all bodies, its active set, the
// neighbour force and the irregular corrector, as nb6_irr_correct_ does
// for a host-chosen set) until a block has a body due a regular step (its
// irregular part done: *reason = 1, the host runs the regular part with
// nb6_blocks_active_ and nb6_regf_correct_), the next block time passes
// *tlimit (*reason = 2, that block not started) or *max_blocks blocks ran
// (*reason = 0).  *nblocks and *nirr count the blocks and irregular steps
// of this call, *tblock is the last block's time, *nact its active count.
// The host's block clock is not needed meanwhile (next_tlist.f's choice is
// made on the device, bit for bit the same).
void nb6_blocks_mode_(int *persistent) { I.blk_persist = *persistent ? 1 : 0; }

void nb6_irr_pv_(int *mode) { I.pv_mode = (*mode >= 0 && *mode <= 2) ? *mode : 1; }
void nb6_irr_tune_(int *chunks) { I.chunks_max = (*chunks >= 1 && *chunks <= IRR_CHUNKS) ? *chunks : IRR_CHUNKS; }

void nb6_blocks_run_(double *tlimit, int *max_blocks, int *reason, long long *nblocks, long long *nirr,
                     double *tblock, int *nact) {
    blocks_run_impl(*tlimit, *max_blocks, reason, nblocks, nirr, tblock, nact);
}

// The last block of nb6_blocks_run_: its active bodies (1-based, in no
// particular order) and their corrector rows out[k][24] as nb6_irr_correct_
// returns them.
void nb6_blocks_active_(int *nact, int *addr, double *rows) { blocks_active_impl(nact, addr, rows); }

// The bodies of the last block of nb6_blocks_run_ that are due a regular
// step (*reason = 1): *nreg of them, ascending 1-based addresses, with
// their corrected x0[3], v0[3] (xv[k][6]) -- the i of nb6_regf_correct_.
void nb6_blocks_regular_(int *nreg, int *addr, double *xv) { blocks_regular_impl(nreg, addr, xv); }

// The resident state of bodies a0 .. a0+n-1 (1-based), rows of 32
// doubles: x0[3], v0[3], F[3], FDOT[3], fi[3], fidot[3], fr[3], frdot[3],
// t0, step, t0r, stepr, rs, mass, 0, 0.
void nb6_hermite_get_(int *a0, int *n, double *out) { hermite_get_impl(*a0, *n, out); }

// Regular force plus the regular corrector on the device for the bodies
// addr[ni] (1-based, grouped by segment iseg[k]; segment c is the j range
// [seg_j0[c], seg_j0[c+1]) of the current j set and holds the bodies from
// address seg_a0[c] on, as nb6_irr_predict_send_ lays them out).  h2, dtr,
// xi, vi, lmax, nnbmax, m_flag as for nb6_regf_seg_.  prm = {ETAR, SMAX,
// DTMIN, 25 / TCR, NNBOPT, learned-radius mode (0 or 2)}; rs[k] is the
// radius body k's h2 was formed from (the device copy is replaced by the
// corrector's result).  For every body
// whose list fits: the Ahmad-Cohen radius update, the neighbour gain/loss
// force moves, the corrector, the new regular step and, in mode 2, the
// learned proposal -- updating the resident state and neighbour list --
// with out[k][32] = x0[3], v0[3], fi[3], fidot[3], fr[3], frdot[3], F[3],
// FDOT[3], step, stepr, rs, nnb, overflow (-nnb, else 0), learned outcome,
// 0, 0.  Overflowed bodies are left untouched for the caller's radius
// shrink and retry with the smaller rs (util_gpu.F:69-100).
void nb6_regf_correct_(double *time, int *ni, int *addr, int *iseg, int *nseg, int *seg_j0, int *seg_a0,
                       double *h2, double *dtr, double *rs, double (*xi)[3], double (*vi)[3], int *lmax,
                       int *nnbmax, int *m_flag, double *prm, double *out) {
    regf_correct_impl(*time, *ni, addr, iseg, *nseg, seg_j0, seg_a0, h2, dtr, rs, xi, vi, *lmax, *nnbmax, *m_flag,
                      prm, out);
}

// Extension (no reference counterpart): device time (ms) of the force
// kernel of the last irr_simd_firr_vec_ call.
float nb6_irr_last_kernel_ms_() {
    if (!I.ev1) return 0.f;
    float ms = 0.f;
    NB6_CUDA_CHECK(cudaEventSynchronize(I.ev1));
    NB6_CUDA_CHECK(cudaEventElapsedTime(&ms, I.ev0, I.ev1));
    return ms;
}

// Extension (no reference counterpart): make the regular-force j set (what
// gpunb_send_ sends) from the resident irregular records, predicted to *t on
// the device.  Segment s is the count[s] records from 1-based address
// addr0[s]; segments are laid out back to back in the j set.  Records staged
// by irr_simd_set_jp_ are uploaded first.  Replaces XBPREDALL + GPUNB_SEND
// (intgrt.F:866-882) with no host prediction and no j upload.
void nb6_irr_predict_send_(double *t, int *nseg, int *addr0, int *count) {
    irr_predict_send_impl(*t, *nseg, addr0, count);
}

// Extension (no reference counterpart; the reference keeps these in common
// blocks, set by ADJUST and CORE, adjust.F:104-199, core.f): the Ahmad-Cohen
// radius rule's quantities for the device regular corrector.  *nb_flag
// selects the rule's form (NB_FLAG of regcor_gpu.F:22: 1 for KZ(39) = 0 or
// 2).  Cluster c holds the bodies of 1-based addresses [a0[c], a0[c+1])
// (a0 has *ncl + 1 entries) and par[8c .. 8c+7] = RDENS[3], RSCALE, RC2,
// RSFAC, BODYM, 0.  Without a table (*ncl = 0) each segment of a call is
// its own cluster with RDENS = 0, RSCALE = RC2 = 1, RSFAC = prm[3] and
// BODYM = 1 / (its body count).
void nb6_hermite_adjust_(int *nb_flag, int *ncl, int *a0, double *par) { hermite_adjust_impl(*nb_flag, *ncl, a0, par); }

// Extension (no reference counterpart): the resident neighbour rows of the
// *n bodies of 1-based addresses addr[] into out[*n][*ls], each [nnb,
// 1-based ids ascending] (at most *ls - 1 ids), zeros over the 8 entries
// after the last id.  For a host that lets the device regular corrector keep
// the lists (density centre, core.f).
void nb6_irr_lists_get_(int *n, const int *addr, int *ls, int *out) { lists_get_impl(*n, addr, *ls, out); }

}  // extern "C"
