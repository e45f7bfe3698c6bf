// hermite.h -- per-body pieces of the Hermite 4th-order block-step scheme
// with the Ahmad-Cohen neighbour split, shared by the single-cluster driver
// (blockstep.cpp) and the ensemble driver (ensemble.cpp).
//
// Restated from the reference's integrator (single stars only):
//   irregular corrector + step   nbint_cor.f:113-173,215-236, tstep.f
//   F, FDOT between regular steps intgrt.F:558-581
//   regular corrector            regcor_gpu.F:131-196 (radius update),
//                                :284-444 (neighbour gain/loss force moves),
//                                :442-537 (corrector), :593-737 (new step)
//   initial steps                fpoly0.F:55-59,100-206
// Bodies keep the reference's Fortran names in lower case (X0, X0DOT, T0,
// STEP, T0R, STEPR, FI, FIDOT, D2, D3, FR, FRDOT, D2R, D3R, F, FDOT, RS,
// LIST); neighbour rows hold 1-based body addresses, self excluded.
#pragma once

#include <dlfcn.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <algorithm>
#include <map>
#include <thread>
#include <vector>

extern "C" {

// Run parameters (names follow the reference's input namelist, input.F).
struct nb6drive_params {
    double eta_i, eta_r;   // ETAI, ETAR
    double smax;           // SMAX, power of two
    double dtmin;          // smallest allowed step (power of two)
    double tcrit;          // end time
    double dt_out;         // energy output interval (power of two, >= smax)
    double rs0;            // initial neighbour radius scale (fpoly0.F:55)
    int nnbopt, nnbmax, lmax, m_flag;
    int chunk;             // i per gpunb_regf call (util_gpu.F: 1024)
    long long max_blocks;  // safety bound on the number of block steps
    // learned neighbour radius: 0 = Ahmad-Cohen only; 1 = Ahmad-Cohen and
    // log (features, target) samples into samples[sample_cap][6]; 2 = the
    // library's proposals, Ahmad-Cohen as fallback
    int mlp_mode;
    int mlp_pad;
    float *samples;
    long long sample_cap;
    // optional initial neighbour radii (one per body); null = RS0 sqrt(1+r^2)
    // (fpoly0.F:55), the reference's rule with RS0 from the input file
    const double *rs_init;
    // ensemble driver, batched mode: 0 = correctors on the host; 1 =
    // irregular corrector on the device (nb6_irr_correct_) when the backend
    // has it; 2 = the regular corrector there too (nb6_regf_correct_; the
    // host one under mlp_mode 1, which logs samples on the host); 3 = the
    // block clock too (nb6_blocks_run_: runs of irregular blocks on the
    // device, the host only for regular steps and output)
    int dev_corrector;
    // ensemble driver, batched mode: 1 = a block whose regular bodies all
    // belong to one cluster also takes the segmented call (nb6_regf_seg_,
    // as the device regular corrector does); 0 = gpunb_regf_ for it
    int seg_single;
    // form of the Ahmad-Cohen radius rule, NB_FLAG of regcor_gpu.F:22 /
    // util_gpu.F:29 (KZ(39) = 0 or 2 give 1, the reference's default):
    // 1 = distances from the density centre, membership reduced outside
    // the half-mass radius, radial-velocity volume factor, overflow shrink
    // by (NNBOPT/NNB)^0.333; 0 = distances from the origin, overflow shrink
    // by 0.9
    int nb_flag;
    // interval of the radius rule's adjust times (DTADJ of input.F): the
    // quantities are refreshed at TIME = 0 and at the first energy output at
    // or after each multiple of it
    double dt_adj;
};

// Counters returned by the drivers.
struct nb6drive_stats {
    long long blocks, irr_steps, reg_steps, reg_calls, overflow_retries;
    long long nb_sum;       // sum of neighbour counts over regular steps
    long long reg_pairs;    // sum of ni * nj over regular-force calls
    double wall_reg, wall_irr, wall_total;
    double t_end;
    int nout;
    long long nsamples;      // samples logged (mlp_mode 1)
    long long mlp_used;      // regular steps that took the learned radius (mlp_mode 2)
    long long mlp_fallback;  // ... that fell back to the Ahmad-Cohen radius
    double nb_absdev;        // sum over regular steps of |nnb - NNBOPT|
};

}  // extern "C"

namespace nb6drv {

typedef void (*fn_open)(int *, int *);
typedef void (*fn_close)();
typedef void (*fn_send)(int *, double *, double (*)[3], double (*)[3]);
typedef void (*fn_regf)(int *, double *, double *, double (*)[3], double (*)[3], double (*)[3],
                        double (*)[3], double *, int *, int *, int *, int *);
typedef void (*fn_regf_seg)(int *, int *, double *, double *, double (*)[3], double (*)[3],
                            double (*)[3], double (*)[3], double *, int *, int *, int *, int *, int *,
                            int *);
typedef void (*fn_pred_send)(double *, int *, int *, int *);
typedef void (*fn_pot)(int *, int *, int *, int *, double *, double (*)[3], double *);
typedef void (*fn_irr_open)(int *, int *, int *);
typedef void (*fn_irr_close)(int *);
typedef void (*fn_irr_set_jp)(int *, double *, double *, double *, double *, double *, double *);
typedef void (*fn_irr_set_list)(int *, int *);
typedef void (*fn_irr_firr)(double *, int *, int *, double (*)[3], double (*)[3], int *);
typedef void (*fn_proposals)(int *, double *);
typedef void (*fn_profile)(int *);
typedef void (*fn_hermite_open)(double *, double *, double *);
typedef void (*fn_hermite_set)(int *, double *, double *, double *, double *, double *, double *, double *,
                               double *);
typedef void (*fn_irr_correct)(double *, int *, int *, double *);
typedef void (*fn_regf_correct)(double *, int *, int *, int *, int *, int *, int *, double *, double *, double *,
                                double (*)[3], double (*)[3], int *, int *, int *, double *, double *);
typedef void (*fn_hermite_get)(int *, int *, double *);
typedef void (*fn_blocks_run)(double *, int *, int *, long long *, long long *, double *, int *);
typedef void (*fn_blocks_active)(int *, int *, double *);
typedef void (*fn_blocks_regular)(int *, int *, double *);
typedef void (*fn_hermite_adjust)(int *, int *, int *, double *);
typedef void (*fn_lists_get)(int *, const int *, int *, int *);

struct Backend {
    void *hreg = nullptr, *hirr = nullptr, *hpot = nullptr;
    fn_open gpunb_open = nullptr;
    fn_close gpunb_close = nullptr;
    fn_send gpunb_send = nullptr;
    fn_regf gpunb_regf = nullptr;
    fn_pot gpupot = nullptr;
    fn_irr_open irr_open = nullptr;
    fn_irr_close irr_close = nullptr;
    fn_irr_set_jp irr_set_jp = nullptr;
    fn_irr_set_list irr_set_list = nullptr;
    fn_irr_firr irr_firr_vec = nullptr;
    // extensions of libnb6b200 (absent from the reference's libraries)
    fn_regf_seg regf_seg = nullptr;
    fn_pred_send predict_send = nullptr;
    fn_proposals proposals = nullptr;
    fn_profile reg_profile = nullptr, irr_profile = nullptr;  // the libraries' timing lines
    fn_hermite_open hermite_open = nullptr;                    // device irregular corrector
    fn_hermite_set hermite_set = nullptr;
    fn_irr_correct irr_correct = nullptr;
    fn_regf_correct regf_correct = nullptr;                    // device regular corrector
    fn_hermite_get hermite_get = nullptr;
    fn_blocks_run blocks_run = nullptr;                        // device block clock
    fn_blocks_active blocks_active = nullptr;
    fn_blocks_regular blocks_regular = nullptr;
    fn_hermite_adjust hermite_adjust = nullptr;                // radius-rule quantities per cluster
    fn_lists_get lists_get = nullptr;                          // resident neighbour rows
};

inline void *must_sym(void *h, const char *name) {
    void *p = dlsym(h, name);
    if (!p) fprintf(stderr, "nb6drive: missing symbol %s\n", name);
    return p;
}

inline bool load_backend(Backend &b, const char *reg, const char *irr, const char *pot) {
    b.hreg = dlopen(reg, RTLD_NOW | RTLD_LOCAL);
    b.hirr = dlopen(irr, RTLD_NOW | RTLD_LOCAL);
    b.hpot = dlopen(pot, RTLD_NOW | RTLD_LOCAL);
    if (!b.hreg || !b.hirr || !b.hpot) {
        fprintf(stderr, "nb6drive: dlopen failed: %s\n", dlerror());
        return false;
    }
    b.gpunb_open = (fn_open)must_sym(b.hreg, "gpunb_open_");
    b.gpunb_close = (fn_close)must_sym(b.hreg, "gpunb_close_");
    b.gpunb_send = (fn_send)must_sym(b.hreg, "gpunb_send_");
    b.gpunb_regf = (fn_regf)must_sym(b.hreg, "gpunb_regf_");
    b.gpupot = (fn_pot)must_sym(b.hpot, "gpupot_");
    b.irr_open = (fn_irr_open)must_sym(b.hirr, "irr_simd_open_");
    b.irr_close = (fn_irr_close)must_sym(b.hirr, "irr_simd_close_");
    b.irr_set_jp = (fn_irr_set_jp)must_sym(b.hirr, "irr_simd_set_jp_");
    b.irr_set_list = (fn_irr_set_list)must_sym(b.hirr, "irr_simd_set_list_");
    b.irr_firr_vec = (fn_irr_firr)must_sym(b.hirr, "irr_simd_firr_vec_");
    // optional: batched calls of libnb6b200, only when reg and irr are the
    // same library (the device j set comes from the irregular records)
    if (b.hreg == b.hirr) {
        b.regf_seg = (fn_regf_seg)dlsym(b.hreg, "nb6_regf_seg_");
        b.predict_send = (fn_pred_send)dlsym(b.hreg, "nb6_irr_predict_send_");
    }
    b.proposals = (fn_proposals)dlsym(b.hreg, "nb6_regf_proposals_");
    b.reg_profile = (fn_profile)dlsym(b.hreg, "gpunb_profile_");
    b.irr_profile = (fn_profile)dlsym(b.hirr, "irr_simd_profile_");
    b.hermite_open = (fn_hermite_open)dlsym(b.hirr, "nb6_hermite_open_");
    b.hermite_set = (fn_hermite_set)dlsym(b.hirr, "nb6_hermite_set_");
    b.irr_correct = (fn_irr_correct)dlsym(b.hirr, "nb6_irr_correct_");
    b.regf_correct = (fn_regf_correct)dlsym(b.hirr, "nb6_regf_correct_");
    b.hermite_get = (fn_hermite_get)dlsym(b.hirr, "nb6_hermite_get_");
    b.blocks_run = (fn_blocks_run)dlsym(b.hirr, "nb6_blocks_run_");
    b.blocks_active = (fn_blocks_active)dlsym(b.hirr, "nb6_blocks_active_");
    b.blocks_regular = (fn_blocks_regular)dlsym(b.hirr, "nb6_blocks_regular_");
    b.hermite_adjust = (fn_hermite_adjust)dlsym(b.hirr, "nb6_hermite_adjust_");
    b.lists_get = (fn_lists_get)dlsym(b.hirr, "nb6_irr_lists_get_");
    return b.gpunb_open && b.gpunb_close && b.gpunb_send && b.gpunb_regf && b.gpupot &&
           b.irr_open && b.irr_close && b.irr_set_jp && b.irr_set_list && b.irr_firr_vec;
}

inline double wtime() {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

// Constants of the reference's integrator (zero.f:113-116), multiplied as
// the Fortran multiplies them.
constexpr double ONE3 = 1.0 / 3.0, ONE6 = 1.0 / 6.0, ONE12 = 1.0 / 12.0;
// The reference is compiled without -fdefault-real-8: a real literal such
// as 0.6 is REAL*4 and enters a REAL*8 expression as its single-precision
// value; R4(0.6) writes that value.
#define R4(c) ((double)(c##f))

// Per-cluster quantities of the radius rule, refreshed at each adjust time
// (adjust.F:104-199, core.f): density centre RDENS, half-mass radius
// RSCALE, core radius squared RC2, RSFAC = MAX(25/TCR, 1.5 VC/RSMIN) and
// the mean mass BODYM.
struct ACPar {
    double rdens[3] = {0.0, 0.0, 0.0};
    double rscale = 1.0, rc2 = 1.0, rsfac = 0.0, bodym = 1.0;
};

// Ahmad-Cohen radius update of a single body at its regular step,
// regcor_gpu.F:19-238.  nnb: new membership (self removed), nnb0: old;
// xi, vi: the body at TIME; xnb, vnb: its first min(nnb, 3) new neighbours
// at TIME.  Returns the new RS; dfirr, dfd receive the irregular force
// change the neighbour moves start from (non-zero only for nnb = 0, the
// small central mass of :108-121).  Single-precision terms as the
// reference computes them (FLOAT() and literals are REAL*4).
inline double ac_radius(int nb_flag, int m_flag, int nnbopt, int nnbmax, const ACPar &a, int nnb,
                        int nnb0, double dtr, const double *xi, const double *vi, const double *xnb,
                        const double *vnb, double rs, double *dfirr, double *dfd) {
    const float zs = 0.01f * (float)nnbmax;                     // input.F:133
    const double znbmin = (double)(zs > 1.0f ? zs : 1.0f);
    for (int k = 0; k < 3; ++k) dfirr[k] = dfd[k] = 0.0;
    double ri2, rh2;
    if (nb_flag) {                                             // :30-37
        const double e0 = xi[0] - a.rdens[0], e1 = xi[1] - a.rdens[1], e2 = xi[2] - a.rdens[2];
        ri2 = e0 * e0 + e1 * e1 + e2 * e2;
        rh2 = a.rscale * a.rscale;
    } else {
        ri2 = xi[0] * xi[0] + xi[1] * xi[1] + xi[2] * xi[2];
        rh2 = R4(9.0) * (a.rscale * a.rscale);
    }
    if (nnb == 0) {                                            // :108-131
        const double r2 = xi[0] * xi[0] + xi[1] * xi[1] + xi[2] * xi[2];
        const double fij = R4(0.01) * a.bodym / (r2 * sqrt(r2));
        const double rdot = 3.0 * (xi[0] * vi[0] + xi[1] * vi[1] + xi[2] * vi[2]) / r2;
        for (int k = 0; k < 3; ++k) {
            dfirr[k] = -fij * xi[k];
            dfd[k] = -(vi[k] - rdot * xi[k]) * fij;
        }
        if (rdot > 0.0) return std::max(R4(0.75) * rs, R4(0.1) * a.rscale);
        return R4(1.1) * rs;
    }
    const float fac_s = 1.0f + 0.1f * ((float)nnbopt - (float)nnb) / (float)nnb;   // :139-150
    double a3 = (double)(float)nnb * (double)fac_s;
    const int nbave = std::min(nnbopt + 150, std::max(nnbmax - 50, (int)znbmin));
    const double cap = (double)(0.9f * (float)nbave);
    a3 = a3 < cap ? a3 : cap;
    const int nbp = (int)a3;
    if (ri2 > rh2 && nb_flag) {                                // :152-156
        const double f = a.rscale / sqrt(ri2);
        a3 = a3 * (f > R4(0.1) ? f : R4(0.1));
    } else {
        a3 = a3 > znbmin ? a3 : znbmin;
    }
    double a4 = a3 / (double)(float)nnb;
    if ((a3 - (double)(float)nnb0) * (a3 - (double)(float)nnb) < 0.0) a4 = sqrt(a4);
    const double ridot = (xi[0] - a.rdens[0]) * vi[0] + (xi[1] - a.rdens[1]) * vi[1] +
                         (xi[2] - a.rdens[2]) * vi[2];              // :162-164
    if (ri2 > a.rc2 && nb_flag && ri2 < R4(100.0) * rh2) a4 = a4 * (1.0 + ridot * dtr / ri2);
    // (:170-181, the perturber range of a c.m. body, applies to I > N only)
    double a5 = a.rsfac * dtr;                                 // :184-192
    a5 = a5 < 0.25 ? a5 : 0.25;
    a4 = a4 - 1.0;
    if (a4 > a5) a4 = a5;
    else a4 = a4 > -a5 ? a4 : -a5;
    const double a3b = ONE3 * a4;                              // :195-213
    double a1 = 1.0 + a3b - a3b * a3b;
    if (nnb < znbmin && nbp > znbmin && a1 < 1.0) a1 = R4(1.05);
    if (fabs(a1 - 1.0) > R4(0.003)) {
        if (rs * rs > ri2 && rs * rs < 2.0 * ri2 && nnb > 5) a1 = sqrt(a1);
        rs = a1 * rs;
    }
    if (nnb > nbave && ridot < 0.0) {                          // :215-220
        const float drs = ((float)nnb - (float)nbave) / (3.0f * (float)nnb);
        rs = rs * (1.0 - (double)drs);
    }
    if (!m_flag && nnb <= 3 && ri2 < R4(100.0) * rh2) {        // :223-238
        double b1 = 2.0 * rs;
        for (int l = 0; l < nnb; ++l) {
            const double *xj = xnb + 3 * l, *vj = vnb + 3 * l;
            const double e0 = xi[0] - xj[0], e1 = xi[1] - xj[1], e2 = xi[2] - xj[2];
            const double rij = sqrt(e0 * e0 + e1 * e1 + e2 * e2);
            const double rsdot = (e0 * (vi[0] - vj[0]) + e1 * (vi[1] - vj[1]) + e2 * (vi[2] - vj[2])) / rij;
            const double t = rij + rsdot * dtr;
            b1 = b1 < t ? b1 : t;
        }
        const double g = R4(1.1) * rs;
        rs = b1 > g ? b1 : g;
    }
    return rs;
}

// Radius of a row that overflowed (util_gpu.F:69-100, fpoly0.F:134-160);
// nb_neg = -NNB.
inline double ac_shrink(int nb_flag, int nnbopt, int nnbmax, int nb_neg, double rs) {
    if (!nb_flag) return R4(0.9) * rs;
    if (-nb_neg > nnbopt) return (double)powf(-(float)nnbopt / (float)nb_neg, 0.333f) * rs;
    return (double)powf((float)nnbopt / (float)nnbmax, 0.4f) * rs;
}

// Density centre, core radius and core rms velocity of a cluster (core.f),
// from the bodies' positions and velocities x, v at TIME, masses m and radii
// rs.  rows_of(jl, rp) gives the neighbour row of each selected central body
// jl[l] (cluster-local index) in rp[l]: [nnb, 1-based addresses], address
// a0 + 1 being body 0 of the cluster.  In: a.rdens and rc_prev from the last
// call (zero and unused at TIME = 0), a.rscale.  Out: a.rdens, a.rc2, the
// returned VC, and rc_prev.
template <class RowsOf>
inline double ac_core(int nc, const double *m, const double *x, const double *v, const double *rs,
                      RowsOf rows_of, int a0, double time, ACPar &a, double &rc_prev) {
    double rcore2 = a.rscale * a.rscale;
    if (time > 0.0) rcore2 = std::max(9.0 * (rc_prev * rc_prev), rcore2);
    std::vector<int> jl;
    for (;;) {
        jl.clear();
        for (int i = 0; i < nc; ++i) {
            const double *p = x + 3 * (size_t)i;
            const double e0 = p[0] - a.rdens[0], e1 = p[1] - a.rdens[1], e2 = p[2] - a.rdens[2];
            if (e0 * e0 + e1 * e1 + e2 * e2 < rcore2) jl.push_back(i);
        }
        if ((int)jl.size() >= nc / 5) break;
        rcore2 = R4(1.5) * rcore2;
    }
    std::vector<const int *> rp(jl.size());
    rows_of(jl, rp);
    std::vector<double> rho(jl.size(), 0.0);
    // each central body's density is its own: blocks of bodies on a few
    // host threads (joined before the sums below)
    auto density = [&](size_t l0, size_t l1) {
      std::vector<double> rl;
      std::vector<int> il;
      for (size_t l = l0; l < l1; ++l) {
        const int i = jl[l];
        const int *row = rp[l];
        const int nnb = row[0];
        if (nnb <= 0) continue;
        const double *xi = x + 3 * (size_t)i;
        double d6 = (double)(2.0f * powf(6.0f / (float)nnb, 0.66f)) * (rs[i] * rs[i]);
        int n6;
        for (;;) {
            il.clear();
            rl.clear();
            for (int lj = 1; lj <= nnb; ++lj) {
                const int j = row[lj] - 1 - a0;
                const double *xj = x + 3 * (size_t)j;
                const double e0 = xi[0] - xj[0], e1 = xi[1] - xj[1], e2 = xi[2] - xj[2];
                const double rij2 = e0 * e0 + e1 * e1 + e2 * e2;
                if (rij2 < d6) {
                    il.push_back(j);
                    rl.push_back(rij2);
                }
            }
            n6 = (int)il.size();
            if (n6 >= 6) break;
            d6 = R4(1.5) * d6;
            if (n6 >= nnb) break;
        }
        for (int ii = 0; ii < n6; ++ii)                        // the exchange sort of :73-84
            for (int jj = ii + 1; jj < n6; ++jj)
                if (rl[jj] < rl[ii]) {
                    std::swap(rl[ii], rl[jj]);
                    std::swap(il[ii], il[jj]);
                }
        const int i6 = std::min(n6, 6);
        double xmass = 0.0;
        for (int lj = 0; lj < i6 - 1; ++lj) xmass += m[il[lj]];
        const double r6 = rl[i6 - 1];
        const double rinv32 = r6 > 0.0 ? 1.0 / (r6 * sqrt(r6)) : 0.0;
        rho[l] = n6 < 6 ? 0.0 : xmass * rinv32;
      }
    };
    const size_t nl = jl.size();
    const unsigned hw = std::thread::hardware_concurrency();
    const size_t nth = std::min<size_t>(std::max(1u, std::min(hw, 16u)), (nl + 4095) / 4096);
    if (nth <= 1) {
        density(0, nl);
    } else {
        std::vector<std::thread> th;
        for (size_t t = 0; t < nth; ++t) th.emplace_back(density, nl * t / nth, nl * (t + 1) / nth);
        for (auto &t : th) t.join();
    }
    double zmass = 0.0;
    for (int i = 0; i < nc; ++i) zmass += m[i];
    double rd[3] = {0.0, 0.0, 0.0}, rho1 = 0.0;
    for (size_t l = 0; l < jl.size(); ++l) {
        for (int k = 0; k < 3; ++k) rd[k] += rho[l] * x[3 * (size_t)jl[l] + k];
        rho1 += rho[l];
    }
    rho1 = std::max(rho1, zmass / (a.rscale * a.rscale * a.rscale));
    for (int k = 0; k < 3; ++k) a.rdens[k] = rd[k] / rho1;
    double rc = 0.0, rho2 = 0.0;
    for (size_t l = 0; l < jl.size(); ++l) {
        const double *p = x + 3 * (size_t)jl[l];
        const double e0 = p[0] - a.rdens[0], e1 = p[1] - a.rdens[1], e2 = p[2] - a.rdens[2];
        rc += rho[l] * rho[l] * (e0 * e0 + e1 * e1 + e2 * e2);
        rho2 += rho[l] * rho[l];
    }
    if (rho2 > 0.0) rc = sqrt(rc / rho2);
    if (rc == 0.0) rc = a.rscale;
    a.rc2 = rc * rc;
    rc_prev = rc;
    int nc1 = 0;
    double vc = 0.0;
    for (size_t l = 0; l < jl.size(); ++l) {
        const double *p = x + 3 * (size_t)jl[l];
        const double e0 = p[0] - a.rdens[0], e1 = p[1] - a.rdens[1], e2 = p[2] - a.rdens[2];
        if (e0 * e0 + e1 * e1 + e2 * e2 < a.rc2) {
            const double *u = v + 3 * (size_t)jl[l];
            nc1++;
            vc += u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
        }
    }
    return sqrt(vc / (double)(float)std::max(nc1, 2));
}

// STEP = sqrt(ETA (|F||F2| + |F1|^2) / (|F1||F3| + |F2|^2))   (tstep.f)
inline double tstep(const double *f, const double *f1, const double *f2, const double *f3, double eta) {
    double F2 = 0, F12 = 0, F22 = 0, F32 = 0;
    for (int k = 0; k < 3; ++k) {
        F2 += f[k] * f[k];
        F12 += f1[k] * f1[k];
        F22 += f2[k] * f2[k];
        F32 += f3[k] * f3[k];
    }
    const double num = sqrt(F2 * F22) + F12;
    const double den = sqrt(F12 * F32) + F22;
    if (!(den > 0)) return 1e30;
    return sqrt(eta * num / den);
}

// Largest power of two <= x, clamped to [lo, hi].
inline double pow2_floor(double x, double lo, double hi) {
    if (!(x > lo)) return lo;
    double p = hi;
    while (p > x && p > lo) p *= 0.5;
    return std::max(p, lo);
}

// State of n bodies (one cluster or several back to back).
struct Bodies {
    int n = 0;
    nb6drive_params P;
    std::vector<double> m, x0, v0, t0, step, t0r, stepr, fi, fidot, d2, d3, fr, frdot, d2r, d3r, f,
        fdot, rs;
    std::vector<int> list;  // n x LS: [nnb, 1-based addresses ascending] (self excluded)
    int LS = 0;             // row stride (lmax + 8 so the AVX library can over-read)
    double tcr = 2.0 * sqrt(2.0);  // crossing time in Henon units
    // initial evaluation (fpoly0.F:100-206): a row holding only the body
    // itself is evaluated again with a larger radius
    bool fpoly0 = false;
    // radius-rule quantities per cluster (one cluster unless set by the
    // ensemble driver): acl[i] = cluster of body i; RSMIN since the last
    // adjust (intgrt.F:927, reset at output, output.F:271); core radius of
    // the last core() call
    std::vector<ACPar> acp{ACPar()};
    std::vector<int> acl;
    std::vector<double> rsmin{0.0}, rc_last{0.0};
    const ACPar &acpar(int i) const { return acp[acl.empty() ? 0 : acl[i]]; }
    void rsmin_seen(int i) {
        double &r = rsmin[acl.empty() ? 0 : acl[i]];
        r = std::min(r, rs[i]);
    }
    // adjust times: TIME = 0, then the first output at or after each
    // multiple of DTADJ (dt_adj <= 0: every output)
    double tnext_adj = 0.0;
    bool adjust_due(double time) {
        if (time < tnext_adj - 1e-15) return false;
        const double d = P.dt_adj > 0.0 ? P.dt_adj : 0.0;
        tnext_adj = d > 0.0 ? (floor(time / d + 1e-12) + 1.0) * d : time;
        return true;
    }
    void adjust_init(int ncl) {
        acp.assign(ncl, ACPar());
        rsmin.assign(ncl, P.rs0);   // RSMIN = RS0 from the input (input.F:137)
        rc_last.assign(ncl, 0.0);
    }

    // Adjust-time quantities of cluster c, whose nc bodies start at body b:
    // what ADJUST computes for the radius rule (adjust.F:104 TCR, :136
    // RSCALE, :150 RSMIN, :154 CORE, :199 RSFAC) followed by OUTPUT's own
    // CORE call and RSMIN reset (output.F:61,271).  x, v: the bodies at
    // `time`; ekin, pot (> 0): the cluster's kinetic and potential energy;
    // rows_of(jl, rp): the neighbour rows of the cluster's bodies jl (see
    // ac_core).
    template <class RowsOf>
    void adjust(int c, int b, int nc, const double *x, const double *v, double ekin, double pot,
                RowsOf rows_of, double time) {
        ACPar &a = acp[c];
        double zmass = 0.0;
        for (int k = 0; k < nc; ++k) zmass += m[b + k];
        const double tcr_c = pow(zmass, 2.5) / pow(2.0 * fabs(ekin - pot), 1.5);
        a.rscale = 0.5 * (zmass * zmass) / pot;
        a.bodym = zmass / (double)(float)nc;
        if (rsmin[c] == 0.0) {  // adjust.F:139-150 (over every body, not only those with neighbours)
            double r0 = a.rscale;
            for (int k = 0; k < nc; ++k) r0 = std::min(r0, rs[b + k]);
            rsmin[c] = r0;
        }
        const double vc = ac_core(nc, &m[b], x, v, &rs[b], rows_of, b, time, a, rc_last[c]);
        a.rsfac = std::max(R4(25.0) / tcr_c, 3.0 * vc / (2.0 * rsmin[c]));
        ac_core(nc, &m[b], x, v, &rs[b], rows_of, b, time, a, rc_last[c]);
        rsmin[c] = R4(100.0);
    }
    nb6drive_stats st{};

    // State at the block time of the bodies being regular-corrected, taken
    // before any of them is corrected: the neighbour gain/loss force moves of
    // one body must see the others as predicted, not as corrected.
    std::vector<unsigned char> snapped;
    std::vector<double> xs, vs;

    int *row(int i) { return &list[(size_t)i * LS]; }

    void alloc() {
        snapped.assign(n, 0);
        xs.assign(3 * (size_t)n, 0.0);
        vs.assign(3 * (size_t)n, 0.0);
        LS = P.lmax + 8;
        list.assign((size_t)n * LS, 0);
        auto z3 = [&](std::vector<double> &v) { v.assign(3 * (size_t)n, 0.0); };
        z3(fi), z3(fidot), z3(d2), z3(d3), z3(fr), z3(frdot), z3(d2r), z3(d3r), z3(f), z3(fdot);
        t0.assign(n, 0.0);
        t0r.assign(n, 0.0);
        step.assign(n, P.smax);
        stepr.assign(n, P.smax);
        rs.assign(n, 0.0);
    }

    // Initial radius and regular step from the distance to the cluster
    // centre (fpoly0.F:55-59); xc is the body's position relative to it.
    void init_radius(int i, const double *xc) {
        const double ri2 = xc[0] * xc[0] + xc[1] * xc[1] + xc[2] * xc[2];
        rs[i] = P.rs_init ? P.rs_init[i] : P.rs0 * sqrt(1.0 + ri2);
        stepr[i] = std::min(P.smax * sqrt(1.0 + ri2), P.smax);
    }

    // Hermite predictor of body j to time t (xbpredall.F:50-59).
    void pred(int j, double t, double *x, double *v) const {
        const double s = t - t0[j], s1 = 1.5 * s, s2 = 2.0 * s;
        for (int k = 0; k < 3; ++k) {
            const size_t q = 3 * (size_t)j + k;
            x[k] = ((fdot[q] * s + f[q]) * s + v0[q]) * s + x0[q];
            v[k] = (fdot[q] * s1 + f[q]) * s2 + v0[q];
        }
    }

    void snapshot(const std::vector<int> &ids, double t) {
        for (int i : ids) {
            pred(i, t, &xs[3 * (size_t)i], &vs[3 * (size_t)i]);
            snapped[i] = 1;
        }
    }
    void release_snapshot(const std::vector<int> &ids) {
        for (int i : ids) snapped[i] = 0;
    }
    // Body j at t: the snapshot if it holds one, else the predictor.
    void pred_at(int j, double t, double *x, double *v) const {
        if (snapped[j]) {
            for (int k = 0; k < 3; ++k) {
                x[k] = xs[3 * (size_t)j + k];
                v[k] = vs[3 * (size_t)j + k];
            }
        } else {
            pred(j, t, x, v);
        }
    }

    // FP64 pair force and jerk of body j (at t) on (xi, vi).
    void pair_force(const double *xi, const double *vi, int j, double t, double *a, double *jd) const {
        double xj[3], vj[3];
        pred_at(j, t, xj, vj);
        const double dx = xj[0] - xi[0], dy = xj[1] - xi[1], dz = xj[2] - xi[2];
        const double dvx = vj[0] - vi[0], dvy = vj[1] - vi[1], dvz = vj[2] - vi[2];
        const double r2 = dx * dx + dy * dy + dz * dz;
        const double dr2i = 1.0 / r2, dr3i = m[j] * dr2i * sqrt(dr2i);
        const double drdp = 3.0 * (dx * dvx + dy * dvy + dz * dvz) * dr2i;
        a[0] = dx * dr3i;
        a[1] = dy * dr3i;
        a[2] = dz * dr3i;
        jd[0] = (dvx - dx * drdp) * dr3i;
        jd[1] = (dvy - dy * drdp) * dr3i;
        jd[2] = (dvz - dz * drdp) * dr3i;
    }

    // Split forces at t = 0 from the first regular and irregular evaluation,
    // and the initial steps from |F|/|FDOT| (two-term form of the criterion).
    void init_forces(int i, const double *freg, const double *fdr, const double *a, const double *jd) {
        double ft[3], fdt[3];
        for (int k = 0; k < 3; ++k) {
            fr[3 * i + k] = freg[k];
            frdot[3 * i + k] = fdr[k];
            fi[3 * i + k] = a[k];
            fidot[3 * i + k] = jd[k];
            f[3 * i + k] = 0.5 * (fi[3 * i + k] + fr[3 * i + k]);
            fdot[3 * i + k] = ONE6 * (fidot[3 * i + k] + frdot[3 * i + k]);
            ft[k] = fi[3 * i + k] + fr[3 * i + k];
            fdt[k] = fidot[3 * i + k] + frdot[3 * i + k];
        }
        double F = 0, FD = 0, FR = 0, FRD = 0;
        for (int k = 0; k < 3; ++k) {
            F += ft[k] * ft[k];
            FD += fdt[k] * fdt[k];
            FR += fr[3 * i + k] * fr[3 * i + k];
            FRD += frdot[3 * i + k] * frdot[3 * i + k];
        }
        const double dti = FD > 0 ? 0.5 * P.eta_i * sqrt(F / FD) : P.smax;
        const double dtr = FRD > 0 ? 0.5 * P.eta_r * sqrt(FR / FRD) : P.smax;
        stepr[i] = pow2_floor(dtr, P.dtmin, P.smax);
        step[i] = std::min(pow2_floor(dti, P.dtmin, P.smax), stepr[i]);
    }

    // Irregular corrector and new irregular step of body i at `time` from its
    // new neighbour force a and jerk jd; returns true when its regular step
    // is due too (otherwise F, FDOT are extrapolated, intgrt.F:570-578).
    bool irr_correct(int i, double time, const double *a, const double *jd) {
        const double s = time - t0[i], s1 = 1.5 * s, s2 = 2.0 * s;
        double xi[3], vi[3];
        for (int k = 0; k < 3; ++k) {
            const size_t c = 3 * (size_t)i + k;
            xi[k] = ((fdot[c] * s + f[c]) * s + v0[c]) * s + x0[c];
            vi[k] = (fdot[c] * s1 + f[c]) * s2 + v0[c];
        }
        const double dt = s, dtsq = dt * dt, dt6 = 6.0 / (dt * dtsq), dt2 = 2.0 / dtsq;
        const double dtsq12 = ONE12 * dtsq, dt13 = ONE3 * dt;
        double ftot[3];
        for (int k = 0; k < 3; ++k) {  // nbint_cor.f:130-150
            const size_t c = 3 * (size_t)i + k;
            const double df = fi[c] - a[k];
            const double fid = fidot[c];
            const double sum = fid + jd[k];
            const double at3 = 2.0 * df + dt * sum;
            const double bt2 = -3.0 * df - dt * (sum + fid);
            x0[c] = xi[k] + (R4(0.6) * at3 + bt2) * dtsq12;
            v0[c] = vi[k] + (0.75 * at3 + bt2) * dt13;
            fi[c] = a[k];
            fidot[c] = jd[k];
            ftot[k] = fi[c] + fr[c];
            d2[c] = (3.0 * at3 + bt2) * dt2;
            d3[c] = at3 * dt6;
        }
        // irregular step (nbint_cor.f:146,215-236)
        double ttmp = tstep(ftot, &fidot[3 * i], &d2[3 * i], &d3[3 * i], P.eta_i);
        const double dt0 = ttmp;
        if (ttmp > 2.0 * step[i]) {
            ttmp = (fmod(time, 2.0 * step[i]) == 0.0) ? std::min(2.0 * step[i], P.smax) : step[i];
        } else if (ttmp < step[i]) {
            ttmp = 0.5 * step[i];
            if (ttmp > dt0) ttmp *= 0.5;
        } else {
            ttmp = step[i];
        }
        step[i] = std::max(ttmp, P.dtmin);
        t0[i] = time;
        st.irr_steps++;
        if (t0r[i] + stepr[i] <= time) return true;
        const double dtr = time - t0r[i];
        for (int k = 0; k < 3; ++k) {
            const size_t c = 3 * (size_t)i + k;
            f[c] = 0.5 * (frdot[c] * dtr + fr[c] + fi[c]);
            fdot[c] = ONE6 * (frdot[c] + fidot[c]);
        }
        // keep the irregular step inside the regular interval
        while (t0[i] + step[i] > t0r[i] + stepr[i] && step[i] > P.dtmin) step[i] *= 0.5;
        return false;
    }

    // Overflow handling of one regular-force row (util_gpu.F:69-100, NB_FLAG
    // branch): shrink RS; the caller re-runs the force.
    void shrink_radius(int i, int nb_neg) { rs[i] = ac_shrink(P.nb_flag, P.nnbopt, P.nnbmax, nb_neg, rs[i]); }

    // Regular corrector of body i at `time`: Ahmad-Cohen radius update, force
    // moves for neighbours gained and lost, Hermite corrector on the regular
    // force, new regular step.  nlist is the new row (1-based, self removed),
    // freg/fdr the new regular force and jerk.  (xi, vi) is i at `time`.
    void reg_correct(int i, double time, const int *nlist, const double *freg, const double *fdr) {
        const int nnb = nlist[0];
        const int nnb0 = row(i)[0];
        const double dtr = time - t0r[i];
        double xi[3], vi[3];
        pred_at(i, time, xi, vi);
        // Ahmad-Cohen radius update (regcor_gpu.F:19-238) from the first
        // min(nnb, 3) new neighbours at `time`; for nnb = 0 it also gives
        // the irregular force change the neighbour moves start from
        double xnb[9] = {0}, vnb[9] = {0};
        for (int l = 0; l < std::min(nnb, 3); ++l) pred_at(nlist[1 + l] - 1, time, &xnb[3 * l], &vnb[3 * l]);
        double dfirr[3], dfd[3];
        rs[i] = ac_radius(P.nb_flag, P.m_flag, P.nnbopt, P.nnbmax, acpar(i), nnb, nnb0, dtr, xi, vi, xnb, vnb,
                          rs[i], dfirr, dfd);
        if (nnb > 0) rsmin_seen(i);
        // neighbour gains and losses: move their force between the parts
        // (regcor_gpu.F:284-444)
        const int *old = row(i);
        int a = 1, b = 1;
        while (a <= nnb0 || b <= nnb) {
            const int jo = a <= nnb0 ? old[a] : 0x7fffffff;
            const int jn = b <= nnb ? nlist[b] : 0x7fffffff;
            double fa[3], fj[3];
            if (jo == jn) {
                ++a;
                ++b;
            } else if (jo < jn) {  // lost
                pair_force(xi, vi, jo - 1, time, fa, fj);
                for (int k = 0; k < 3; ++k) {
                    dfirr[k] -= fa[k];
                    dfd[k] -= fj[k];
                }
                ++a;
            } else {  // gained
                pair_force(xi, vi, jn - 1, time, fa, fj);
                for (int k = 0; k < 3; ++k) {
                    dfirr[k] += fa[k];
                    dfd[k] += fj[k];
                }
                ++b;
            }
        }
        // regular corrector (regcor_gpu.F:442-537)
        const double dtsq = dtr * dtr, dt6 = 6.0 / (dtr * dtsq), dt2 = 2.0 / dtsq;
        const double dtsq12 = ONE12 * dtsq, dtr13 = ONE3 * dtr;
        for (int k = 0; k < 3; ++k) {
            const size_t c = 3 * (size_t)i + k;
            const double dfr = fr[c] - freg[k] - dfirr[k];
            const double fdr0 = fdr[k] + dfd[k];
            const double frd = frdot[c];
            const double sum = frd + fdr0;
            const double at3 = 2.0 * dfr + dtr * sum;
            const double bt2 = -3.0 * dfr - dtr * (sum + frd);
            x0[c] += (R4(0.6) * at3 + bt2) * dtsq12;
            v0[c] += (0.75 * at3 + bt2) * dtr13;
            fi[c] += dfirr[k];
            fr[c] = freg[k];
            fidot[c] += dfd[k];
            frdot[c] = fdr[k];
            d3r[c] = at3 * dt6;
            d2r[c] = (3.0 * at3 + bt2) * dt2;
        }
        // the ids, plus zeros over the 8-id window a SIMD list reader may
        // touch past nnb (irr.avx.cpp:468-489)
        const int keep = std::min(LS, nnb + 1);
        memcpy(row(i), nlist, sizeof(int) * keep);
        for (int k = keep; k < std::min(LS, keep + 8); ++k) row(i)[k] = 0;
        st.nb_sum += nnb;
        st.nb_absdev += fabs((double)(nnb - P.nnbopt));
        // new regular step (regcor_gpu.F:593-737)
        double ttmp = tstep(&fr[3 * i], &frdot[3 * i], &d2r[3 * i], &d3r[3 * i], P.eta_r);
        const double dt0 = ttmp;
        if (ttmp > 2.0 * stepr[i]) {
            ttmp = (fmod(time, 2.0 * dtr) == 0.0) ? std::min(2.0 * dtr, P.smax) : stepr[i];
        } else if (ttmp < dtr) {
            ttmp = 0.5 * dtr;
            if (ttmp > dt0) ttmp *= 0.5;
        } else {
            ttmp = stepr[i];
        }
        ttmp = std::max(std::min(ttmp, P.smax), P.dtmin);
        stepr[i] = ttmp;
        t0r[i] = time;
        for (int k = 0; k < 3; ++k) {
            const size_t c = 3 * (size_t)i + k;
            f[c] = 0.5 * (fi[c] + fr[c]);
            fdot[c] = ONE6 * (fidot[c] + frdot[c]);
        }
        if (step[i] > stepr[i]) step[i] = stepr[i];
        st.reg_steps++;
    }

    // ---- learned neighbour radius ----------------------------------------
    // Features of body i at a regular step, the same formula as the library's
    // epilogue (mlp.cuh): log(1+nnb) with self counted, log RS,
    // log(1+nnb) - 1.5 log h2, log|a_reg|, -log2 dtr.
    static void features(double nnb_self, double h2, double a2, double dtr, float *f) {
        const double ln = log(1.0 + fabs(nnb_self));
        const double lh = log(h2 > 1e-300 ? h2 : 1e-300);
        f[0] = (float)ln;
        f[1] = (float)(0.5 * lh);
        f[2] = (float)(ln - 1.5 * lh);
        f[3] = (float)(0.5 * log(a2 > 1e-300 ? a2 : 1e-300));
        f[4] = (float)(-log2(dtr > 1e-300 ? dtr : 1e-300));
    }
    std::vector<float> feat;            // [n][5] at the body's last regular step
    std::vector<double> rs_feat;        // RS used at that step
    std::vector<unsigned char> have_feat;

    // Mode 1, before the corrector of body i: the sample of its previous
    // regular step is completed with this step's outcome -- target
    // log(RS* / RS_prev), RS* = RS_used (NNBOPT / nnb)^(1/3) -- and this
    // step's features are kept for the next one.
    void learn_log(int i, int nnb_noself, double rs_used, double h2_used, const double *freg,
                   double dtr_used) {
        if (feat.empty()) {
            feat.assign(5 * (size_t)n, 0.f);
            rs_feat.assign(n, 0.0);
            have_feat.assign(n, 0);
        }
        if (have_feat[i] && nnb_noself > 0 && st.nsamples < P.sample_cap && P.samples) {
            float *o = P.samples + 6 * (size_t)st.nsamples;
            for (int k = 0; k < 5; ++k) o[k] = feat[5 * (size_t)i + k];
            o[5] = (float)(log(rs_used / rs_feat[i]) + log((double)P.nnbopt / nnb_noself) / 3.0);
            st.nsamples++;
        }
        const double a2 = freg[0] * freg[0] + freg[1] * freg[1] + freg[2] * freg[2];
        features(nnb_noself + 1, h2_used, a2, dtr_used, &feat[5 * (size_t)i]);
        rs_feat[i] = rs_used;
        have_feat[i] = 1;
    }

    // Mode 2, after the corrector: take RS_used exp(dlog) when the count it
    // implies (nnb ~ RS^3) stays inside [NNBOPT/2, NNBMAX]; otherwise keep the
    // Ahmad-Cohen radius the corrector just set.  The proposal is clamped to
    // a factor 2 change of RS per regular step (a guard against noisy count
    // estimates from few neighbours; the Ahmad-Cohen rule itself moves RS by
    // at most 25% per step).
    void learn_apply(int i, int nnb_noself, double rs_used, double dlog) {
        const double lim = 0.69314718055994531;  // log 2
        dlog = dlog > lim ? lim : (dlog < -lim ? -lim : dlog);
        const double r = rs_used * exp(dlog);
        const double expect = nnb_noself * exp(3.0 * dlog);
        if (nnb_noself > 0 && dlog == dlog && expect >= 0.5 * P.nnbopt && expect <= P.nnbmax) {
            rs[i] = r;
            st.mlp_used++;
        } else {
            st.mlp_fallback++;
        }
    }

    // ---- block clock ------------------------------------------------------
    // Next block: every body with the smallest t0 + step (next_tlist.f picks
    // the same set from its level lists).  A body's t0 + step only changes
    // when it is active.  Bodies wait in buckets keyed by their exact next
    // time: one bucket per step level (every body on a level shares its next
    // time, since t0 is a multiple of the step), with a general map for any
    // body whose time does not match its level's bucket.  A block costs O(k)
    // for its k bodies instead of a scan of all n.
    static constexpr int NLEV = 64;
    std::vector<int> lev_ids[NLEV];
    double lev_t[NLEV];
    std::map<double, std::vector<int>> clock_other;

    static int level_of(double step) {
        int e = 0;
        const double mant = frexp(step, &e);  // step = mant 2^e
        if (mant != 0.5) return -1;
        const int L = 1 - e;                  // step = 2^-L
        return (L >= 0 && L < NLEV) ? L : -1;
    }

    void clock_add(int i) {
        const double t = t0[i] + step[i];
        const int L = level_of(step[i]);
        if (L >= 0 && (lev_ids[L].empty() || lev_t[L] == t)) {
            lev_t[L] = t;
            lev_ids[L].push_back(i);
        } else {
            clock_other[t].push_back(i);
        }
    }

    void clock_reset() {
        for (auto &v : lev_ids) v.clear();
        clock_other.clear();
        for (int i = 0; i < n; ++i) clock_add(i);
    }

    // Pops the next block into `active` (ascending body order); returns its
    // time, or a value above tcrit when there is none left.
    double clock_next(std::vector<int> &active) {
        active.clear();
        double tmin = 1e300;
        for (int L = 0; L < NLEV; ++L)
            if (!lev_ids[L].empty()) tmin = std::min(tmin, lev_t[L]);
        if (!clock_other.empty()) tmin = std::min(tmin, clock_other.begin()->first);
        if (tmin == 1e300) return tmin;
        for (int L = 0; L < NLEV; ++L)
            if (!lev_ids[L].empty() && lev_t[L] == tmin) {
                active.insert(active.end(), lev_ids[L].begin(), lev_ids[L].end());
                lev_ids[L].clear();
            }
        if (!clock_other.empty() && clock_other.begin()->first == tmin) {
            auto it = clock_other.begin();
            active.insert(active.end(), it->second.begin(), it->second.end());
            clock_other.erase(it);
        }
        std::sort(active.begin(), active.end());
        return tmin;
    }

    void clock_push(const std::vector<int> &ids) {
        for (int i : ids) clock_add(i);
    }

    // Regular force of bodies idx[q0..q1) through gpunb_regf_ in calls of at
    // most P.chunk (util_gpu.F:33-60) against the nj bodies last sent.  A
    // row that overflows gets the radius shrink of util_gpu.F:69-100 and is
    // evaluated again; only those rows go into the next call (the others'
    // results do not depend on which rows share a call).  fill(i, xi, vi)
    // gives body i at the block time; take(q, i, row, acc, jrk) receives a
    // finished row (row = [nnb, ids]); prop[q] gets the learned proposal in
    // mlp_mode 2.
    template <class Fill, class Take>
    void regf_rows(const Backend &B, const std::vector<int> &idx, int q0, int q1, int nj, double bodym,
                   Fill fill, Take take, std::vector<double> &prop) {
        const int C = P.chunk;
        std::vector<double> h2(C + 4), dtr(C + 4), xi(3 * (C + 4)), vi(3 * (C + 4)), acc(3 * (C + 4)),
            jrk(3 * (C + 4)), pot(C + 4), pr(C + 4);
        std::vector<int> lst((size_t)(C + 4) * P.lmax), rows, again;
        for (int c0 = q0; c0 < q1; c0 += C) {
            rows.clear();
            for (int q = c0; q < std::min(q1, c0 + C); ++q) rows.push_back(q);
            while (!rows.empty()) {
                const int ni = (int)rows.size();
                for (int p = 0; p < ni; ++p) {
                    const int i = idx[rows[p]];
                    h2[p] = h2_of(i, bodym);
                    dtr[p] = stepr[i];
                    fill(i, &xi[3 * (size_t)p], &vi[3 * (size_t)p]);
                }
                for (int p = ni; p < ni + 4; ++p) {  // a SIMD library reads 4 i at a time
                    h2[p] = 0;
                    dtr[p] = 0;
                    for (int k = 0; k < 3; ++k) xi[3 * p + k] = vi[3 * p + k] = 0;
                }
                int nni = ni, lmax = P.lmax, nnbmax = P.nnbmax, mf = P.m_flag;
                B.gpunb_regf(&nni, h2.data(), dtr.data(), (double(*)[3])xi.data(), (double(*)[3])vi.data(),
                             (double(*)[3])acc.data(), (double(*)[3])jrk.data(), pot.data(), &lmax, &nnbmax,
                             lst.data(), &mf);
                st.reg_calls++;
                st.reg_pairs += (long long)ni * nj;
                if (P.mlp_mode == 2) B.proposals(&nni, pr.data());
                again.clear();
                for (int p = 0; p < ni; ++p) {
                    const int q = rows[p], i = idx[q];
                    const int *row = &lst[(size_t)p * P.lmax];
                    if (row[0] < 0) {
                        shrink_radius(i, row[0]);
                        again.push_back(q);
                        continue;
                    }
                    if (fpoly0 && row[0] < 2) {  // only itself: RS = 1.5 RS (fpoly0.F:157)
                        rs[i] = R4(1.5) * rs[i];
                        again.push_back(q);
                        continue;
                    }
                    if (P.mlp_mode == 2) prop[q] = pr[p];
                    take(q, i, row, &acc[3 * (size_t)p], &jrk[3 * (size_t)p]);
                }
                if (!again.empty()) st.overflow_retries++;
                rows.swap(again);
            }
        }
    }

    // neighbour-sphere criterion h2 of body i for gpunb_regf (m_flag: per
    // unit mass, util_gpu.F:45-52; bodym = mean mass of its cluster)
    double h2_of(int i, double bodym) const {
        return P.m_flag ? rs[i] * rs[i] / bodym : rs[i] * rs[i];
    }
};

}  // namespace nb6drv
