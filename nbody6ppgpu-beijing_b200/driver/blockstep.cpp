// blockstep.cpp -- Hermite 4th-order block-step integrator with the
// Ahmad-Cohen neighbour scheme, for single stars, driving the force path
// through the reference's own C ABI (gpunb_*, irr_simd_*, gpupot_).
//
// This is a restatement of the essentials of the reference's driver so the
// force libraries can be run to T = 1 / T = 10 without the Fortran program
// (no Fortran compiler is available):
//   block selection              intgrt.F:233-295 (next_tlist)
//   irregular force + corrector  intgrt.F:533-581, nbint_cor.f:17-160
//   irregular step               nbint_cor.f:146-236, tstep.f
//   regular force                util_gpu.F:33-111 (1024-i calls, overflow retry)
//   regular corrector            regcor_gpu.F:120-537 (radius update, list
//                                gain/loss force moves, Hermite corrector)
//   regular step                 regcor_gpu.F:593-737
//   F, FDOT bookkeeping          intgrt.F:558-581,911-935
//   energy                       energy.F:28-62 (GPUPOT), ZKIN
// Left out: KS/chain regularisation, stellar evolution, external fields,
// the checkl/fpcorr options (KZ(37), KZ(38)) and the SMIN neighbour retention.
//
// The same code runs on any backend that exports the ABI: libnb6b200.so or
// the reference's CPU libraries compiled from source.  Backends are loaded
// with dlopen(RTLD_LOCAL) from the paths the caller gives.
#include <dlfcn.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <algorithm>
#include <vector>

namespace {

typedef void (*fn_open)(int *, int *);
typedef void (*fn_close)();
typedef void (*fn_send)(int *, double *, double (*)[3], double (*)[3]);
typedef void (*fn_regf)(int *, double *, double *, double (*)[3], double (*)[3], double (*)[3],
                        double (*)[3], double *, int *, int *, int *, int *);
typedef void (*fn_pot)(int *, int *, int *, int *, double *, double (*)[3], double *);
typedef void (*fn_irr_open)(int *, int *, int *);
typedef void (*fn_irr_close)(int *);
typedef void (*fn_irr_set_jp)(int *, double *, double *, double *, double *, double *, double *);
typedef void (*fn_irr_set_list)(int *, int *);
typedef void (*fn_irr_firr)(double *, int *, int *, double (*)[3], double (*)[3], int *);

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
};

void *must_sym(void *h, const char *name) {
    void *p = dlsym(h, name);
    if (!p) fprintf(stderr, "nb6drive: missing symbol %s\n", name);
    return p;
}

bool load_backend(Backend &b, const char *reg, const char *irr, const char *pot) {
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
    return b.gpunb_open && b.gpunb_close && b.gpunb_send && b.gpunb_regf && b.gpupot &&
           b.irr_open && b.irr_close && b.irr_set_jp && b.irr_set_list && b.irr_firr_vec;
}

}  // namespace

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
};

// Counters returned by nb6drive_run.
struct nb6drive_stats {
    long long blocks, irr_steps, reg_steps, reg_calls, overflow_retries;
    long long nb_sum;       // sum of neighbour counts over regular steps
    long long reg_pairs;    // sum of ni * nj over gpunb_regf calls
    double wall_reg, wall_irr, wall_total;
    double t_end;
    int nout;
};

}  // extern "C"

namespace {

double wtime() {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

// STEP = sqrt(ETA (|F||F2| + |F1|^2) / (|F1||F3| + |F2|^2))   (tstep.f)
double tstep(const double *f, const double *f1, const double *f2, const double *f3, double eta) {
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
double pow2_floor(double x, double lo, double hi) {
    if (!(x > lo)) return lo;
    double p = hi;
    while (p > x && p > lo) p *= 0.5;
    return std::max(p, lo);
}

struct Sim {
    int n = 0;
    nb6drive_params P;
    Backend B;
    std::vector<double> m, x0, v0, t0, step, t0r, stepr, fi, fidot, d2, d3, fr, frdot, d2r, d3r, f,
        fdot, rs;
    std::vector<int> list;  // n x LS: [nnb, 1-based ids ascending] (self excluded)
    int LS = 0;             // row stride (lmax + 8 so the AVX library can over-read)
    double time = 0, tcr = 2.0 * sqrt(2.0), rscale = 1.0;
    nb6drive_stats st{};
    std::vector<double> xp, vp;  // predicted positions / velocities (all bodies)

    int *row(int i) { return &list[(size_t)i * LS]; }

    void predict_all(double t) {
        for (int j = 0; j < n; ++j) {
            const double s = t - t0[j], s1 = 1.5 * s, s2 = 2.0 * s;
            for (int k = 0; k < 3; ++k) {
                const size_t q = 3 * (size_t)j + k;
                xp[q] = ((fdot[q] * s + f[q]) * s + v0[q]) * s + x0[q];
                vp[q] = (fdot[q] * s1 + f[q]) * s2 + v0[q];
            }
        }
    }

    void set_jp(int i) {
        int a = i + 1;
        double mm = m[i], tt = t0[i];
        B.irr_set_jp(&a, &x0[3 * i], &v0[3 * i], &f[3 * i], &fdot[3 * i], &mm, &tt);
    }

    void set_list(int i) {
        int a = i + 1;
        B.irr_set_list(&a, row(i));
    }

    // Regular force for the bodies in idx (chunks of P.chunk) against all
    // bodies predicted to `time`; returns the new lists through nlist
    // (rows of LS, 1-based, self removed).  Overflow shrinks RS and re-runs the
    // chunk (util_gpu.F:69-100, NB_FLAG branch).
    void regular_forces(const std::vector<int> &idx, std::vector<double> &freg,
                        std::vector<double> &fdr, std::vector<int> &nlist) {
        const double t_0 = wtime();
        predict_all(time);
        int nn = n;
        B.gpunb_send(&nn, m.data(), (double(*)[3])xp.data(), (double(*)[3])vp.data());
        const int C = P.chunk;
        std::vector<double> h2(C + 4), dtr(C + 4), xi(3 * (C + 4)), vi(3 * (C + 4)), acc(3 * (C + 4)),
            jrk(3 * (C + 4)), pot(C + 4);
        std::vector<int> lst((size_t)(C + 4) * P.lmax);
        const double bodym = 1.0 / n;
        freg.assign(3 * idx.size(), 0.0);
        fdr.assign(3 * idx.size(), 0.0);
        nlist.assign(idx.size() * (size_t)LS, 0);
        for (size_t c0 = 0; c0 < idx.size(); c0 += C) {
            const int ni = (int)std::min<size_t>(C, idx.size() - c0);
            for (;;) {
                for (int q = 0; q < ni; ++q) {
                    const int i = idx[c0 + q];
                    h2[q] = P.m_flag ? rs[i] * rs[i] / bodym : rs[i] * rs[i];
                    dtr[q] = stepr[i];
                    for (int k = 0; k < 3; ++k) {
                        xi[3 * q + k] = xp[3 * (size_t)i + k];
                        vi[3 * q + k] = vp[3 * (size_t)i + k];
                    }
                }
                for (int q = ni; q < ni + 4 && q < C + 4; ++q) {  // AVX library reads 4 at a time
                    h2[q] = 0;
                    dtr[q] = 0;
                    for (int k = 0; k < 3; ++k) xi[3 * q + k] = vi[3 * q + k] = 0;
                }
                int nni = ni, lmax = P.lmax, nnbmax = P.nnbmax, mf = P.m_flag;
                B.gpunb_regf(&nni, h2.data(), dtr.data(), (double(*)[3])xi.data(), (double(*)[3])vi.data(),
                             (double(*)[3])acc.data(), (double(*)[3])jrk.data(), pot.data(), &lmax,
                             &nnbmax, lst.data(), &mf);
                st.reg_calls++;
                st.reg_pairs += (long long)ni * n;
                bool retry = false;
                for (int q = 0; q < ni; ++q) {
                    const int nb = lst[(size_t)q * P.lmax];
                    if (nb < 0) {
                        const int i = idx[c0 + q];
                        if (-nb > P.nnbopt) rs[i] *= pow((double)P.nnbopt / (double)(-nb), 0.333);
                        else rs[i] *= pow((double)P.nnbopt / (double)P.nnbmax, 0.4);
                        retry = true;
                    }
                }
                if (retry) {
                    st.overflow_retries++;
                    continue;
                }
                break;
            }
            for (int q = 0; q < ni; ++q) {
                const int i = idx[c0 + q];
                for (int k = 0; k < 3; ++k) {
                    freg[3 * (c0 + q) + k] = acc[3 * q + k];
                    fdr[3 * (c0 + q) + k] = jrk[3 * q + k];
                }
                const int nb = lst[(size_t)q * P.lmax];
                int *out = &nlist[(c0 + q) * (size_t)LS];
                int l1 = 0;
                for (int l = 1; l <= nb; ++l) {
                    const int j = lst[(size_t)q * P.lmax + l];
                    if (j != i) out[1 + l1++] = j + 1;
                }
                out[0] = l1;
            }
        }
        st.wall_reg += wtime() - t_0;
    }

    void pair_force(const double *xi, const double *vi, int j, double *a, double *jd) {
        const double dx = xp[3 * (size_t)j] - xi[0], dy = xp[3 * (size_t)j + 1] - xi[1],
                     dz = xp[3 * (size_t)j + 2] - xi[2];
        const double dvx = vp[3 * (size_t)j] - vi[0], dvy = vp[3 * (size_t)j + 1] - vi[1],
                     dvz = vp[3 * (size_t)j + 2] - vi[2];
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

    bool init();
    void regular_step(const std::vector<int> &reg);
    bool run(double *eout, int nout_max);
    void energy(double &ekin, double &epot);
};

bool Sim::init() {
    LS = P.lmax + 8;
    list.assign((size_t)n * LS, 0);
    auto z3 = [&](std::vector<double> &v) { v.assign(3 * (size_t)n, 0.0); };
    z3(fi), z3(fidot), z3(d2), z3(d3), z3(fr), z3(frdot), z3(d2r), z3(d3r), z3(f), z3(fdot);
    xp.assign(3 * (size_t)n, 0);
    vp.assign(3 * (size_t)n, 0);
    t0.assign(n, 0.0);
    t0r.assign(n, 0.0);
    step.assign(n, P.smax);
    stepr.assign(n, P.smax);
    rs.assign(n, 0.0);
    for (int i = 0; i < n; ++i) {
        const double ri2 = x0[3 * i] * x0[3 * i] + x0[3 * i + 1] * x0[3 * i + 1] + x0[3 * i + 2] * x0[3 * i + 2];
        rs[i] = P.rs0 * sqrt(1.0 + ri2);                         // fpoly0.F:55
        stepr[i] = std::min(P.smax * sqrt(1.0 + ri2), P.smax);    // fpoly0.F:57-59
    }
    int nb = n + 10, rank = 0;
    B.gpunb_open(&nb, &rank);
    int nmax = n, lmax = P.lmax;
    B.irr_open(&nmax, &lmax, &rank);
    time = 0.0;
    // regular force and lists at t = 0 (fpoly0.F:100-206)
    std::vector<int> all(n);
    for (int i = 0; i < n; ++i) all[i] = i;
    std::vector<double> freg, fdr;
    std::vector<int> nl;
    regular_forces(all, freg, fdr, nl);
    for (int i = 0; i < n; ++i) {
        memcpy(row(i), &nl[(size_t)i * LS], sizeof(int) * LS);
        for (int k = 0; k < 3; ++k) {
            fr[3 * i + k] = freg[3 * i + k];
            frdot[3 * i + k] = fdr[3 * i + k];
        }
    }
    // irregular force from the lists: state at t = 0 with F = FDOT = 0 so the
    // libraries' prediction is the identity
    for (int i = 0; i < n; ++i) {
        set_jp(i);
        set_list(i);
    }
    std::vector<int> addr(n);
    for (int i = 0; i < n; ++i) addr[i] = i + 1;
    std::vector<double> a(3 * (size_t)n), jd(3 * (size_t)n);
    std::vector<int> nnbid(n);
    double t = 0.0;
    int nn = n;
    B.irr_firr_vec(&t, &nn, addr.data(), (double(*)[3])a.data(), (double(*)[3])jd.data(), nnbid.data());
    for (int i = 0; i < n; ++i) {
        double ft[3], fdt[3];
        for (int k = 0; k < 3; ++k) {
            fi[3 * i + k] = a[3 * i + k];
            fidot[3 * i + k] = jd[3 * i + k];
            f[3 * i + k] = 0.5 * (fi[3 * i + k] + fr[3 * i + k]);
            fdot[3 * i + k] = (fidot[3 * i + k] + frdot[3 * i + k]) / 6.0;
            ft[k] = fi[3 * i + k] + fr[3 * i + k];
            fdt[k] = fidot[3 * i + k] + frdot[3 * i + k];
        }
        // initial steps from |F|/|FDOT| (two-term form of the step criterion)
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
        set_jp(i);
    }
    return true;
}

void Sim::regular_step(const std::vector<int> &reg) {
    std::vector<double> freg, fdr;
    std::vector<int> nl;
    regular_forces(reg, freg, fdr, nl);
    const double znbmin = 0.2 * P.nnbopt;
    const double rsfac = std::max(25.0 / tcr, 0.0);
    for (size_t q = 0; q < reg.size(); ++q) {
        const int i = reg[q];
        const int *nlist = &nl[q * (size_t)LS];
        const int nnb = nlist[0];
        const int nnb0 = row(i)[0];
        const double dtr = time - t0r[i];
        const double *xi = &xp[3 * (size_t)i];
        const double *vi = &vp[3 * (size_t)i];
        const double ri2 = xi[0] * xi[0] + xi[1] * xi[1] + xi[2] * xi[2];
        const double rh2 = 9.0 * rscale * rscale;
        // Ahmad-Cohen radius update (regcor_gpu.F:131-196, NB_FLAG = 0 form)
        if (nnb > 0) {
            const double fac = 1.0 + 0.1 * (double)(P.nnbopt - nnb) / (double)nnb;
            double a3 = nnb * fac;
            const double nbave = std::min(P.nnbopt + 150, std::max(P.nnbmax - 50, (int)znbmin));
            a3 = std::min(a3, 0.9 * nbave);
            const int nbp = (int)a3;
            a3 = std::max(a3, znbmin);
            double a4 = a3 / nnb;
            if ((a3 - nnb0) * (a3 - nnb) < 0.0) a4 = sqrt(a4);
            const double a5 = std::min(rsfac * dtr, 0.25);
            a4 -= 1.0;
            a4 = a4 > a5 ? a5 : std::max(a4, -a5);
            const double a3b = a4 / 3.0;
            double a1 = 1.0 + a3b - a3b * a3b;
            if (nnb < znbmin && nbp > znbmin && a1 < 1.0) a1 = 1.05;
            if (fabs(a1 - 1.0) > 0.003) {
                if (rs[i] * rs[i] > ri2 && rs[i] * rs[i] < 2.0 * ri2 && nnb > 5) a1 = sqrt(a1);
                rs[i] *= a1;
            }
            const double ridot = xi[0] * vi[0] + xi[1] * vi[1] + xi[2] * vi[2];
            if (nnb > nbave && ridot < 0.0) rs[i] *= 1.0 - (nnb - nbave) / (3.0 * nnb);
        } else {
            rs[i] *= 1.5;  // zero membership (fpoly0.F:140-160)
        }
        (void)rh2;
        // neighbour gains and losses: move their force between the parts
        // (regcor_gpu.F:284-444)
        double dfirr[3] = {0, 0, 0}, dfd[3] = {0, 0, 0};
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
                pair_force(xi, vi, jo - 1, fa, fj);
                for (int k = 0; k < 3; ++k) {
                    dfirr[k] -= fa[k];
                    dfd[k] -= fj[k];
                }
                ++a;
            } else {  // gained
                pair_force(xi, vi, jn - 1, fa, fj);
                for (int k = 0; k < 3; ++k) {
                    dfirr[k] += fa[k];
                    dfd[k] += fj[k];
                }
                ++b;
            }
        }
        // regular corrector (regcor_gpu.F:442-537)
        const double dtsq = dtr * dtr, dt6 = 6.0 / (dtr * dtsq), dt2 = 2.0 / dtsq;
        const double dtsq12 = dtsq / 12.0, dtr13 = dtr / 3.0;
        for (int k = 0; k < 3; ++k) {
            const size_t c = 3 * (size_t)i + k;
            const double dfr = fr[c] - freg[3 * q + k] - dfirr[k];
            const double fdr0 = fdr[3 * q + k] + dfd[k];
            const double frd = frdot[c];
            const double sum = frd + fdr0;
            const double at3 = 2.0 * dfr + dtr * sum;
            const double bt2 = -3.0 * dfr - dtr * (sum + frd);
            x0[c] += (0.6 * at3 + bt2) * dtsq12;
            v0[c] += (0.75 * at3 + bt2) * dtr13;
            fi[c] += dfirr[k];
            fr[c] = freg[3 * q + k];
            fidot[c] += dfd[k];
            frdot[c] = fdr[3 * q + k];
            d3r[c] = at3 * dt6;
            d2r[c] = (3.0 * at3 + bt2) * dt2;
        }
        memcpy(row(i), nlist, sizeof(int) * LS);
        st.nb_sum += nnb;
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
            fdot[c] = (fidot[c] + frdot[c]) / 6.0;
        }
        if (step[i] > stepr[i]) step[i] = stepr[i];
        st.reg_steps++;
        set_list(i);
    }
}

void Sim::energy(double &ekin, double &epot) {
    predict_all(time);
    std::vector<double> phi(n + 8);
    int rank = 0, istart = 1, ni = n, nn = n;
    B.gpupot(&rank, &istart, &ni, &nn, m.data(), (double(*)[3])xp.data(), phi.data());
    ekin = 0;
    epot = 0;
    for (int i = 0; i < n; ++i) {
        const double v2 = vp[3 * i] * vp[3 * i] + vp[3 * i + 1] * vp[3 * i + 1] + vp[3 * i + 2] * vp[3 * i + 2];
        ekin += 0.5 * m[i] * v2;
        epot -= 0.5 * m[i] * phi[i];
    }
}

bool Sim::run(double *eout, int nout_max) {
    const double tw = wtime();
    int nout = 0;
    double ek, ep;
    energy(ek, ep);
    if (nout < nout_max) {
        eout[4 * nout] = 0.0;
        eout[4 * nout + 1] = ek;
        eout[4 * nout + 2] = ep;
        eout[4 * nout + 3] = ek + ep;
        nout++;
    }
    double tnext_out = P.dt_out;
    std::vector<int> active, reg, addr;
    std::vector<double> a, jd;
    std::vector<int> nnbid;
    while (st.blocks < P.max_blocks) {
        double tmin = 1e300;
        for (int i = 0; i < n; ++i) tmin = std::min(tmin, t0[i] + step[i]);
        if (tmin > P.tcrit + 1e-12) break;
        time = tmin;
        active.clear();
        for (int i = 0; i < n; ++i)
            if (t0[i] + step[i] == tmin) active.push_back(i);
        st.blocks++;
        // irregular force at the block time (intgrt.F:533) and corrector
        const int na = (int)active.size();
        addr.resize(na);
        for (int q = 0; q < na; ++q) addr[q] = active[q] + 1;
        a.assign(3 * (size_t)na, 0.0);
        jd.assign(3 * (size_t)na, 0.0);
        nnbid.assign(na, 0);
        const double ti0 = wtime();
        double t = time;
        int nna = na;
        B.irr_firr_vec(&t, &nna, addr.data(), (double(*)[3])a.data(), (double(*)[3])jd.data(), nnbid.data());
        st.wall_irr += wtime() - ti0;
        reg.clear();
        for (int q = 0; q < na; ++q) {
            const int i = active[q];
            const double s = time - t0[i], s1 = 1.5 * s, s2 = 2.0 * s;
            double xi[3], vi[3];
            for (int k = 0; k < 3; ++k) {
                const size_t c = 3 * (size_t)i + k;
                xi[k] = ((fdot[c] * s + f[c]) * s + v0[c]) * s + x0[c];
                vi[k] = (fdot[c] * s1 + f[c]) * s2 + v0[c];
            }
            const double dt = s, dtsq = dt * dt, dt6 = 6.0 / (dt * dtsq), dt2 = 2.0 / dtsq;
            const double dtsq12 = dtsq / 12.0, dt13 = dt / 3.0;
            double ftot[3];
            for (int k = 0; k < 3; ++k) {  // nbint_cor.f:130-150
                const size_t c = 3 * (size_t)i + k;
                const double df = fi[c] - a[3 * q + k];
                const double fid = fidot[c];
                const double sum = fid + jd[3 * q + k];
                const double at3 = 2.0 * df + dt * sum;
                const double bt2 = -3.0 * df - dt * (sum + fid);
                x0[c] = xi[k] + (0.6 * at3 + bt2) * dtsq12;
                v0[c] = vi[k] + (0.75 * at3 + bt2) * dt13;
                fi[c] = a[3 * q + k];
                fidot[c] = jd[3 * q + k];
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
            if (t0r[i] + stepr[i] <= time) {
                reg.push_back(i);
            } else {  // intgrt.F:570-578
                const double dtr = time - t0r[i];
                for (int k = 0; k < 3; ++k) {
                    const size_t c = 3 * (size_t)i + k;
                    f[c] = 0.5 * (frdot[c] * dtr + fr[c] + fi[c]);
                    fdot[c] = (frdot[c] + fidot[c]) / 6.0;
                }
                // keep the irregular step inside the regular interval
                while (t0[i] + step[i] > t0r[i] + stepr[i] && step[i] > P.dtmin) step[i] *= 0.5;
            }
        }
        if (!reg.empty()) regular_step(reg);
        for (int q = 0; q < na; ++q) set_jp(active[q]);
        if (time >= tnext_out - 1e-15) {
            energy(ek, ep);
            if (nout < nout_max) {
                eout[4 * nout] = time;
                eout[4 * nout + 1] = ek;
                eout[4 * nout + 2] = ep;
                eout[4 * nout + 3] = ek + ep;
                nout++;
            }
            tnext_out += P.dt_out;
        }
    }
    st.t_end = time;
    st.nout = nout;
    st.wall_total = wtime() - tw;
    return true;
}

}  // namespace

extern "C" {

// Integrate n single stars from (x, v) to p->tcrit on the given backend
// libraries (paths to shared objects exporting gpunb_*, irr_simd_* and
// gpupot_).  x and v (double[n][3]) are overwritten with the final state
// predicted to the end time.  Energies (t, kinetic, potential, total) are
// written every p->dt_out into eout[nout_max][4].  Returns 0 on success.
int nb6drive_run(const char *reg_lib, const char *irr_lib, const char *pot_lib, int n,
                 const double *mass, double *x, double *v, const nb6drive_params *p, double *eout,
                 int nout_max, nb6drive_stats *stats) {
    Sim s;
    s.n = n;
    s.P = *p;
    if (!load_backend(s.B, reg_lib, irr_lib, pot_lib)) return 1;
    s.m.assign(mass, mass + n);
    s.x0.assign(x, x + 3 * (size_t)n);
    s.v0.assign(v, v + 3 * (size_t)n);
    if (!s.init()) return 2;
    s.run(eout, nout_max);
    s.predict_all(s.time);
    memcpy(x, s.xp.data(), sizeof(double) * 3 * n);
    memcpy(v, s.vp.data(), sizeof(double) * 3 * n);
    int rank = 0;
    s.B.irr_close(&rank);
    s.B.gpunb_close();
    if (stats) *stats = s.st;
    return 0;
}

}  // extern "C"
