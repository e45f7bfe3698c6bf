/*
 * nb6_oracle.c -- FP64 CPU restatement of the Nbody6++GPU force hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product).  Each function
 * cites the reference lines it restates; arithmetic is plain IEEE double with
 * no reassociation tricks, so it is the "FP64 direct-sum oracle" that the
 * CUDA kernels' relative errors are stated against.
 */
#include "nb6_oracle.h"

#include <math.h>
#include <stdlib.h>

long orc_regf(int nj, const double *mj, const double *xj, const double *vj,
              int ni, const double *h2, const double *dtr,
              const double *xi, const double *vi,
              int lmax, int nnbmax, int m_flag,
              double *acc, double *jrk, double *pot, int *list)
{
    long total = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : total)
    for (int i = 0; i < ni; i++) {
        const double x0 = xi[3 * i], x1 = xi[3 * i + 1], x2 = xi[3 * i + 2];
        const double v0 = vi[3 * i], v1 = vi[3 * i + 1], v2 = vi[3 * i + 2];
        const double hh = h2[i], dt = dtr[i];
        double ax = 0, ay = 0, az = 0, jx = 0, jy = 0, jz = 0, po = 0;
        int *row = list + (long)i * lmax;
        int nnb = 0;
        const int cap = (nnbmax < lmax - 1) ? nnbmax : lmax - 1;
        /* ids go to scratch first: an overflowed row gets no ids */
        int *ids = (int *)malloc(sizeof(int) * (size_t)(cap > 0 ? cap : 1));
        for (int j = 0; j < nj; j++) {
            /* gpunb.velocity.cu:169-185 / regint.f:41-58 */
            const double dx = xj[3 * j] - x0;
            const double dy = xj[3 * j + 1] - x1;
            const double dz = xj[3 * j + 2] - x2;
            const double dvx = vj[3 * j] - v0;
            const double dvy = vj[3 * j + 1] - v1;
            const double dvz = vj[3 * j + 2] - v2;
            const double r2 = dx * dx + dy * dy + dz * dz;
            const double px = dx + dt * dvx, py = dy + dt * dvy, pz = dz + dt * dvz;
            const double r2p = px * px + py * py + pz * pz;
            const double rmin = (r2 < r2p) ? r2 : r2p;
            const double crit = m_flag ? mj[j] * hh : hh;
            if (rmin < crit) {
                /* neighbour: recorded, contributes nothing (:188-193) */
                if (nnb < cap) ids[nnb] = j;
                nnb++;
                continue;
            }
            const double rv = dx * dvx + dy * dvy + dz * dvz;
            const double rinv2 = 1.0 / r2;
            const double rinv = sqrt(rinv2);
            const double mr = mj[j] * rinv;
            const double mr3 = mr * rinv2;
            const double alpha = -3.0 * rv * rinv2;
            po += mr;
            ax += mr3 * dx;
            ay += mr3 * dy;
            az += mr3 * dz;
            jx += mr3 * (dvx + alpha * dx);
            jy += mr3 * (dvy + alpha * dy);
            jz += mr3 * (dvz + alpha * dz);
        }
        acc[3 * i] = ax; acc[3 * i + 1] = ay; acc[3 * i + 2] = az;
        jrk[3 * i] = jx; jrk[3 * i + 1] = jy; jrk[3 * i + 2] = jz;
        pot[i] = po;
        /* overflow contract: reg.avx.cpp:320-327 (negative count) */
        row[0] = (nnb > cap) ? -nnb : nnb;
        if (nnb <= cap)
            for (int k = 0; k < nnb; k++) row[1 + k] = ids[k];
        free(ids);
        total += nnb;
    }
    return total;
}

void orc_pot(int n, const double *m, const double *x, int istart, int ni,
             double *pot)
{
    const int i0 = istart - 1;
#pragma omp parallel for schedule(dynamic, 8)
    for (int k = 0; k < ni; k++) {
        const int i = i0 + k;
        const double x0 = x[3 * i], x1 = x[3 * i + 1], x2 = x[3 * i + 2];
        double p = 0.0;
        for (int j = 0; j < n; j++) {
            const double dx = x[3 * j] - x0;
            const double dy = x[3 * j + 1] - x1;
            const double dz = x[3 * j + 2] - x2;
            const double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 > 0.0) p += m[j] / sqrt(r2); /* gpupot.gpu.cu:48-52 */
        }
        pot[k] = p;
    }
}

static inline void pred1(double s, const double *x0, const double *x0dot,
                         const double *f, const double *fdot, double *x,
                         double *xd)
{
    /* xbpredall.F:50-59 */
    const double s1 = 1.5 * s, s2 = 2.0 * s;
    for (int k = 0; k < 3; k++) {
        x[k] = ((fdot[k] * s + f[k]) * s + x0dot[k]) * s + x0[k];
        xd[k] = (fdot[k] * s1 + f[k]) * s2 + x0dot[k];
    }
}

void orc_predict(int n, double time, const double *t0, const double *x0,
                 const double *x0dot, const double *f, const double *fdot,
                 double *x, double *xdot)
{
#pragma omp parallel for schedule(static)
    for (int j = 0; j < n; j++)
        pred1(time - t0[j], x0 + 3 * j, x0dot + 3 * j, f + 3 * j,
              fdot + 3 * j, x + 3 * j, xdot + 3 * j);
}

void orc_firr(double ti, int ni, const int *addr, int nmax,
              const double *x0, const double *v0, const double *acc2,
              const double *jrk6, const double *mass, const double *t0,
              const int *lists, int lmax,
              double *acc, double *jrk, int *nnbid)
{
    (void)nmax;
#pragma omp parallel for schedule(dynamic, 4)
    for (int k = 0; k < ni; k++) {
        const int i = addr[k] - 1;
        double xi[3], vi[3];
        pred1(ti - t0[i], x0 + 3 * i, v0 + 3 * i, acc2 + 3 * i, jrk6 + 3 * i,
              xi, vi);
        const int *row = lists + (long)i * lmax;
        const int nnb = row[0];
        double ax = 0, ay = 0, az = 0, jx = 0, jy = 0, jz = 0;
        double rmin = INFINITY;
        int imin = -1;
        for (int l = 1; l <= nnb; l++) {
            /* nbint.F:133-158 */
            const int j = row[l] - 1;
            double xj[3], vj[3];
            pred1(ti - t0[j], x0 + 3 * j, v0 + 3 * j, acc2 + 3 * j,
                  jrk6 + 3 * j, xj, vj);
            const double dx = xj[0] - xi[0], dy = xj[1] - xi[1], dz = xj[2] - xi[2];
            const double dvx = vj[0] - vi[0], dvy = vj[1] - vi[1], dvz = vj[2] - vi[2];
            const double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 < rmin) { rmin = r2; imin = j + 1; }
            const double rinv2 = 1.0 / r2;
            const double mr3 = mass[j] * rinv2 * sqrt(rinv2);
            const double drdp = 3.0 * (dx * dvx + dy * dvy + dz * dvz) * rinv2;
            ax += dx * mr3; ay += dy * mr3; az += dz * mr3;
            jx += (dvx - dx * drdp) * mr3;
            jy += (dvy - dy * drdp) * mr3;
            jz += (dvz - dz * drdp) * mr3;
        }
        acc[3 * k] = ax; acc[3 * k + 1] = ay; acc[3 * k + 2] = az;
        jrk[3 * k] = jx; jrk[3 * k + 1] = jy; jrk[3 * k + 2] = jz;
        nnbid[k] = imin;
    }
}

/* Force and jerk on a body at (xi, vi) from a point mass m at (xj, vj), in
 * the operation order of cmfirr_cor.f:47-93 / cmfirr_ucor.f:58-104. */
static void cm_pair(const double *xi, const double *vi, const double *xj,
                    const double *vj, double m, double *f, double *fd)
{
    double dx[3], dv[3], dr2 = 0.0, drdv = 0.0;
    for (int l = 0; l < 3; l++) {
        dx[l] = xj[l] - xi[l];
        dv[l] = vj[l] - vi[l];
        dr2 += dx[l] * dx[l];
        drdv += dx[l] * dv[l];
    }
    const double dr2i = 1.0 / dr2;
    const double dr3i = m * dr2i * sqrt(dr2i);
    drdv = 3.0 * drdv * dr2i;
    for (int l = 0; l < 3; l++) {
        f[l] = dx[l] * dr3i;
        fd[l] = (dv[l] - dx[l] * drdv) * dr3i;
    }
}

void orc_ks_cmcorr(double ti, int ni, const int *addr, const double *x0,
                   const double *v0, const double *acc2, const double *jrk6,
                   const double *mass, const double *t0, const int *lists,
                   int lmax, const int *slot, const double *xk,
                   const double *vk, const double *mk, const int *pofs,
                   const int *plist, double *acc, double *jrk)
{
#pragma omp parallel for schedule(dynamic, 4)
    for (int k = 0; k < ni; k++) {
        const int i = addr[k] - 1;
        const int *row = lists + (long)i * lmax;
        if (row[0] == 0) continue;  /* nbint_cor.f:37-49: no corrections */
        double xi[3], vi[3];
        pred1(ti - t0[i], x0 + 3 * i, v0 + 3 * i, acc2 + 3 * i, jrk6 + 3 * i, xi, vi);
        double cf[3] = {0, 0, 0}, cd[3] = {0, 0, 0};
        const int p = slot[i];
        if (p >= 0) {
            /* cmfirr_cor.f: perturbed pair i, corrections over the
             * perturbers of its first component */
            const double *x1 = xk + 6 * p, *x2 = xk + 6 * p + 3;
            const double *v1 = vk + 6 * p, *v2 = vk + 6 * p + 3;
            const double m1 = mk[2 * p], m2 = mk[2 * p + 1], mi = mass[i];
            for (int l = pofs[p]; l < pofs[p + 1]; l++) {
                const int j = plist[l] - 1;
                double xj[3], vj[3], fcm[3], fcmd[3];
                pred1(ti - t0[j], x0 + 3 * j, v0 + 3 * j, acc2 + 3 * j, jrk6 + 3 * j, xj, vj);
                cm_pair(xi, vi, xj, vj, mass[j], fcm, fcmd);
                const int q = slot[j];
                const int nk = q >= 0 ? 2 : 1;   /* resolve a perturbed pair j */
                for (int c = 0; c < nk; c++) {
                    const double *xkk = q >= 0 ? xk + 6 * q + 3 * c : xj;
                    const double *vkk = q >= 0 ? vk + 6 * q + 3 * c : vj;
                    const double mkk = q >= 0 ? mk[2 * q + c] : mass[j];
                    double fp1[3], fpd1[3], fp2[3], fpd2[3];
                    cm_pair(x1, v1, xkk, vkk, mkk, fp1, fpd1);
                    cm_pair(x2, v2, xkk, vkk, mkk, fp2, fpd2);
                    for (int d = 0; d < 3; d++) {
                        /* the c.m. term enters once, with the first component */
                        const double sc = c == 0 ? fcm[d] : 0.0, sd = c == 0 ? fcmd[d] : 0.0;
                        cf[d] += (m1 * fp1[d] + m2 * fp2[d]) / mi - sc;
                        cd[d] += (m1 * fpd1[d] + m2 * fpd2[d]) / mi - sd;
                    }
                }
            }
        } else {
            /* cmfirr_ucor.f: neighbours that are perturbed pairs summed over
             * their components */
            for (int l = 1; l <= row[0]; l++) {
                const int j = row[l] - 1;
                const int q = slot[j];
                if (q < 0) continue;
                double xj[3], vj[3], fcm[3], fcmd[3], fp1[3], fpd1[3], fp2[3], fpd2[3];
                pred1(ti - t0[j], x0 + 3 * j, v0 + 3 * j, acc2 + 3 * j, jrk6 + 3 * j, xj, vj);
                cm_pair(xi, vi, xj, vj, mass[j], fcm, fcmd);
                cm_pair(xi, vi, xk + 6 * q, vk + 6 * q, mk[2 * q], fp1, fpd1);
                cm_pair(xi, vi, xk + 6 * q + 3, vk + 6 * q + 3, mk[2 * q + 1], fp2, fpd2);
                for (int d = 0; d < 3; d++) {
                    cf[d] += fp1[d] + fp2[d] - fcm[d];
                    cd[d] += fpd1[d] + fpd2[d] - fcmd[d];
                }
            }
        }
        for (int d = 0; d < 3; d++) {
            acc[3 * k + d] += cf[d];
            jrk[3 * k + d] += cd[d];
        }
    }
}

/* ------------------------------------------------------------------------
 * Ahmad-Cohen neighbour-radius rule of the regular corrector,
 * regcor_gpu.F:19-238 (single bodies, I <= N), and the overflow shrink of
 * util_gpu.F:69-100 / fpoly0.F:134-160.
 *
 * The reference is compiled without -fdefault-real-8, so its real literals
 * (0.1, 0.9, 0.003, 1.05, 1.1, ...) and FLOAT(int) are REAL*4: mixed with a
 * REAL*8 operand such a literal enters as its single-precision value, and an
 * expression of REAL*4 terms only (FAC, DRS, the overflow factors) is
 * evaluated in single precision.  R4() writes those literals; the single
 * precision expressions are computed in float.  No FMA contraction (the
 * Fortran is compiled for -mavx without FMA).
 * ------------------------------------------------------------------------ */
#define R4(c) ((double)(c##f))

void orc_ac_radius(int n, int kz39, int nnbopt, int nnbmax, const double *adj,
                   const int *nnb_in, const int *nnb0_in, const double *dtr_in,
                   const double *xi, const double *vi,
                   const double *xnb, const double *vnb,
                   double *rs, double *dfirr, double *dfd)
{
    const int m_flag = (kz39 == 2 || kz39 == 3);   /* regcor_gpu.F:21-22 */
    const int nb_flag = (kz39 == 0 || kz39 == 2);
    const double *rdens = adj;
    const double rscale = adj[3], rc2 = adj[4], rsfac = adj[5], bodym = adj[6];
    const double one3 = 1.0 / 3.0;                 /* zero.f:113 */
    /* input.F:133: ZNBMIN = MAX(0.01*FLOAT(NNBMAX),1.0) */
    const float zs = 0.01f * (float)nnbmax;
    const double znbmin = (double)(zs > 1.0f ? zs : 1.0f);
    for (int i = 0; i < n; i++) {
        const double *x = xi + 3 * i, *v = vi + 3 * i;
        const int nnb = nnb_in[i], nnb0 = nnb0_in[i];
        const double dtr = dtr_in[i];
        double *df = dfirr + 3 * i, *dd = dfd + 3 * i;
        df[0] = df[1] = df[2] = dd[0] = dd[1] = dd[2] = 0.0;
        double ri2, rh2;
        if (nb_flag) {                                /* :30-37 */
            const double a = x[0] - rdens[0], b = x[1] - rdens[1], c = x[2] - rdens[2];
            ri2 = a * a + b * b + c * c;
            rh2 = rscale * rscale;
        } else {
            ri2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
            rh2 = R4(9.0) * (rscale * rscale);
        }
        if (nnb == 0) {                               /* :108-131 */
            const double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
            const double fij = R4(0.01) * bodym / (r2 * sqrt(r2));
            const double rdot = 3.0 * (x[0] * v[0] + x[1] * v[1] + x[2] * v[2]) / r2;
            for (int k = 0; k < 3; k++) {
                df[k] = -fij * x[k];
                dd[k] = -(v[k] - rdot * x[k]) * fij;
            }
            if (rdot > 0.0) {
                const double a = R4(0.75) * rs[i], b = R4(0.1) * rscale;
                rs[i] = a > b ? a : b;
            } else {
                rs[i] = R4(1.1) * rs[i];
            }
            continue;                                 /* GO TO 50 */
        }
        /* :139-150 */
        const float fac_s = 1.0f + 0.1f * ((float)nnbopt - (float)nnb) / (float)nnb;
        const double fac = (double)fac_s;
        double a3 = (double)(float)nnb * fac;
        int nbave = nnbmax - 50 > (int)znbmin ? nnbmax - 50 : (int)znbmin;
        nbave = nnbopt + 150 < nbave ? nnbopt + 150 : nbave;
        const double cap = (double)(0.9f * (float)nbave);
        a3 = a3 < cap ? a3 : cap;
        const int nbp = (int)a3;
        if (ri2 > rh2 && nb_flag) {                   /* :152-156 */
            const double f = rscale / sqrt(ri2);
            a3 = a3 * (f > R4(0.1) ? f : R4(0.1));
        } else {
            a3 = a3 > znbmin ? a3 : znbmin;
        }
        double a4 = a3 / (double)(float)nnb;
        if ((a3 - (double)(float)nnb0) * (a3 - (double)(float)nnb) < 0.0) a4 = sqrt(a4);
        /* :162-167, RIDOT relative to the density centre in both forms */
        const double ridot = (x[0] - rdens[0]) * v[0] + (x[1] - rdens[1]) * v[1] +
                             (x[2] - rdens[2]) * v[2];
        if (ri2 > rc2 && nb_flag && ri2 < R4(100.0) * rh2)
            a4 = a4 * (1.0 + ridot * dtr / ri2);
        /* (:170-181, the c.m. perturber range, applies to I > N only) */
        double a5 = rsfac * dtr;                      /* :184-192 */
        a5 = a5 < 0.25 ? a5 : 0.25;
        a4 = a4 - 1.0;
        if (a4 > a5) a4 = a5;
        else a4 = a4 > -a5 ? a4 : -a5;
        const double a3b = one3 * a4;                 /* :195-213 */
        double a1 = 1.0 + a3b - a3b * a3b;
        if (nnb < znbmin && nbp > znbmin)
            if (a1 < 1.0) a1 = R4(1.05);
        if (fabs(a1 - 1.0) > R4(0.003)) {
            if (rs[i] * rs[i] > ri2 && rs[i] * rs[i] < 2.0 * ri2 && nnb > 5) a1 = sqrt(a1);
            rs[i] = a1 * rs[i];
        }
        if (nnb > nbave && ridot < 0.0) {             /* :215-220 */
            const float drs = ((float)nnb - (float)nbave) / (3.0f * (float)nnb);
            rs[i] = rs[i] * (1.0 - (double)drs);
        }
        if (!m_flag && nnb <= 3 && ri2 < R4(100.0) * rh2) {   /* :223-238 */
            double a1b = 2.0 * rs[i];
            for (int l = 0; l < nnb; l++) {
                const double *xj = xnb + 9 * i + 3 * l, *vj = vnb + 9 * i + 3 * l;
                const double ex = x[0] - xj[0], ey = x[1] - xj[1], ez = x[2] - xj[2];
                const double rij = sqrt(ex * ex + ey * ey + ez * ez);
                const double rsdot = (ex * (v[0] - vj[0]) + ey * (v[1] - vj[1]) +
                                      ez * (v[2] - vj[2])) / rij;
                const double t = rij + rsdot * dtr;
                a1b = a1b < t ? a1b : t;
            }
            const double g = R4(1.1) * rs[i];
            rs[i] = a1b > g ? a1b : g;
        }
    }
}

void orc_ac_shrink(int n, int kz39, int nnbopt, int nnbmax, const int *nnb_neg, double *rs)
{
    const int nb_flag = (kz39 == 0 || kz39 == 2);
    for (int i = 0; i < n; i++) {
        const int nnb = nnb_neg[i];                   /* negative: the overflow count */
        if (nb_flag) {                                /* util_gpu.F:80-85 */
            float f;
            if (-nnb > nnbopt) f = powf(-(float)nnbopt / (float)nnb, 0.333f);
            else f = powf((float)nnbopt / (float)nnbmax, 0.4f);
            rs[i] = (double)f * rs[i];
        } else {
            rs[i] = R4(0.9) * rs[i];                  /* :87 */
        }
    }
}
