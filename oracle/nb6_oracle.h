/*
 * nb6_oracle.h -- FP64 CPU restatement of the Nbody6++GPU force hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the parity checker for the CUDA library,
 * never the thing measured or shipped: only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline leg load it.
 *
 * Parity pin: the restatement is checked against the reference's own CPU
 * libraries (reg.avx.cpp, pot.avx.cpp, irr.avx.cpp compiled from their
 * sources into oracle/_ref) on seeded inputs; the committed fixtures under
 * tests/golden/ were produced by those libraries (tests/golden/make_golden.py).
 *
 * Arrays follow the reference ABI: Fortran X(3,N) == C double[N][3] (AoS),
 * list rows are list[i*lmax + k].
 */
#ifndef NB6_ORACLE_H
#define NB6_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Regular force + jerk + potential + neighbour list, gpunb_regf_ semantics
 * (gpunb.velocity.cu:163-258 pair rule; FP64 loop form of regint.f:39-79).
 * j runs over all nj particles (self included as a neighbour, r2 = 0).
 * Neighbour:  min(r2, |dx + dtr*dv|^2) < h2      (m_flag == 0)
 *             min(r2, |dx + dtr*dv|^2) < m_j*h2  (m_flag != 0)
 * acc/jrk/pot sum over non-neighbours only; pot is positive (sum m/r).
 * list[i*lmax] = nnb, list[i*lmax+1..nnb] = 0-based ascending j; on overflow
 * (nnb > nnbmax or nnb > lmax-1) list[i*lmax] = -nnb and no ids are written.
 * Returns the total neighbour count over all i. */
long orc_regf(int nj, const double *mj, const double *xj, const double *vj,
              int ni, const double *h2, const double *dtr,
              const double *xi, const double *vi,
              int lmax, int nnbmax, int m_flag,
              double *acc, double *jrk, double *pot, int *list);

/* N^2 potential, gpupot_ semantics (gpupot.gpu.cu:32-57; FP64 form of
 * energy.F:65-99): pot[k] = sum_{j: r2>0} m_j / r_ij for
 * i = istart-1+k, k in [0, ni); istart is 1-based. */
void orc_pot(int n, const double *m, const double *x, int istart, int ni,
             double *pot);

/* Hermite predictor of all particles (xbpredall.F:49-61, jpred_int.f:16-25):
 * s = time - t0[j]; x = ((fdot*s + f)*s + x0dot)*s + x0;
 * xdot = (fdot*1.5s + f)*2s + x0dot.  f = a/2, fdot = adot/6. */
void orc_predict(int n, double time, const double *t0, const double *x0,
                 const double *x0dot, const double *f, const double *fdot,
                 double *x, double *xdot);

/* Irregular force + jerk + nearest neighbour over resident lists,
 * irr_simd_firr_vec_ semantics (irr.avx.cpp:499-565) computed in FP64 as in
 * nbint.F:121-159 with jpred_int.f prediction of both i and j to ti.
 * addr[] and list ids are 1-based (Fortran); lists[(a-1)*lmax] = nnb,
 * lists[(a-1)*lmax + 1..nnb] = 1-based j.  nnbid = 1-based j of the minimum
 * r2 (first in list order on ties), or -1 for an empty list. */
void orc_firr(double ti, int ni, const int *addr, int nmax,
              const double *x0, const double *v0, const double *acc2,
              const double *jrk6, const double *mass, const double *t0,
              const int *lists, int lmax,
              double *acc, double *jrk, int *nnbid);

/* KS c.m. corrections of the irregular force, added into acc/jrk of the
 * active bodies addr[ni] (1-based) as NBINT_COR adds them to FIRR and FD
 * (nbint_cor.f:37-65): none for an empty neighbour list; for the c.m. of a
 * perturbed pair, cmfirr_cor.f:13-130 over the pair's perturber list (each
 * perturber that is itself a perturbed pair resolved into its components);
 * for any other body, cmfirr_ucor.f:14-116 over the neighbours that are
 * perturbed pairs.  slot[a-1] = pair p >= 0 when body a is the c.m. of
 * perturbed pair p, else -1; pair p: components' positions xk[p][2][3] and
 * velocities vk[p][2][3] at ti, masses mk[p][2], perturbers
 * plist[pofs[p] .. pofs[p+1]) (1-based).  Bodies are predicted to ti as in
 * orc_firr.  (The chain terms KCPERT_COR / CHFIRR are not restated.) */
void orc_ks_cmcorr(double ti, int ni, const int *addr, const double *x0,
                   const double *v0, const double *acc2, const double *jrk6,
                   const double *mass, const double *t0, const int *lists,
                   int lmax, const int *slot, const double *xk,
                   const double *vk, const double *mk, const int *pofs,
                   const int *plist, double *acc, double *jrk);


/* Ahmad-Cohen neighbour-radius rule of the regular corrector for single
 * bodies, regcor_gpu.F:19-238, with the reference's KZ(39) switch
 * (kz39 = 0 or 2: NB_FLAG = 1; 2 or 3: M_FLAG = 1).  adj = {RDENS[3],
 * RSCALE, RC2, RSFAC, BODYM}: density centre and core radius squared
 * (core.f), half-mass radius (adjust.F:136), RSFAC (adjust.F:199), mean
 * mass.  Per body i: nnb (new list, self removed), nnb0 (old list), dtr =
 * TIME - T0R, xi/vi at TIME, and for nnb <= 3 the first nnb neighbours of
 * the new list at TIME in xnb/vnb[i][3][3].  rs[i] is RS(I) in, the new RS
 * out; dfirr/dfd[i][3] receive the irregular force change the rule starts
 * the neighbour moves with (non-zero only for nnb = 0: the small central
 * mass of :108-118).  Real literals and FLOAT() are single precision as in
 * the reference's build. */
void orc_ac_radius(int n, int kz39, int nnbopt, int nnbmax, const double *adj,
                   const int *nnb, const int *nnb0, const double *dtr,
                   const double *xi, const double *vi,
                   const double *xnb, const double *vnb,
                   double *rs, double *dfirr, double *dfd);

/* Radius shrink of an overflowed regular-force row (util_gpu.F:69-100,
 * fpoly0.F:134-160): nnb_neg[i] < 0 is the row's -NNB. */
void orc_ac_shrink(int n, int kz39, int nnbopt, int nnbmax, const int *nnb_neg, double *rs);

#ifdef __cplusplus
}
#endif
#endif
