/*
 * nb6b200.h -- C ABI of libnb6b200.so, the sm_100a (B200) force hot path of
 * Nbody6++GPU.
 *
 * The first three groups are drop-in replacements for the reference's
 * Fortran-callable libraries: every argument by pointer, Fortran name
 * mangling (lower case, trailing underscore), Fortran X(3,N) arrays passed as
 * C double[N][3].  A Fortran build links this library in place of
 * gpunb.velocity.o / gpunb.gpu.o / gpupot.gpu.o / irr.avx.o; no caller change
 * is needed.  Error behaviour follows the reference (bad input aborts) unless
 * nb6_set_abort_on_error_(0) switches to record-and-return.
 *
 * The last group (nb6_*) are extensions with no reference counterpart.
 */
#ifndef NB6B200_H
#define NB6B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Regular force + jerk + potential + neighbour list                         */
/* replaces gpunb.velocity.cu:905-940 (and gpunb.gpu.cu:820-849,            */
/* reg.avx.cpp:353-385)                                                      */
/* ------------------------------------------------------------------------ */

/* Pick the device: GPU_LIST (first id), NB_GPU_DEVICE, else irank % ngpu.
 * replaces GPUNB_devinit, gpunb.velocity.cu:575-627,906-908 */
void gpunb_devinit_(int *irank);

/* Allocate for up to nbmax j-particles.  gpunb.velocity.cu:629-667,909-911 */
void gpunb_open_(int *nbmax, int *irank);

/* Release device buffers.  gpunb.velocity.cu:669-702,912-914 */
void gpunb_close_(void);

/* Copy nj j-particles (mass, position, velocity) to the device; the caller
 * may overwrite its arrays on return.  gpunb.velocity.cu:704-730,915-921 */
void gpunb_send_(int *nj, double *mj, double (*xj)[3], double (*vj)[3]);

/* For ni i-particles against the last-sent j set: regular acceleration,
 * jerk (adot) and potential (positive, sum m/r) over non-neighbours, and the
 * neighbour list list[i*lmax + 0] = nnb, list[i*lmax + 1..nnb] = 0-based j
 * ascending, self included.  Neighbour: min(r2, |dx + dtr*dv|^2) < h2
 * (m_flag == 0) or < m_j*h2 (m_flag != 0).  If nnb > nnbmax (or lmax-1):
 * list[i*lmax] = -nnb and no ids are written.
 * gpunb.velocity.cu:732-881,922-936 */
void gpunb_regf_(int *ni, double *h2, double *dtr, double (*xi)[3], double (*vi)[3],
                 double (*acc)[3], double (*jrk)[3], double *pot, int *lmax, int *nnbmax,
                 int *list, int *m_flag);

/* Print the "[R.x GPU Reg.F ] ..." line (60 flops per pair) and reset the
 * counters.  gpunb.velocity.cu:883-903,937-939 */
void gpunb_profile_(int *irank);

/* ------------------------------------------------------------------------ */
/* N^2 potential                                                             */
/* replaces gpupot.gpu.cu:116-127 (pot.avx.cpp:354-365)                     */
/* ------------------------------------------------------------------------ */

/* pot[k] = sum_{j: r2 > 0} m_j / r_ij for i = istart-1+k, k in [0, ni);
 * istart is 1-based.  gpupot.gpu.cu:61-114 */
void gpupot_(int *irank, int *istart, int *ni, int *n, double *m, double (*x)[3],
             double *pot);

/* ------------------------------------------------------------------------ */
/* Irregular force + jerk + nearest neighbour over resident lists           */
/* replaces irr.avx.cpp:568-606 (irr.sse.cpp)                               */
/* ------------------------------------------------------------------------ */

/* Allocate state for nmax particles, lists of up to lmax-1 ids.
 * irr.avx.cpp:368-405,569-571 */
void irr_simd_open_(int *nmax, int *lmax, int *rank);

/* irr.avx.cpp:424-438,572-574 */
void irr_simd_close_(int *rank);

/* Print "[R.x GPU Irr.F ] ..." and reset counters.  irr.avx.cpp:407-422,575-577 */
void irr_simd_profile_(int *rank);

/* Set particle addr (1-based): position, velocity, acc2 = F = a/2,
 * jrk6 = FDOT = adot/6, mass, time of last step.  irr.avx.cpp:440-450,579-589 */
void irr_simd_set_jp_(int *addr, double pos[3], double vel[3], double acc2[3], double jrk6[3],
                      double *mass, double *time);

/* Set the neighbour list of addr: nblist[0] = nnb, nblist[1..nnb] = 1-based
 * ids (Fortran LIST(1,I)).  irr.avx.cpp:452-497,590-595 */
void irr_simd_set_list_(int *addr, int *nblist);

/* For ni particles addr[] (1-based): predict them and their neighbours to ti,
 * sum acceleration and jerk over the list; nnbid = 1-based id of the nearest
 * neighbour (-1 for an empty list).  irr.avx.cpp:499-565,596-605 */
void irr_simd_firr_vec_(double *ti, int *ni, int addr[], double acc[][3], double jrk[][3],
                        int nnbid[]);

/* NBODY6/GPU names of the same library, the calls commented out in
 * fpoly0.F:42,70,202,383 and intgrt.F:1329.  gpuirr_open_(nmax, lmax) and
 * gpuirr_close_() use rank 0. */
void gpuirr_open_(int *nmax, int *lmax);
void gpuirr_close_(void);
void gpuirr_set_jp_(int *addr, double pos[3], double vel[3], double acc2[3], double jrk6[3],
                    double *mass, double *time);
void gpuirr_set_list_(int *addr, int *nblist);

/* ------------------------------------------------------------------------ */
/* Extensions (no reference counterpart)                                     */
/* ------------------------------------------------------------------------ */

/* Error policy: flag != 0 aborts on bad input (the reference's behaviour,
 * default), 0 records the code and returns.  nb6_last_status_ returns and
 * clears the first recorded code (0 = ok, 2 bad argument, 3 NaN input,
 * 4 CUDA error, 5 not open, 6 too large, 1 device wait timeout). */
void nb6_set_abort_on_error_(int *flag);
int nb6_last_status_(void);
int nb6_device_(void);

/* gpunb_regf_ on DEVICE arrays (same layout), results kept on the device:
 * nb6_regf_outputs_ returns outf [ni][8] = (acc3, jrk3, pot, 0) and
 * outl [ni][W], W = min(nnbmax, lmax-1) + 1.  Enqueued, no sync. */
void nb6_regf_device_(int *ni, const double *d_h2, const double *d_dtr, const double *d_x,
                      const double *d_v, int *lmax, int *nnbmax, int *m_flag);
void nb6_regf_outputs_(double **d_outf, int **d_outl);
float nb6_regf_last_kernel_ms_(void);
/* geom = (variant, i-grid, j-slices) of the last launch; variant > 0 is the
 * i-parallel kernel with that many i per thread, variant < 0 the j-parallel
 * kernel with -variant i per CTA. */
void nb6_regf_last_geometry_(int *geom);
/* Force a variant (1, 2, 4, -1, -2, -4, -8; 0 = automatic) and a slice count
 * (0 = automatic). */
void nb6_regf_tune_(int *variant, int *nslices);
/* Measured autotuner keyed on (log2 N_active, log2 N_j, m_flag): 1 on
 * (default, or NB6_AUTOTUNE=0 in the environment for off), 0 off, -1 clears
 * the cached choices. */
void nb6_regf_autotune_(int *flag);
/* The autotuner's choices so far (no reference counterpart): *n buckets,
 * out[4k..4k+3] = (log2 N_active, log2 N_j, m_flag, variant) for the first
 * *cap of them, ascending. */
void nb6_regf_tuned_(int *n, int *cap, int *out);
/* Regular-force calls (gpunb_regf_, nb6_regf_device_) are submitted as one
 * CUDA graph launch each: the graph of a call kind is built once and its
 * nodes re-parameterised per call.  flag 1 = on (default; NB6_GRAPHS=0 in
 * the environment for off), 0 = off (plain launches), other values leave it
 * unchanged.  counts[3] receives {graphs built, graph launches, on}. */
void nb6_regf_graphs_(int *flag, long long *counts);
/* After each send the j set is also kept in Morton (Z-curve) order with a
 * bounding box per 128-body tile; the packed kernel skips the neighbour
 * candidate test for tiles out of reach of a whole warp.  Neighbour ids stay
 * the caller's.  Applied to j sets of at least NB6_JSORT_MIN bodies
 * (default 32768).  flag 1 = on (default; NB6_JSORT=0 in the environment for
 * off), 0 = off, other values query.  Returns the setting. */
int nb6_regf_jsort_(int *flag);

/* Segmented regular force for ensembles of independent clusters sent
 * together (one persistent launch for all of them).  Segment c is the j
 * range [seg_j0[c], seg_j0[c+1]) of the last send; active particle k belongs
 * to segment iseg[k] (non-decreasing) and interacts with that segment only.
 * Outputs as gpunb_regf_ (reference layout), list ids relative to
 * seg_j0[iseg[k]].  No reference counterpart: the reference runs one cluster
 * per process. */
void nb6_regf_seg_(int *ni, int *iseg, double *h2, double *dtr, double (*xi)[3], double (*vi)[3],
                   double (*acc)[3], double (*jrk)[3], double *pot, int *lmax, int *nnbmax,
                   int *list, int *m_flag, int *nseg, int *seg_j0);

/* The regular-force j set made on the device from the irregular library's
 * resident records (irr_simd_set_jp_), predicted to *t: segment s is the
 * count[s] records from 1-based address addr0[s], laid out back to back.
 * Replaces XBPREDALL + GPUNB_SEND (intgrt.F:866-882) without host
 * prediction or j upload.  Needs gpunb_open_ and irr_simd_open_. */
void nb6_irr_predict_send_(double *t, int *nseg, int *addr0, int *count);
/* Device time (ms) of the force kernel of the last irr_simd_firr_vec_. */
float nb6_irr_last_kernel_ms_(void);

/* Irregular corrector on the device (the Hermite state stays resident; the
 * host's NBINT_COR work of nbint_cor.f:113-173,215-236 and intgrt.F:533-581
 * per active body).  After irr_simd_open_: nb6_hermite_open_ allocates the
 * per-body state; nb6_hermite_set_ stages a body's FI, FIDOT, FR, FRDOT,
 * STEP, T0R, STEPR, RS (1-based address) like irr_simd_set_jp_ stages its
 * record.  nb6_irr_correct_ computes the neighbour force of the active
 * bodies at *time, applies the corrector, chooses the new irregular step,
 * tests whether the regular step is due and otherwise extrapolates F and
 * FDOT -- updating the device state -- and returns per body out[k][24] =
 * x0[3], v0[3], fi[3], fidot[3], F[3], FDOT[3], step, regular-due (0/1),
 * nnbid, 0, 0, 0.  Each operation is rounded separately in the order of the
 * driver's host corrector, so both give the same bits.  No reference
 * counterpart: the reference corrects on the host. */
void nb6_hermite_open_(double *eta_i, double *smax, double *dtmin);
void nb6_hermite_set_(int *addr, double fi[3], double fidot[3], double fr[3], double frdot[3],
                      double *step, double *t0r, double *stepr, double *rs);
void nb6_irr_correct_(double *time, int *ni, int *addr, double *out);

/* Regular force plus regular corrector on the device (the host's REGCOR_GPU
 * work of regcor_gpu.F:19-238 radius update, :284-444 neighbour gain/loss
 * force moves, :442-537 corrector, :593-737 new regular step), after
 * nb6_irr_predict_send_ has put the j set of the segments on the device and
 * the irregular corrector of the block has run.  addr[ni] are the bodies
 * (1-based, grouped by segment iseg[k]); segment c is j range
 * [seg_j0[c], seg_j0[c+1]) holding the bodies from address seg_a0[c] on.
 * h2, dtr, xi, vi, lmax, nnbmax, m_flag as for nb6_regf_seg_; rs[k] is the
 * radius h2[k] was formed from; prm = {ETAR, SMAX, DTMIN, 25 / TCR, NNBOPT,
 * learned-radius mode (0, or 2 to take the network's proposal as in the
 * driver)}.  The radius rule takes its form and per-cluster quantities from
 * nb6_hermite_adjust_ (prm[3] is RSFAC only while no table is set).  Each
 * body whose list fits gets its
 * radius, neighbour list, Hermite state and regular step updated on the
 * device; out[k][32] = x0[3], v0[3], fi[3], fidot[3], fr[3], frdot[3],
 * F[3], FDOT[3], step, stepr, rs, nnb, overflow (-nnb, else 0),
 * learned-radius outcome (0 none, 1 taken, 2 fallback), 0, 0.  An
 * overflowed body is left as it was, for the caller to shrink its radius
 * and call again with it on the same j set (util_gpu.F:69-100).
 * Operations are rounded as in the driver's host corrector: the same bits
 * with the learned radius off. */
void nb6_regf_correct_(double *time, int *ni, int *addr, int *iseg, int *nseg, int *seg_j0, int *seg_a0,
                       double *h2, double *dtr, double *rs, double (*xi)[3], double (*vi)[3], int *lmax,
                       int *nnbmax, int *m_flag, double *prm, double *out);
/* The Ahmad-Cohen radius rule's form and quantities for nb6_regf_correct_
 * (no reference counterpart as a call: the reference keeps them in common
 * blocks set by ADJUST and CORE, adjust.F:104-199, core.f).  *nb_flag is
 * NB_FLAG of regcor_gpu.F:22 (1 for KZ(39) = 0 or 2: distances from the
 * density centre, membership reduced outside the half-mass radius,
 * radial-velocity volume factor).  Cluster c holds the bodies of 1-based
 * addresses [a0[c], a0[c+1]) (*ncl + 1 entries) with par[8c .. 8c+7] =
 * RDENS[3], RSCALE, RC2, RSFAC = MAX(25/TCR, 1.5 VC/RSMIN), BODYM, 0.  With
 * *ncl = 0 each segment of a call is its own cluster with RDENS = 0,
 * RSCALE = RC2 = 1, RSFAC = prm[3], BODYM = 1 / its body count. */
void nb6_hermite_adjust_(int *nb_flag, int *ncl, int *a0, double *par);
/* The resident neighbour rows of the *n bodies of 1-based addresses addr[]
 * into out[*n][*ls]: [nnb, 1-based ids ascending] with at most *ls - 1 ids
 * and zeros over the 8 entries after the last (no reference counterpart:
 * the reference's host keeps LIST; this is for a host that lets the device
 * regular corrector keep the lists, e.g. for the density centre of
 * core.f). */
void nb6_irr_lists_get_(int *n, const int *addr, int *ls, int *out);
/* KS c.m. corrections of the irregular force (cmfirr_cor.f:13-130,
 * cmfirr_ucor.f:14-116, called from nbint_cor.f:37-65; no reference
 * counterpart in the force libraries: the reference applies them on the
 * host after irr_simd_firr_vec_).  Replaces the table of perturbed KS
 * pairs; *npair = 0 clears it.  Pair p: c.m. body cm[p] (1-based address),
 * component positions xk[p][2][3] and velocities vk[p][2][3] at the time of
 * the coming irregular calls (the host's KS resolution), masses mk[p][2],
 * perturbers of the first component plist[pofs[p] .. pofs[p+1]) (1-based,
 * pofs[0] = 0).  While a table is set, irr_simd_firr_vec_ and
 * nb6_irr_correct_ return FIRR and FD with the corrections included: for a
 * neighbour that is a perturbed pair, its two components replace its
 * point mass; for the c.m. of a perturbed pair, the perturbation of its
 * components by each perturber (resolved too when it is a perturbed pair)
 * minus that perturber's c.m. force is added; an empty neighbour list gets
 * none.  The caller then skips CMFIRR_COR and CMFIRR_UCOR.  The chain terms
 * (KCPERT_COR, CHFIRR, FCHAIN) stay on the host. */
void nb6_ks_set_(int *npair, int *cm, double *xk, double *vk, double *mk, int *pofs, int *plist);

/* Device block clock (no reference counterpart; next_tlist.f and the block
 * loop of intgrt.F run on the host there).  After nb6_hermite_open_ and the
 * state of every body: runs blocks of irregular steps on the device, each
 * block the bodies with the earliest T0 + STEP (bit for bit the host's
 * choice) corrected as by nb6_irr_correct_, until a block has bodies due a
 * regular step (*reason = 1: that block's irregular part is done), the next
 * block time passes *tlimit (*reason = 2: not started) or *max_blocks
 * blocks ran (*reason = 0).  *nblocks, *nirr: blocks and irregular steps of
 * the call; *tblock, *nact: time and active count of the last block.
 * nb6_blocks_regular_ then gives that block's regular-due bodies (ascending
 * 1-based addresses, their corrected x0[3], v0[3] in xv[k][6]) for
 * nb6_irr_predict_send_ + nb6_regf_correct_; nb6_blocks_active_ its whole
 * active set (in no particular order) with the 24-double corrector rows of
 * nb6_irr_correct_. */
void nb6_blocks_run_(double *tlimit, int *max_blocks, int *reason, long long *nblocks, long long *nirr,
                     double *tblock, int *nact);
void nb6_blocks_regular_(int *nreg, int *addr, double *xv);
void nb6_blocks_active_(int *nact, int *addr, double *rows);
/* Launches a large irr_simd_firr_vec_ call is split into (no reference
 * counterpart): 1-4, anything else restores the default 4.  Each launch's
 * results are downloaded and copied into the caller's arrays while the
 * later launches run; 1 gives one launch over every body, then one download
 * and copy. */
void nb6_irr_tune_(int *chunks);
/* Neighbour gathers of irr_simd_firr_vec_ and nb6_irr_correct_ (no
 * reference counterpart): *mode = 1 (the default, or environment
 * NB6_IRR_PV) predicts every record set so far to the call's time once per
 * call, into 64-byte bodies (x, m, v), and walks the lists over those when
 * the call's list entries (active bodies x the mean list length) number at
 * least 4 per body set; 2 always does;
 * 0 never does (each lane then predicts each neighbour from its 128-byte
 * record).  Both walks give the same bits.  Calls with a KS pair table
 * (nb6_ks_set_) always take the record walk. */
void nb6_irr_pv_(int *mode);
/* Form of the device block clock for the following nb6_blocks_run_ calls
 * (no reference counterpart): *persistent = 0 (the default) runs each block
 * as a CUDA graph of two launches; 1 (or environment NB6_BLK_PERSIST=1)
 * runs a whole call as one cooperative launch that loops over blocks, with
 * two grid-wide barriers per block.  Both give the same results bit for
 * bit. */
void nb6_blocks_mode_(int *persistent);

/* The device-resident state of bodies *a0 .. *a0 + *n - 1 (1-based), for a
 * host that lets the device correctors keep it (energy output, the end of
 * a run): rows of 32 doubles x0[3], v0[3], F[3], FDOT[3], fi[3], fidot[3],
 * fr[3], frdot[3], t0, step, t0r, stepr, rs, mass, 0, 0. */
void nb6_hermite_get_(int *a0, int *n, double *out);

/* Learned neighbour radius (no reference counterpart; its fallback is the
 * reference's Ahmad-Cohen rule, regcor_gpu.F:131-196).  A 5-64-64-1 SiLU
 * network, bf16 parameters, FP32 sums, proposing dlog = log(RS_next / RS)
 * from a particle's regular-step features: log(1+nnb), log RS,
 * log(1+nnb) - 1.5 log h2, log|a_reg|, -log2 dtr.  A model is
 * nb6_mlp_size_() floats: 4609 parameters then in_mean[5], in_scale[5],
 * out_mean, out_std.  Training runs on the GPU (Adam, mean squared error in
 * standardised units); x is [n][5], y [n]. */
int nb6_mlp_size_(void);
void nb6_mlp_init_(int *seed);
void nb6_mlp_set_(const float *model);
void nb6_mlp_get_(float *model);
void nb6_mlp_grad_(int *n, const float *x, const float *y, float *grad, float *loss);
void nb6_mlp_train_(int *n, const float *x, const float *y, int *epochs, int *batch, float *lr,
                    int *seed, float *loss_hist);
void nb6_mlp_predict_(int *n, const float *x, float *y);
/* 1: every regular-force call also evaluates the model in its epilogue on
 * its own results; nb6_regf_proposals_ returns the last call's dlog per
 * active particle.  0: off (default). */
void nb6_mlp_enable_(int *flag);
void nb6_regf_proposals_(int *ni, double *out);

/* Synchronise the library stream (and check the device status); the stream
 * handle itself for callers that record events on it. */
void nb6_sync_(void);
void *nb6_stream_(void);

/* gpupot_ on DEVICE arrays; *d_out receives the device result pointer. */
void nb6_pot_device_(int *istart, int *ni, int *n, const double *d_m, const double *d_x,
                     double **d_out);
float nb6_pot_last_kernel_ms_(void);

/* Device-resident Hermite state and predictor (xbpredall.F:48-62 on the GPU).
 * nb6_predict_send_ predicts bodies [ifirst, ifirst+nn) and packs them as the
 * gpunb j set: XBPREDALL + GPUNB_SEND without host traffic. */
void nb6_state_open_(int *nmax);
void nb6_state_close_(void);
void nb6_state_set_(int *n, double *body, double *t0, double (*x0)[3], double (*x0dot)[3],
                    double (*f)[3], double (*fdot)[3]);
void nb6_state_update_(int *nu, int *idx, double *body, double *t0, double (*x0)[3],
                       double (*x0dot)[3], double (*f)[3], double (*fdot)[3]);
void nb6_predict_(double *time, double (*x)[3], double (*xdot)[3]);
void nb6_predict_device_(double *time, double **d_x, double **d_xdot);
void nb6_predict_send_(double *time, int *ifirst, int *nn);
float nb6_predict_last_kernel_ms_(void);

/* Measured FP32 FMA throughput (TFLOP/s) of the current GPU. */
double nb6_fp32_peak_probe_(int *iters);

/* Regular force + jerk + potential + neighbour list that allocates nothing.
 * No counterpart in the reference.  It is for callers that cannot let the
 * library allocate device memory, because another allocator owns the GPU's
 * memory or the run's allocation state must not change mid-run.  Inputs and
 * outputs are caller-provided device-accessible arrays in the gpunb_regf_
 * layouts: j set m[nj], x[nj][3], v[nj][3]; i set h2, dtr, x[ni][3],
 * v[ni][3]; outputs acc[ni][3], jrk[ni][3], pot[ni], list[ni][lmax].
 * Working memory is one fixed 12 MiB device array inside the library,
 * resident on each GPU that loads it until exit.  That bounds a call to
 * ni <= 1024 and min(nnbmax, lmax-1) <= 511; larger sizes are rejected.
 * Work is enqueued on `stream` (a cudaStream_t, 0 = default stream) without
 * waiting.  The first call on a device looks up the array's address, so make
 * it before any stream capture.  Calls share the array: calls that overlap on
 * the GPU race and must not be issued. */
void nb6_regf_noalloc_(int *nj, const double *d_mj, const double *d_xj, const double *d_vj,
                       int *ni, const double *d_h2, const double *d_dtr, const double *d_xi,
                       const double *d_vi, double *d_acc, double *d_jrk, double *d_pot, int *lmax,
                       int *nnbmax, int *d_list, int *m_flag, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* NB6B200_H */
