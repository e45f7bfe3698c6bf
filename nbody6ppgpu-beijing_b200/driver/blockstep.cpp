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
//   radius-rule quantities       adjust.F:104-199, core.f, output.F:61,271
//                                at TIME = 0 and every DTADJ (at outputs)
// The per-body steps live in hermite.h (shared with the ensemble driver).
// Left out: KS/chain regularisation, stellar evolution, external fields,
// the checkl/fpcorr options (KZ(37), KZ(38)) and the SMIN neighbour retention.
//
// The same code runs on any backend that exports the ABI: libnb6b200.so or
// the reference's CPU libraries compiled from source.  Backends are loaded
// with dlopen(RTLD_LOCAL) from the paths the caller gives.
#include "hermite.h"

namespace {

using namespace nb6drv;

struct Sim : Bodies {
    Backend B;
    double time = 0;
    std::vector<double> xp, vp;  // predicted positions / velocities (all bodies)
    std::vector<double> prop;    // learned dlog RS of the last regular_forces rows

    void predict_all(double t) {
        for (int j = 0; j < n; ++j) pred(j, t, &xp[3 * (size_t)j], &vp[3 * (size_t)j]);
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
    // row (util_gpu.F:69-100).
    void regular_forces(const std::vector<int> &idx, std::vector<double> &freg,
                        std::vector<double> &fdr, std::vector<int> &nlist) {
        const double t_0 = wtime();
        predict_all(time);
        int nn = n;
        B.gpunb_send(&nn, m.data(), (double(*)[3])xp.data(), (double(*)[3])vp.data());
        const double bodym = 1.0 / n;
        freg.assign(3 * idx.size(), 0.0);
        fdr.assign(3 * idx.size(), 0.0);
        nlist.assign(idx.size() * (size_t)LS, 0);
        prop.assign(idx.size(), 0.0);
        auto fill = [&](int i, double *xi, double *vi) {
            for (int k = 0; k < 3; ++k) {
                xi[k] = xp[3 * (size_t)i + k];
                vi[k] = vp[3 * (size_t)i + k];
            }
        };
        auto take = [&](int q, int i, const int *row, const double *acc, const double *jrk) {
            for (int k = 0; k < 3; ++k) {
                freg[3 * (size_t)q + k] = acc[k];
                fdr[3 * (size_t)q + k] = jrk[k];
            }
            int *out = &nlist[(size_t)q * LS];
            int l1 = 0;
            for (int l = 1; l <= row[0]; ++l)
                if (row[l] != i) out[1 + l1++] = row[l] + 1;
            out[0] = l1;
        };
        regf_rows(B, idx, 0, (int)idx.size(), n, bodym, fill, take, prop);
        st.wall_reg += wtime() - t_0;
    }

    // the neighbour rows core.f reads, from the host's lists
    auto host_rows() {
        return [this](const std::vector<int> &jl, std::vector<const int *> &rp) {
            for (size_t l = 0; l < jl.size(); ++l) rp[l] = row(jl[l]);
        };
    }

    bool init();
    void regular_step(const std::vector<int> &reg);
    bool run(double *eout, int nout_max);
    void energy(double &ekin, double &epot);
};

bool Sim::init() {
    alloc();
    adjust_init(1);
    xp.assign(3 * (size_t)n, 0);
    vp.assign(3 * (size_t)n, 0);
    for (int i = 0; i < n; ++i) init_radius(i, &x0[3 * (size_t)i]);
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
    fpoly0 = true;
    regular_forces(all, freg, fdr, nl);
    fpoly0 = false;
    for (int i = 0; i < n; ++i) memcpy(row(i), &nl[(size_t)i * LS], sizeof(int) * LS);
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
        init_forces(i, &freg[3 * (size_t)i], &fdr[3 * (size_t)i], &a[3 * (size_t)i], &jd[3 * (size_t)i]);
        set_jp(i);
    }
    return true;
}

void Sim::regular_step(const std::vector<int> &reg) {
    std::vector<double> freg, fdr;
    std::vector<int> nl;
    regular_forces(reg, freg, fdr, nl);
    snapshot(reg, time);
    const double bodym = 1.0 / n;
    for (size_t q = 0; q < reg.size(); ++q) {
        const int i = reg[q];
        const int *row_new = &nl[q * (size_t)LS];
        const double rs_used = rs[i];
        if (P.mlp_mode == 1) learn_log(i, row_new[0], rs_used, h2_of(i, bodym), &freg[3 * q], stepr[i]);
        reg_correct(i, time, row_new, &freg[3 * q], &fdr[3 * q]);
        if (P.mlp_mode == 2) learn_apply(i, row_new[0], rs_used, prop[q]);
        set_list(i);
    }
    release_snapshot(reg);
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
    if (adjust_due(time)) adjust(0, 0, n, xp.data(), vp.data(), ek, -ep, host_rows(), time);
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
    clock_reset();
    while (st.blocks < P.max_blocks) {
        const double tmin = clock_next(active);
        if (tmin > P.tcrit + 1e-12) break;
        time = tmin;
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
        for (int q = 0; q < na; ++q)
            if (irr_correct(active[q], time, &a[3 * (size_t)q], &jd[3 * (size_t)q])) reg.push_back(active[q]);
        if (!reg.empty()) regular_step(reg);
        for (int q = 0; q < na; ++q) set_jp(active[q]);
        clock_push(active);
        if (time >= tnext_out - 1e-15) {
            energy(ek, ep);
            if (adjust_due(time)) adjust(0, 0, n, xp.data(), vp.data(), ek, -ep, host_rows(), time);
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
    if (s.P.mlp_mode == 2 && !s.B.proposals) {
        fprintf(stderr, "nb6drive: mlp_mode 2 needs a backend with nb6_regf_proposals_\n");
        return 4;
    }
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

// The driver's Ahmad-Cohen radius rule (ac_radius) for n bodies of one
// cluster, with the argument layout of the oracle's restatement:
// kz39 selects NB_FLAG and M_FLAG as regcor_gpu.F:21-22 does; adj =
// RDENS[3], RSCALE, RC2, RSFAC, BODYM; xnb/vnb[n][3][3] the first
// min(nnb, 3) new neighbours.  rs in/out; dfirr/dfd[n][3] out.  For tests.
void nb6drive_ac_radius(int n, int kz39, int nnbopt, int nnbmax, const double *adj, const int *nnb,
                        const int *nnb0, const double *dtr, const double *xi, const double *vi,
                        const double *xnb, const double *vnb, double *rs, double *dfirr, double *dfd) {
    ACPar a;
    for (int k = 0; k < 3; ++k) a.rdens[k] = adj[k];
    a.rscale = adj[3];
    a.rc2 = adj[4];
    a.rsfac = adj[5];
    a.bodym = adj[6];
    const int nb_flag = (kz39 == 0 || kz39 == 2), m_flag = (kz39 == 2 || kz39 == 3);
    for (int i = 0; i < n; ++i)
        rs[i] = ac_radius(nb_flag, m_flag, nnbopt, nnbmax, a, nnb[i], nnb0[i], dtr[i], xi + 3 * i, vi + 3 * i,
                          xnb + 9 * i, vnb + 9 * i, rs[i], dfirr + 3 * i, dfd + 3 * i);
}

// The driver's overflow shrink (ac_shrink) of n radii; nnb_neg[i] = -NNB.
void nb6drive_ac_shrink(int n, int kz39, int nnbopt, int nnbmax, const int *nnb_neg, double *rs) {
    const int nb_flag = (kz39 == 0 || kz39 == 2);
    for (int i = 0; i < n; ++i) rs[i] = ac_shrink(nb_flag, nnbopt, nnbmax, nnb_neg[i], rs[i]);
}

// The driver's core.f restatement (ac_core) on one cluster of n bodies:
// rows[n][ls] = [nnb, 1-based neighbour ids]; io = {RDENS[3], RSCALE, RC
// of the last call} in, {RDENS[3], RSCALE, RC, RC2, VC} out.  For tests.
void nb6drive_core(int n, const double *m, const double *x, const double *v, const double *rs, const int *rows,
                   int ls, double time, double *io) {
    ACPar a;
    for (int k = 0; k < 3; ++k) a.rdens[k] = io[k];
    a.rscale = io[3];
    double rc = io[4];
    auto rows_of = [rows, ls](const std::vector<int> &jl, std::vector<const int *> &rp) {
        for (size_t l = 0; l < jl.size(); ++l) rp[l] = rows + (size_t)jl[l] * ls;
    };
    const double vc = ac_core(n, m, x, v, rs, rows_of, 0, time, a, rc);
    for (int k = 0; k < 3; ++k) io[k] = a.rdens[k];
    io[4] = rc;
    io[5] = a.rc2;
    io[6] = vc;
}

}  // extern "C"
