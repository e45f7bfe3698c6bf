// ensemble.cpp -- block-step integration of an ensemble of independent star
// clusters on one GPU, with each force kind issued once per block for all
// clusters together.
//
// Each cluster keeps its own Henon units and its own block-step hierarchy:
// the per-body steps are those of the single-cluster driver (hermite.h), and
// a body's step sequence depends only on its own cluster, so every cluster
// follows the trajectory it would follow alone.  What changes is how the
// force calls are issued.  The bodies of all clusters share one address
// space (cluster c holds addresses base[c]+1 .. base[c]+n[c]); at each global
// block time (the earliest t0 + step over all bodies):
//   * one irr_simd_firr_vec_ for the active bodies of every cluster (their
//     neighbour lists only hold bodies of their own cluster);
//   * when regular steps are due: the j set of the clusters involved made on
//     the device from the irregular library's resident records
//     (nb6_irr_predict_send_), and one nb6_regf_seg_ for all due bodies,
//     segment = cluster.
// With a backend lacking those two extension calls (the reference's CPU
// libraries) or with batched = 0, the regular force falls back to one
// host-predicted gpunb_send_ and chunked gpunb_regf_ calls per cluster, which
// is what running each cluster alone does.
//
// Energies are computed per cluster (gpupot_ on the cluster's own bodies).
#include "hermite.h"

#include <functional>

namespace {

using namespace nb6drv;

struct Ensemble : Bodies {
    Backend B;
    bool batched = true;
    int ncl = 0;
    std::vector<int> base, cnt, cl_of;
    double time = 0;
    std::vector<double> prop;  // learned dlog RS per row of the last regular_forces
    std::vector<double> crow;  // device corrector rows of the last block
    std::vector<double> rrow;  // device regular corrector rows of the last call
    double t_pred = 0;         // wall time in nb6_irr_predict_send_ (device regular corrector)
    double t_rcall = 0;        // ... in nb6_regf_correct_
    double t_out = 0;          // ... in energy output (state read-back + energies)
    double t_breg = 0;         // ... in nb6_blocks_regular_
    // per-call buffers of the batched regular force, kept across calls (the
    // library writes every entry that is read back)
    std::vector<int> b_iseg, b_lst;
    std::vector<double> b_h2, b_dtr, b_xi, b_vi, b_acc, b_jrk, b_pot, b_prop;

    int cluster_count(int c) const { return cnt[c]; }

    void set_jp(int i) {
        int a = i + 1;
        double mm = m[i], tt = t0[i];
        B.irr_set_jp(&a, &x0[3 * i], &v0[3 * i], &f[3 * i], &fdot[3 * i], &mm, &tt);
    }

    void set_list(int i) {
        int a = i + 1;
        B.irr_set_list(&a, row(i));
    }

    // irregular corrector on the device (batched mode, backend permitting)
    bool dev_corr() const { return batched && P.dev_corrector && B.irr_correct && B.hermite_set && B.hermite_open; }

    // regular corrector on the device too (needs the irregular one there)
    bool dev_reg() const {
        return dev_corr() && P.dev_corrector >= 2 && B.regf_correct && B.hermite_get && B.predict_send &&
               P.mlp_mode != 1;
    }

    // With both correctors on the device the host keeps only what the block
    // clock and the force calls need (t0, step, t0r, stepr, rs, and x0, v0
    // of the bodies due a regular step); the rest is read back here for
    // energies and at the end.
    void pull_state() {
        const int chunk = 1 << 16;
        std::vector<double> rowbuf(32 * (size_t)std::min(n, chunk));
        for (int a = 0; a < n; a += chunk) {
            int a0 = a + 1, k = std::min(chunk, n - a);
            B.hermite_get(&a0, &k, rowbuf.data());
            for (int q = 0; q < k; ++q) {
                const int i = a + q;
                const double *o = &rowbuf[32 * (size_t)q];
                for (int c = 0; c < 3; ++c) {
                    const size_t j = 3 * (size_t)i + c;
                    x0[j] = o[c];
                    v0[j] = o[3 + c];
                    f[j] = o[6 + c];
                    fdot[j] = o[9 + c];
                    fi[j] = o[12 + c];
                    fidot[j] = o[15 + c];
                    fr[j] = o[18 + c];
                    frdot[j] = o[21 + c];
                }
                t0[i] = o[24];
                step[i] = o[25];
                t0r[i] = o[26];
                stepr[i] = o[27];
                rs[i] = o[28];
            }
        }
    }

    void set_hermite(int i) {
        int a = i + 1;
        double s = step[i], tr = t0r[i], sr = stepr[i], r = rs[i];
        B.hermite_set(&a, &fi[3 * (size_t)i], &fidot[3 * (size_t)i], &fr[3 * (size_t)i], &frdot[3 * (size_t)i], &s,
                      &tr, &sr, &r);
    }

    // Regular force and regular corrector of the bodies in idx (ascending)
    // on the device, one nb6_regf_correct_ per pass: the j set of the
    // clusters involved is predicted once (every body as it stands before
    // any regular correction of this block, as the host snapshot has it);
    // rows that overflowed come back untouched, get a smaller radius here
    // and go again.  The host keeps the new steps and radii of the rows.
    // per-call buffers of regular_on_device, kept across calls
    std::vector<int> r_runc, r_segq, r_addr0, r_count, r_segj0, r_pend, r_again, r_addr;
    std::vector<double> r_rs;

    // xv: when given, x0, v0 of the bodies in idx order (6 doubles each),
    // else the host copies x0, v0 are read
    void regular_on_device(const std::vector<int> &idx, const double *xv = nullptr) {
        const double t_0 = wtime();
        const size_t ni = idx.size();
        auto grow = [](auto &v, size_t k) {
            if (v.size() < k) v.resize(k);
        };
        std::vector<int> &runc = r_runc, &seg_of_q = r_segq;
        runc.clear();
        grow(seg_of_q, ni);
        for (size_t q = 0; q < ni; ++q) {
            if (q == 0 || cl_of[idx[q]] != cl_of[idx[q - 1]]) runc.push_back(cl_of[idx[q]]);
            seg_of_q[q] = (int)runc.size() - 1;
        }
        int nseg = (int)runc.size();
        std::vector<int> &addr0 = r_addr0, &count = r_count, &seg_j0 = r_segj0;
        addr0.resize(nseg);
        count.resize(nseg);
        seg_j0.assign(nseg + 1, 0);
        for (int r = 0; r < nseg; ++r) {
            addr0[r] = base[runc[r]] + 1;
            count[r] = cnt[runc[r]];
            seg_j0[r + 1] = seg_j0[r] + count[r];
        }
        double t = time;
        const double tp = wtime();
        B.predict_send(&t, &nseg, addr0.data(), count.data());
        t_pred += wtime() - tp;
        double prm[6] = {P.eta_r, P.smax, P.dtmin, std::max(25.0 / tcr, 0.0), (double)P.nnbopt,
                         (double)P.mlp_mode};
        std::vector<int> &pend = r_pend, &again = r_again, &addr = r_addr;
        std::vector<double> &rsv = r_rs;
        pend.resize(ni);
        for (size_t q = 0; q < ni; ++q) pend[q] = (int)q;
        while (!pend.empty()) {
            const int np = (int)pend.size();
            grow(b_iseg, np);
            grow(b_h2, np);
            grow(b_dtr, np);
            grow(b_xi, 3 * (size_t)np);
            grow(b_vi, 3 * (size_t)np);
            grow(rrow, 32 * (size_t)np);
            grow(addr, np);
            grow(rsv, np);
            for (int p = 0; p < np; ++p) {
                const int q = pend[p], i = idx[q];
                addr[p] = i + 1;
                b_iseg[p] = seg_of_q[q];
                b_h2[p] = h2_of(i, 1.0 / cnt[cl_of[i]]);
                b_dtr[p] = stepr[i];
                rsv[p] = rs[i];
                // t0 = time: the body is at x0, v0
                const double *px = xv ? xv + 6 * (size_t)q : &x0[3 * (size_t)i];
                const double *pv = xv ? xv + 6 * (size_t)q + 3 : &v0[3 * (size_t)i];
                for (int c = 0; c < 3; ++c) {
                    b_xi[3 * (size_t)p + c] = px[c];
                    b_vi[3 * (size_t)p + c] = pv[c];
                }
            }
            int nni = np, lmax = P.lmax, nnbmax = P.nnbmax, mf = P.m_flag;
            const double tc = wtime();
            B.regf_correct(&t, &nni, addr.data(), b_iseg.data(), &nseg, seg_j0.data(), addr0.data(), b_h2.data(),
                           b_dtr.data(), rsv.data(), (double(*)[3])b_xi.data(), (double(*)[3])b_vi.data(), &lmax,
                           &nnbmax, &mf, prm, rrow.data());
            t_rcall += wtime() - tc;
            st.reg_calls++;
            again.clear();
            for (int p = 0; p < np; ++p) {
                const int q = pend[p], i = idx[q];
                st.reg_pairs += cnt[cl_of[i]];
                const double *o = &rrow[32 * (size_t)p];
                if (o[28] != 0.0) {
                    shrink_radius(i, (int)o[28]);
                    again.push_back(q);
                    continue;
                }
                step[i] = o[24];
                stepr[i] = o[25];
                rs[i] = o[26];
                t0r[i] = time;
                const int nnb = (int)o[27];
                if (nnb > 0) rsmin_seen(i);
                st.nb_sum += nnb;
                st.nb_absdev += fabs((double)(nnb - P.nnbopt));
                st.reg_steps++;
                if (o[29] == 1.0) st.mlp_used++;
                if (o[29] == 2.0) st.mlp_fallback++;
            }
            if (!again.empty()) st.overflow_retries++;
            pend.swap(again);
        }
        st.wall_reg += wtime() - t_0;
    }

    // Regular force and new lists (global 1-based, self removed) of the
    // bodies in idx (ascending, so grouped by cluster) at `time`.
    void regular_forces(const std::vector<int> &idx, std::vector<double> &freg, std::vector<double> &fdr,
                        std::vector<int> &nlist) {
        const double t_0 = wtime();
        const size_t ni = idx.size();
        freg.resize(3 * ni);
        fdr.resize(3 * ni);
        // grow only (a shrink then grow would zero the whole buffer again);
        // take_row writes each row's ids and a zero pad
        if (nlist.size() < ni * (size_t)LS) nlist.resize(ni * (size_t)LS);
        prop.assign(ni, 0.0);
        // runs of idx per cluster
        std::vector<int> run0, runc;
        for (size_t q = 0; q < ni; ++q)
            if (q == 0 || cl_of[idx[q]] != cl_of[idx[q - 1]]) {
                run0.push_back((int)q);
                runc.push_back(cl_of[idx[q]]);
            }
        run0.push_back((int)ni);
        const int nrun = (int)runc.size();
        if (batched && B.regf_seg && B.predict_send && (nrun > 1 || P.seg_single)) {
            regular_batched(idx, run0, runc, nrun, freg, fdr, nlist);
        } else if (batched && B.predict_send && nrun == 1) {
            // one cluster: its j set predicted on the device, then the
            // reference-ABI calls (the packed tile kernel, tuned per N_active)
            const int c = runc[0];
            double t = time;
            int nseg = 1, a0 = base[c] + 1, cntc = cnt[c];
            B.predict_send(&t, &nseg, &a0, &cntc);
            regular_one_cluster(idx, run0[0], run0[1], c, freg, fdr, nlist, true);
        } else {
            for (int r = 0; r < nrun; ++r) regular_one_cluster(idx, run0[r], run0[r + 1], runc[r], freg, fdr, nlist);
        }
        st.wall_reg += wtime() - t_0;
    }

    // Copy one result row into the global list layout.
    void take_row(int i, int c, const int *src, const double *acc, const double *jrk, size_t q,
                  std::vector<double> &freg, std::vector<double> &fdr, std::vector<int> &nlist) {
        for (int k = 0; k < 3; ++k) {
            freg[3 * q + k] = acc[k];
            fdr[3 * q + k] = jrk[k];
        }
        const int nb = src[0];
        int *out = &nlist[q * (size_t)LS];
        int l1 = 0;
        const int self = i - base[c];
        for (int l = 1; l <= nb; ++l) {
            const int j = src[l];
            if (j != self) out[1 + l1++] = base[c] + j + 1;
        }
        out[0] = l1;
        for (int k = l1 + 1; k < std::min(LS, l1 + 9); ++k) out[k] = 0;
    }

    void regular_batched(const std::vector<int> &idx, const std::vector<int> &run0,
                         const std::vector<int> &runc, int nrun, std::vector<double> &freg,
                         std::vector<double> &fdr, std::vector<int> &nlist) {
        // the bodies corrected in this block must be on the device first
        // (their t0 is the block time, so they predict to themselves)
        std::vector<int> addr0(nrun), count(nrun), seg_j0(nrun + 1, 0);
        for (int r = 0; r < nrun; ++r) {
            addr0[r] = base[runc[r]] + 1;
            count[r] = cnt[runc[r]];
            seg_j0[r + 1] = seg_j0[r] + count[r];
        }
        double t = time;
        int nseg = nrun;
        B.predict_send(&t, &nseg, addr0.data(), count.data());
        // pending rows: first all, then the overflowed ones after a shrink
        std::vector<int> pend(idx.size());
        for (size_t q = 0; q < idx.size(); ++q) pend[q] = (int)q;
        std::vector<int> seg_of_q(idx.size());
        for (int r = 0; r < nrun; ++r)
            for (int q = run0[r]; q < run0[r + 1]; ++q) seg_of_q[q] = r;
        while (!pend.empty()) {
            const int np = (int)pend.size();
            auto grow = [](auto &v, size_t k) {
                if (v.size() < k) v.resize(k);
            };
            grow(b_iseg, np);
            grow(b_h2, np);
            grow(b_dtr, np);
            grow(b_xi, 3 * (size_t)np);
            grow(b_vi, 3 * (size_t)np);
            grow(b_acc, 3 * (size_t)np);
            grow(b_jrk, 3 * (size_t)np);
            grow(b_pot, np);
            grow(b_prop, np);
            grow(b_lst, (size_t)np * P.lmax);
            int *iseg = b_iseg.data(), *lst = b_lst.data();
            double *h2 = b_h2.data(), *dtr = b_dtr.data(), *xi = b_xi.data(), *vi = b_vi.data(),
                   *acc = b_acc.data(), *jrk = b_jrk.data(), *pot = b_pot.data(), *pr = b_prop.data();
            for (int p = 0; p < np; ++p) {
                const int q = pend[p], i = idx[q], c = cl_of[i];
                iseg[p] = seg_of_q[q];
                h2[p] = h2_of(i, 1.0 / cnt[c]);
                dtr[p] = stepr[i];
                pred_at(i, time, &xi[3 * (size_t)p], &vi[3 * (size_t)p]);
            }
            int nni = np, lmax = P.lmax, nnbmax = P.nnbmax, mf = P.m_flag;
            B.regf_seg(&nni, iseg, h2, dtr, (double(*)[3])xi, (double(*)[3])vi, (double(*)[3])acc,
                       (double(*)[3])jrk, pot, &lmax, &nnbmax, lst, &mf, &nseg, seg_j0.data());
            st.reg_calls++;
            if (P.mlp_mode == 2) B.proposals(&nni, pr);
            std::vector<int> again;
            for (int p = 0; p < np; ++p) {
                prop[pend[p]] = P.mlp_mode == 2 ? pr[p] : 0.0;
                const int q = pend[p], i = idx[q], c = cl_of[i];
                st.reg_pairs += cnt[c];
                const int *src = &lst[(size_t)p * P.lmax];
                if (src[0] < 0) {
                    shrink_radius(i, src[0]);
                    again.push_back(q);
                    continue;
                }
                take_row(i, c, src, acc + 3 * (size_t)p, jrk + 3 * (size_t)p, (size_t)q, freg, fdr, nlist);
            }
            if (!again.empty()) st.overflow_retries++;
            pend.swap(again);
        }
    }

    // One cluster as the single-cluster driver does it: host prediction of
    // its bodies, gpunb_send_, gpunb_regf_ in chunks with overflow retry.
    // With sent = true the cluster's j set is already on the device and only
    // the active bodies are predicted on the host.
    void regular_one_cluster(const std::vector<int> &idx, int q0, int q1, int c, std::vector<double> &freg,
                             std::vector<double> &fdr, std::vector<int> &nlist, bool sent = false) {
        const int nc = cnt[c], b = base[c];
        std::vector<double> xp, vp;
        if (!sent) {
            xp.resize(3 * (size_t)nc);
            vp.resize(3 * (size_t)nc);
            for (int j = 0; j < nc; ++j) pred_at(b + j, time, &xp[3 * (size_t)j], &vp[3 * (size_t)j]);
            int nn = nc;
            B.gpunb_send(&nn, &m[b], (double(*)[3])xp.data(), (double(*)[3])vp.data());
        }
        auto fill = [&](int i, double *xi, double *vi) {
            if (sent) {
                pred_at(i, time, xi, vi);
                return;
            }
            for (int k = 0; k < 3; ++k) {
                xi[k] = xp[3 * (size_t)(i - b) + k];
                vi[k] = vp[3 * (size_t)(i - b) + k];
            }
        };
        auto take = [&](int q, int i, const int *row, const double *acc, const double *jrk) {
            take_row(i, c, row, acc, jrk, (size_t)q, freg, fdr, nlist);
        };
        regf_rows(B, idx, q0, q1, nc, 1.0 / nc, fill, take, prop);
    }

    bool init() {
        alloc();
        cl_of.assign(n, 0);
        for (int c = 0; c < ncl; ++c)
            for (int k = 0; k < cnt[c]; ++k) cl_of[base[c] + k] = c;
        adjust_init(ncl);
        acl = cl_of;
        for (int i = 0; i < n; ++i) init_radius(i, &x0[3 * (size_t)i]);
        int nb = n + 10, rank = 0;
        B.gpunb_open(&nb, &rank);
        int nmax = n, lmax = P.lmax;
        B.irr_open(&nmax, &lmax, &rank);
        time = 0.0;
        // F = FDOT = 0 at t = 0: the records predict to themselves
        for (int i = 0; i < n; ++i) set_jp(i);
        std::vector<int> all(n);
        for (int i = 0; i < n; ++i) all[i] = i;
        std::vector<double> freg, fdr;
        std::vector<int> nl;
        fpoly0 = true;
        regular_forces(all, freg, fdr, nl);
        fpoly0 = false;
        for (int i = 0; i < n; ++i) {
            const int *src = &nl[(size_t)i * LS];
            memcpy(row(i), src, sizeof(int) * std::min(LS, src[0] + 1));  // rows start zeroed
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
        if (dev_corr()) {
            double eta = P.eta_i, smax = P.smax, dtmin = P.dtmin;
            B.hermite_open(&eta, &smax, &dtmin);
            for (int i = 0; i < n; ++i) set_hermite(i);
        }
        return true;
    }

    // Kinetic and potential energy of cluster c at `time`; xp, vp receive
    // its bodies at `time`.
    void energy(int c, double &ekin, double &epot, std::vector<double> &xp, std::vector<double> &vp) {
        const int nc = cnt[c], b = base[c];
        xp.resize(3 * (size_t)nc);
        vp.resize(3 * (size_t)nc);
        std::vector<double> phi(nc + 8);
        for (int j = 0; j < nc; ++j) pred(b + j, time, &xp[3 * (size_t)j], &vp[3 * (size_t)j]);
        int rank = 0, istart = 1, ni = nc, nn = nc;
        B.gpupot(&rank, &istart, &ni, &nn, &m[b], (double(*)[3])xp.data(), phi.data());
        ekin = 0;
        epot = 0;
        for (int j = 0; j < nc; ++j) {
            const double *v = &vp[3 * (size_t)j];
            ekin += 0.5 * m[b + j] * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            epot -= 0.5 * m[b + j] * phi[j];
        }
    }

    // Energy output of every cluster, and the radius rule's quantities of
    // each (Bodies::adjust) from the same bodies at `time`; with the
    // regular corrector on the device the neighbour rows are read back for
    // it first, and the new quantities go to the device.
    void record(double *tout, double *eout, int &nout, int nout_max) {
        std::vector<double> xp, vp;
        const bool adj = adjust_due(time);
        for (int c = 0; c < ncl; ++c) {
            double ek, ep;
            energy(c, ek, ep, xp, vp);
            if (adj) adjust(c, base[c], cnt[c], xp.data(), vp.data(), ek, -ep, rows_for(c), time);
            if (nout < nout_max) {
                double *e = eout + ((size_t)nout * ncl + c) * 3;
                e[0] = ek;
                e[1] = ep;
                e[2] = ek + ep;
            }
        }
        if (adj && dev_reg() && B.hermite_adjust) push_adjust();
        if (nout < nout_max) tout[nout++] = time;
    }

    // The neighbour rows core.f reads for cluster c: the host's lists, or,
    // once the device regular corrector keeps them, the rows of the central
    // bodies read back from the device.
    std::vector<int> core_rows, core_addr;
    std::function<void(const std::vector<int> &, std::vector<const int *> &)> rows_for(int c) {
        return [this, c](const std::vector<int> &jl, std::vector<const int *> &rp) {
            const int b = base[c];
            if (!(dev_reg() && B.lists_get && time > 0.0)) {   // at TIME = 0 the host's rows are current
                for (size_t l = 0; l < jl.size(); ++l) rp[l] = row(b + jl[l]);
                return;
            }
            const int k = (int)jl.size();
            core_addr.resize(std::max(k, 1));
            core_rows.resize((size_t)std::max(k, 1) * LS);
            for (int l = 0; l < k; ++l) core_addr[l] = b + jl[l] + 1;
            int nn = k, ls = LS;
            if (k) B.lists_get(&nn, core_addr.data(), &ls, core_rows.data());
            for (int l = 0; l < k; ++l) rp[l] = &core_rows[(size_t)l * LS];
        };
    }

    // The radius rule's quantities of every cluster to the device corrector.
    void push_adjust() {
        std::vector<int> a0(ncl + 1);
        std::vector<double> par(8 * (size_t)ncl, 0.0);
        for (int c = 0; c < ncl; ++c) {
            a0[c] = base[c] + 1;
            const ACPar &a = acp[c];
            double *q = &par[8 * (size_t)c];
            q[0] = a.rdens[0];
            q[1] = a.rdens[1];
            q[2] = a.rdens[2];
            q[3] = a.rscale;
            q[4] = a.rc2;
            q[5] = a.rsfac;
            q[6] = a.bodym;
        }
        a0[ncl] = n + 1;
        int nbf = P.nb_flag, nc = ncl;
        B.hermite_adjust(&nbf, &nc, a0.data(), par.data());
    }

    // block clock on the device too
    bool dev_clock() const { return dev_reg() && P.dev_corrector >= 3 && B.blocks_run && B.blocks_regular; }

    // The block loop with the device's block clock: runs of irregular blocks
    // on the device (nb6_blocks_run_) until a block has bodies due a regular
    // step or the next output time is reached; the host runs those regular
    // steps (regular_on_device) and the energy output.  Same arithmetic and
    // order as run()'s host clock, so the same trajectory.
    void run_device_clock(double *tout, double *eout, int nout_max) {
        const double tw = wtime();
        int nout = 0;
        record(tout, eout, nout, nout_max);
        double tnext_out = P.dt_out;
        std::vector<int> act, reg;
        std::vector<double> rows;
        double t_reg = 0;
        bool step_past = false;  // run one block past the output time (see below)
        for (;;) {
            double tlimit = step_past ? P.tcrit : std::min(tnext_out, P.tcrit);
            const long long left = P.max_blocks - st.blocks;
            if (left <= 0) break;
            int maxb = (int)std::min<long long>(step_past ? 1 : left, 1 << 30), reason = 0, nact = 0;
            step_past = false;
            long long nb = 0, nirr = 0;
            double tb = time;
            const double ti0 = wtime();
            B.blocks_run(&tlimit, &maxb, &reason, &nb, &nirr, &tb, &nact);
            st.wall_irr += wtime() - ti0;
            st.blocks += nb;
            st.irr_steps += nirr;
            if (nb > 0) time = tb;
            if (reason == 1) {
                // the block's bodies due a regular step, ascending, with
                // their corrected x0, v0 (the i of the regular call)
                const double w0 = wtime();
                if (act.size() < (size_t)std::max(nact, 1)) act.resize(std::max(nact, 1));
                if (rows.size() < 6 * (size_t)std::max(nact, 1)) rows.resize(6 * (size_t)std::max(nact, 1));
                int nr = 0;
                const double tq = wtime();
                B.blocks_regular(&nr, act.data(), rows.data());
                t_breg += wtime() - tq;
                reg.resize(nr);
                for (int q = 0; q < nr; ++q) reg[q] = act[q] - 1;
                regular_on_device(reg, rows.data());  // (the host copies of x0, v0 are refreshed at output)
                t_reg += wtime() - w0;
            }
            if (time >= tnext_out - 1e-15) {
                const double to = wtime();
                pull_state();
                record(tout, eout, nout, nout_max);
                tnext_out += P.dt_out;
                t_out += wtime() - to;
            }
            if (reason == 2 && tlimit >= P.tcrit) break;      // next block beyond the end
            // No block fell on the output time (steps that do not divide
            // it): the host clock records after the first block past it,
            // so run exactly that one block next.
            if (reason == 2 && time < tnext_out - 1e-15) {
                step_past = true;
                continue;
            }
            if (reason == 0 && P.max_blocks - st.blocks <= 0) break;  // block budget spent
        }
        pull_state();
        st.t_end = time;
        st.nout = nout;
        st.wall_total = wtime() - tw;
        if (getenv("NB6_VERBOSE")) {
            fprintf(stderr,
                    "# nb6 ensemble (device clock): wall %.3f s = block runs %.3f + regular part %.3f (j-set "
                    "prediction %.3f, regular calls %.3f, due list %.3f) + output %.3f + other\n",
                    st.wall_total, st.wall_irr, t_reg, t_pred, t_rcall, t_breg, t_out);
            int rank = 0;
            if (B.reg_profile) B.reg_profile(&rank);
            if (B.irr_profile) B.irr_profile(&rank);
        }
    }

    void run(double *tout, double *eout, int nout_max) {
        if (dev_clock()) {
            run_device_clock(tout, eout, nout_max);
            return;
        }
        const double tw = wtime();
        int nout = 0;
        record(tout, eout, nout, nout_max);
        double tnext_out = P.dt_out;
        std::vector<int> active, reg, addr, nnbid;
        std::vector<double> a, jd, freg, fdr;
        std::vector<int> nl;
        clock_reset();
        double t_clock = 0, t_icor = 0, t_rcor = 0, t_jp = 0;
        while (st.blocks < P.max_blocks) {
            double w0 = wtime();
            const double tmin = clock_next(active);
            t_clock += wtime() - w0;
            if (tmin > P.tcrit + 1e-12) break;
            time = tmin;
            st.blocks++;
            const int na = (int)active.size();
            addr.resize(na);
            for (int q = 0; q < na; ++q) addr[q] = active[q] + 1;
            a.assign(3 * (size_t)na, 0.0);
            jd.assign(3 * (size_t)na, 0.0);
            nnbid.assign(na, 0);
            const double ti0 = wtime();
            double t = time;
            int nna = na;
            const bool dc = dev_corr(), dr = dc && dev_reg();
            reg.clear();
            if (dc) {
                // force + corrector + new step on the device; the host
                // takes back the corrected state (with the regular corrector
                // on the device too: the step, and x0, v0 of the bodies due
                // a regular step, which the regular call takes as its i)
                crow.resize(24 * (size_t)na);
                B.irr_correct(&t, &nna, addr.data(), crow.data());
                st.wall_irr += wtime() - ti0;
                w0 = wtime();
                for (int q = 0; q < na && dr; ++q) {
                    const int i = active[q];
                    const double *o = &crow[24 * (size_t)q];
                    step[i] = o[18];
                    t0[i] = time;
                    st.irr_steps++;
                    if (o[19] != 0.0) {
                        reg.push_back(i);
                        for (int c = 0; c < 3; ++c) {
                            x0[3 * (size_t)i + c] = o[c];
                            v0[3 * (size_t)i + c] = o[3 + c];
                        }
                    }
                }
                for (int q = 0; q < na && !dr; ++q) {
                    const int i = active[q];
                    const double *o = &crow[24 * (size_t)q];
                    for (int c = 0; c < 3; ++c) {
                        const size_t k = 3 * (size_t)i + c;
                        x0[k] = o[c];
                        v0[k] = o[3 + c];
                        fi[k] = o[6 + c];
                        fidot[k] = o[9 + c];
                        f[k] = o[12 + c];
                        fdot[k] = o[15 + c];
                    }
                    step[i] = o[18];
                    t0[i] = time;
                    st.irr_steps++;
                    if (o[19] != 0.0) reg.push_back(i);
                }
                t_icor += wtime() - w0;
            } else {
                B.irr_firr_vec(&t, &nna, addr.data(), (double(*)[3])a.data(), (double(*)[3])jd.data(),
                               nnbid.data());
                st.wall_irr += wtime() - ti0;
                w0 = wtime();
                for (int q = 0; q < na; ++q)
                    if (irr_correct(active[q], time, &a[3 * (size_t)q], &jd[3 * (size_t)q])) reg.push_back(active[q]);
                t_icor += wtime() - w0;
            }
            if (!reg.empty() && dr) {
                regular_on_device(reg);
            } else if (!reg.empty()) {
                // corrected states of this block to the device before the
                // j set is predicted there (already there when the device
                // ran the corrector)
                if (batched && B.predict_send && !dc)
                    for (int q = 0; q < na; ++q) set_jp(active[q]);
                regular_forces(reg, freg, fdr, nl);
                w0 = wtime();
                snapshot(reg, time);
                for (size_t q = 0; q < reg.size(); ++q) {
                    const int i = reg[q];
                    const int *row_new = &nl[q * (size_t)LS];
                    const double rs_used = rs[i];
                    if (P.mlp_mode == 1)
                        learn_log(i, row_new[0], rs_used, h2_of(i, 1.0 / cnt[cl_of[i]]), &freg[3 * q], stepr[i]);
                    reg_correct(i, time, row_new, &freg[3 * q], &fdr[3 * q]);
                    if (P.mlp_mode == 2) learn_apply(i, row_new[0], rs_used, prop[q]);
                    set_list(i);
                }
                release_snapshot(reg);
                t_rcor += wtime() - w0;
            }
            w0 = wtime();
            if (dr) {
                // nothing changed on the host alone
            } else if (dc) {
                // only the regular corrector changed state on the host
                for (int i : reg) {
                    set_jp(i);
                    set_hermite(i);
                }
            } else {
                for (int q = 0; q < na; ++q) set_jp(active[q]);
            }
            t_jp += wtime() - w0;
            w0 = wtime();
            clock_push(active);
            t_clock += wtime() - w0;
            if (time >= tnext_out - 1e-15) {
                if (dr) pull_state();
                record(tout, eout, nout, nout_max);
                tnext_out += P.dt_out;
            }
        }
        if (dev_corr() && dev_reg()) pull_state();
        st.t_end = time;
        st.nout = nout;
        st.wall_total = wtime() - tw;
        if (getenv("NB6_VERBOSE")) {
            fprintf(stderr,
                    "# nb6 ensemble: wall %.3f s = irr calls %.3f + reg calls %.3f + irr corrector %.3f"
                    " + reg corrector %.3f + set_jp %.3f + clock %.3f + other (j-set prediction %.3f of reg calls)\n",
                    st.wall_total, st.wall_irr, st.wall_reg, t_icor, t_rcor, t_jp, t_clock, t_pred);
            int rank = 0;
            if (B.reg_profile) B.reg_profile(&rank);
            if (B.irr_profile) B.irr_profile(&rank);
        }
    }
};

}  // namespace

extern "C" {

// Integrate ncl independent clusters (counts[c] bodies each, stored back to
// back in mass[], x[][3], v[][3], each in its own Henon units) to p->tcrit.
// batched = 1 issues every force kind once per block for all clusters when
// the backend has the batched calls; 0 issues the regular force per cluster.
// x and v are overwritten with the final state predicted to the end time;
// tout[k] and eout[k][c][3] = (kinetic, potential, total) of cluster c at
// every p->dt_out.  Returns 0 on success.
int nb6drive_ensemble(const char *reg_lib, const char *irr_lib, const char *pot_lib, int ncl,
                      const int *counts, const double *mass, double *x, double *v,
                      const nb6drive_params *p, int batched, double *tout, double *eout, int nout_max,
                      nb6drive_stats *stats) {
    Ensemble e;
    e.P = *p;
    e.ncl = ncl;
    e.batched = batched != 0;
    if (ncl <= 0) return 3;
    e.base.assign(ncl, 0);
    e.cnt.assign(counts, counts + ncl);
    long long total = 0;
    for (int c = 0; c < ncl; ++c) {
        if (counts[c] < 2) return 3;
        e.base[c] = (int)total;
        total += counts[c];
    }
    if (total > (1LL << 30)) return 3;
    e.n = (int)total;
    if (!load_backend(e.B, reg_lib, irr_lib, pot_lib)) return 1;
    if (e.P.mlp_mode == 2 && !e.B.proposals) {
        fprintf(stderr, "nb6drive: mlp_mode 2 needs a backend with nb6_regf_proposals_\n");
        return 4;
    }
    e.m.assign(mass, mass + e.n);
    e.x0.assign(x, x + 3 * (size_t)e.n);
    e.v0.assign(v, v + 3 * (size_t)e.n);
    if (!e.init()) return 2;
    e.run(tout, eout, nout_max);
    for (int j = 0; j < e.n; ++j) e.pred(j, e.time, &x[3 * (size_t)j], &v[3 * (size_t)j]);
    int rank = 0;
    e.B.irr_close(&rank);
    e.B.gpunb_close();
    if (stats) *stats = e.st;
    return 0;
}

}  // extern "C"
