// chem_tables.h -- host-side compaction of the Chemkin tables of scfd_chem
// (the module arrays of store/therm_lib/chemkin/core/mod_chem.raw.f90, 0-based)
// into the flat device tables of DevChem, shared by the flow solver and the
// batched reactors.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <type_traits>
#include <vector>

#include "scfd_internal.h"

namespace scfd {

struct ChemTables {
    std::vector<double> coeff, tc, inv, mw, men, abe, cabe, troe, trange, trans, wc1, wc2;
    std::vector<int> rs, ind, num, snu, ex, nm, im, tr, nsec;
    std::vector<int> pp, pe, mp, me, mref, np_, ne_, dref;  // RateLists
    int ns = 0, nr = 0, nt = 0;
    double rtol = 0.0, atol = 0.0;

    ChemTables() = default;
    explicit ChemTables(const scfd_chem& h) : ns(h.ns), nr(h.nr), nt(h.nt), rtol(h.rtol), atol(h.atol) {
        for (int k = 0; k < ns; ++k) {
            for (int s = 0; s < 2; ++s)
                for (int i = 0; i < 7; ++i) coeff.push_back(h.coeff[k][s][i]);
            tc.push_back(h.tthre[k][2]);
            inv.push_back(1.0 / h.mws[k]);
            mw.push_back(h.mws[k]);
        }
        for (int i = 0; i < nr; ++i) {
            rs.push_back(h.rstate[i][0]);
            rs.push_back(h.rstate[i][1]);
            for (int s = 0; s < 2; ++s)
                for (int k = 0; k < 3; ++k) ind.push_back(h.indnu[i][s][k]);
            num.push_back(h.numnu[i][0]);
            num.push_back(h.numnu[i][1]);
            snu.push_back(h.snu[i]);
            ex.push_back(h.exist_m[i]);
            nm.push_back(h.numm[i]);
            for (int k = 0; k < ns; ++k) {
                im.push_back(h.indm[i][k]);
                men.push_back(h.men[i][k]);
            }
            for (int k = 0; k < 3; ++k) {
                abe.push_back(h.abe[i][k]);
                cabe.push_back(h.cabe[i][k]);
            }
            for (int k = 0; k < 4; ++k) troe.push_back(h.troe[i][k]);
        }
        for (int i = 0; i < nt; ++i) {
            tr.push_back(h.tr2th[i]);
            nsec.push_back(h.num_sctn_trans[i]);
            for (int l = 0; l < 5; ++l) {
                for (int m = 0; m < 2; ++m) trange.push_back(h.trange_trans[i][l][m]);
                for (int m = 0; m < 4; ++m) trans.push_back(h.trans[i][l][m]);
            }
        }
        rate_lists(h);
        // Wilke mixing-rule constants per species pair
        for (int i = 0; i < nt; ++i)
            for (int j = 0; j < nt; ++j) {
                const double mi = h.mws[h.tr2th[i]], mj = h.mws[h.tr2th[j]];
                wc1.push_back(std::pow(mj / mi, 0.25));
                wc2.push_back(std::sqrt(2.0 * mj / (mi + mj)));
            }
    }

    // RateLists of scfd_internal.h: per-species contribution lists in the
    // reference's accumulation order (Fex_var FJ.f90:301-453, Fex / Jex 152-709)
    void rate_lists(const scfd_chem& h) {
        pp.assign(ns + 1, 0);
        mp.assign(ns + 1, 0);
        np_.assign(ns + 1, 0);
        mref.assign(nr > 0 ? nr : 1, -1);
        dref.assign(nr > 0 ? nr : 1, -1);
        std::vector<std::vector<int>> pl(ns), ml(ns), nl(ns);
        int last = -1, lastd = -1;
        for (int i = 0; i < nr; ++i) {
            if (h.exist_m[i]) last = i;
            mref[i] = last;
            const int rs0 = h.rstate[i][0], rs1 = h.rstate[i][1];
            if (rs1 >= 4 || (rs0 == 0 && (rs1 == 2 || rs1 == 3))) lastd = i;
            dref[i] = lastd;
            for (int k = 0; k < h.numnu[i][0]; ++k) nl[h.indnu[i][0][k]].push_back(2 * i + 1);
            for (int k = 0; k < h.numnu[i][1]; ++k) nl[h.indnu[i][1][k]].push_back(2 * i);
            const int nreac = h.numnu[i][0], nprod = h.numnu[i][1];
            for (int k = 0; k < nreac; ++k) ml[h.indnu[i][0][k]].push_back(2 * i);
            for (int k = 0; k < nprod; ++k) pl[h.indnu[i][1][k]].push_back(2 * i);
            if (h.rstate[i][0] == 0) {
                for (int k = 0; k < nreac; ++k) pl[h.indnu[i][0][k]].push_back(2 * i + 1);
                for (int k = 0; k < nprod; ++k) ml[h.indnu[i][1][k]].push_back(2 * i + 1);
            }
        }
        for (int j = 0; j < ns; ++j) {
            pe.insert(pe.end(), pl[j].begin(), pl[j].end());
            me.insert(me.end(), ml[j].begin(), ml[j].end());
            ne_.insert(ne_.end(), nl[j].begin(), nl[j].end());
            pp[j + 1] = (int)pe.size();
            mp[j + 1] = (int)me.size();
            np_[j + 1] = (int)ne_.size();
        }
    }

    template <typename T>
    static size_t slot(const std::vector<T>& a) {
        return ((a.empty() ? 1 : a.size()) * sizeof(T) + 255) & ~(size_t)255;
    }
    // device bytes when every table starts on a 256-byte boundary
    size_t bytes() const {
        size_t b = 0;
        for (const auto* a : {&coeff, &tc, &inv, &mw, &men, &abe, &cabe, &troe, &trange, &trans, &wc1, &wc2})
            b += slot(*a);
        for (const auto* a : {&rs, &ind, &num, &snu, &ex, &nm, &im, &tr, &nsec, &pp, &pe, &mp, &me, &mref, &np_, &ne_,
                              &dref})
            b += slot(*a);
        return b;
    }
    // Copies the tables to the device memory at p (advanced past them) on
    // stream s and points ch at them; the host vectors must outlive the copies.
    cudaError_t upload(DevChem& ch, char*& p, cudaStream_t s) const {
        cudaError_t err = cudaSuccess;
        auto put = [&](const auto& a) {
            using T = typename std::decay_t<decltype(a)>::value_type;
            T* d = reinterpret_cast<T*>(p);
            if (!a.empty() && err == cudaSuccess)
                err = cudaMemcpyAsync(d, a.data(), a.size() * sizeof(T), cudaMemcpyHostToDevice, s);
            p += slot(a);
            return d;
        };
        ch.ns = ns;
        ch.nr = nr;
        ch.nt = nt;
        ch.coeff = put(coeff);
        ch.tcommon = put(tc);
        ch.inv_mw = put(inv);
        ch.mws = put(mw);
        ch.rstate = put(rs);
        ch.indnu = put(ind);
        ch.numnu = put(num);
        ch.snu = put(snu);
        ch.exist_m = put(ex);
        ch.numm = put(nm);
        ch.indm = put(im);
        ch.men = put(men);
        ch.abe = put(abe);
        ch.cabe = put(cabe);
        ch.troe = put(troe);
        ch.tr2th = put(tr);
        ch.nsec = put(nsec);
        ch.trange = put(trange);
        ch.trans = put(trans);
        ch.wc1 = put(wc1);
        ch.wc2 = put(wc2);
        ch.rl.p_ptr = put(pp);
        ch.rl.p_ent = put(pe);
        ch.rl.m_ptr = put(mp);
        ch.rl.m_ent = put(me);
        ch.rl.mref = put(mref);
        ch.rl.n_ptr = put(np_);
        ch.rl.n_ent = put(ne_);
        ch.rl.dref = put(dref);
        ch.rtol = rtol;
        ch.atol = atol;
        return err;
    }
};

}  // namespace scfd
