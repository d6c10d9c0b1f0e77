// Thermal solve with metals, one leaf per lane, the metal rate cache in
// shared memory (included by balance.cu inside its namespace; uses its
// argument types and H/He helpers).
//
// The per-leaf work of gas_thermal_update with metals (thermal_mod.f90:
// 124-249 with the bracketed solves) is dominated by the stage-chain sums of
// species_metal_sums (species_mod.f90:566-614), many per trial temperature,
// each reading the (leaf, T) rate cache of species_ne_prepare (:517-536).
// Three choices make that cheap on a GPU:
//
// * the cache lives in shared memory, [slot][thread], sized to the
//   transitions actually present: a transition without charge exchange keeps
//   2 slots (gamma / alpha and C_ci / alpha, the ratio n_{i+1}/n_i being
//   gamma/(n_e alpha) + C_ci/alpha), one with charge exchange keeps gamma,
//   C_ci, alpha and its CX coefficients (3 + 1..2 slots);
// * an element's stage fractions come from one division: with n_t the
//   ionising and d_t = max(recombining, tiny) rate of transition t,
//   f_i = (prod_{t<i} n_t)(prod_{t>=i} d_t) / sum_j (same), which is
//   r_t = n_t / d_t, f_1 = 1/(1 + r_1 + r_1 r_2 + ...) rearranged (the ratio
//   form is kept for the case the products leave the double range);
// * the root searches are flat per-lane state machines: within one trial
//   temperature every lane makes one cascade sum per trip, whatever root
//   (n_e or the H fraction) it is in, so a lane's sums are not held back by
//   the other lanes' nested iterations; the trial temperatures stay in
//   lockstep (every lane prepares its cache and evaluates its net rate
//   together), and a lane whose leaf is solved writes it and claims the next
//   leaf of the work order from a global counter at once.
// Each lane's sequence of trial points and root iterates is that of
// thermal_bracketed / solve_cell_fast / hydrogen_neutral_fraction_warm; only
// the rounding of the chain arithmetic differs.

// Slots of one transition: kind bit 0 = CX recombination, bit 1 = CX
// ionisation.  Kind 0: P = gamma/alpha, Q = C_ci/alpha.  Otherwise gamma,
// C_ci, alpha, [cxi], [cxr].
__host__ __device__ __forceinline__ int lane_slots(int kind) { return kind == 0 ? 2 : 3 + (kind & 1) + ((kind >> 1) & 1); }

struct LaneLayout {
    unsigned char kind[kMaxTr];
    unsigned short off[kMaxTr];
    int nslot;
};

__host__ __device__ __forceinline__ int lane_kind(const MetalTr& t) { return (t.cxr_form > 0 ? 1 : 0) | (t.cxi_form > 0 ? 2 : 0); }

// The layout of m's transitions, written by one thread.
__device__ void lane_layout_build(const MetalDev& m, LaneLayout& L) {
    int o = 0;
    for (int j = 0; j < m.ntr; ++j) {
        const int k = lane_kind(m.tr[j]);
        L.kind[j] = (unsigned char)k;
        L.off[j] = (unsigned short)o;
        o += lane_slots(k);
    }
    L.nslot = o;
}

// One lane's view of the shared cache: slot s of this lane at S[s * stride].
struct LaneCache {
    double* S;
    int stride;
    const LaneLayout* L;
    const MetalDev* m;
    const MetalEl* el;   // m's elements, copied here for the cascade sums
    int nel;
    __device__ __forceinline__ double& at(int s) const { return S[s * stride]; }
};

// The 4-point Lagrange stencil of T on the ln T nodes of the T tables
// (i0 < 0: T outside them, or no tables).
struct TNode {
    int i0;
    double w0, w1, w2, w3;
};
__device__ __forceinline__ TNode t_node(const MetalDev& m, double T) {
    TNode n = {-1, 0.0, 0.0, 0.0, 0.0};
    if (m.tnt > 0) {
        const double s = (log(T) - m.tu0) / m.tdu;
        const int i = (int)floor(s);
        if (i >= 1 && i <= m.tnt - 3) {
            const double t = s - (double)i;
            n.w0 = -t * (t - 1.0) * (t - 2.0) / 6.0;
            n.w1 = (t + 1.0) * (t - 1.0) * (t - 2.0) / 2.0;
            n.w2 = -(t + 1.0) * t * (t - 2.0) / 2.0;
            n.w3 = (t + 1.0) * t * (t - 1.0) / 6.0;
            n.i0 = i - 1;
        }
    }
    return n;
}

// species_ne_prepare at T for leaf il (as metal_prepare: the T table inside
// its range, the clamped CX fits and any T outside it evaluated directly).
__device__ __noinline__ void lane_prepare(const LaneCache c, long long il, double T) {
    const MetalDev& m = *c.m;
    const TNode tn = t_node(m, T);
    const int i0 = tn.i0;
    const double w0 = tn.w0, w1 = tn.w1, w2 = tn.w2, w3 = tn.w3;
    for (int j = 0; j < m.ntr; ++j) {
        const MetalTr& r = m.tr[j];
        const double gam = m.egam[il * m.ntr + j];
        double ci, rec, cxi, cxr;
        if (i0 >= 0) {
            const double* Lt = m.ttab + (size_t)j * 4 * m.tnt + i0;
            ci = exp(w0 * Lt[0] + w1 * Lt[1] + w2 * Lt[2] + w3 * Lt[3]);
            Lt += m.tnt;
            rec = exp(w0 * Lt[0] + w1 * Lt[1] + w2 * Lt[2] + w3 * Lt[3]);
            Lt += m.tnt;
            cxi = r.cxi_form <= 0 ? 0.0 : r.cxi_form >= 6 ? metal_cx_rate(r.cxi_form, r.cxi, T)
                                                          : exp(w0 * Lt[0] + w1 * Lt[1] + w2 * Lt[2] + w3 * Lt[3]);
            Lt += m.tnt;
            cxr = r.cxr_form <= 0 ? 0.0 : r.cxr_form >= 6 ? metal_cx_rate(r.cxr_form, r.cxr, T)
                                                          : exp(w0 * Lt[0] + w1 * Lt[1] + w2 * Lt[2] + w3 * Lt[3]);
        } else {
            ci = metal_coef(r, 0, T);
            rec = metal_coef(r, 1, T);
            cxi = metal_coef(r, 2, T);
            cxr = metal_coef(r, 3, T);
        }
        const int k = c.L->kind[j], o = c.L->off[j];
        if (k == 0) {
            const double ra = fmax(rec, 1.0e-300);
            c.at(o) = gam / ra;
            c.at(o + 1) = ci / ra;
        } else {
            c.at(o) = gam;
            c.at(o + 1) = ci;
            c.at(o + 2) = rec;
            int q = o + 3;
            if (k & 2) c.at(q++) = cxi;
            if (k & 1) c.at(q) = cxr;
        }
    }
}

// The ionising (n) and recombining (d) rates of an element's transitions and
// their CX coefficients (0 where the transition has none).
__device__ __forceinline__ void lane_rates(const LaneCache& c, const MetalEl& e, double ne, double nHI, double nHII,
                                           double (&n)[kMaxSt - 1], double (&d)[kMaxSt - 1],
                                           double (&xi)[kMaxSt - 1], double (&xr)[kMaxSt - 1]) {
    const int nt = e.nstage - 1;
#pragma unroll
    for (int t = 0; t < kMaxSt - 1; ++t) {
        n[t] = 0.0;
        d[t] = 1.0;
        xi[t] = 0.0;
        xr[t] = 0.0;
        if (t < nt) {
            const int j = e.tr0 + t, k = c.L->kind[j], o = c.L->off[j];
            if (k == 0) {
                n[t] = c.at(o) + ne * c.at(o + 1);
                d[t] = ne;
            } else {
                double rion = c.at(o) + ne * c.at(o + 1);
                double rrec = ne * c.at(o + 2);
                int q = o + 3;
                if (k & 2) {
                    xi[t] = c.at(q++);
                    if (xi[t] > 0.0) rion = rion + nHII * xi[t];
                }
                if (k & 1) {
                    xr[t] = c.at(q);
                    if (xr[t] > 0.0) rrec = rrec + nHI * xr[t];
                }
                n[t] = rion;
                d[t] = fmax(rrec, kTinest);
            }
        }
    }
}

// Stage fractions f[0..nstage-1] of one element (metal_chain).
__device__ __forceinline__ void lane_fracs(int ns, const double (&n)[kMaxSt - 1], const double (&d)[kMaxSt - 1],
                                           double (&f)[kMaxSt]) {
    constexpr int E = kMaxSt - 1;
    const int nt = ns - 1;
    double sd[kMaxSt];
    sd[E] = 1.0;
    double acc = 1.0;
#pragma unroll
    for (int t = E - 1; t >= 0; --t) {
        if (t < nt) acc = acc * d[t];
        sd[t] = acc;
    }
    double pn = 1.0, num = sd[0];
    f[0] = sd[0];
#pragma unroll
    for (int i = 1; i < kMaxSt; ++i) {
        f[i] = 0.0;
        if (i <= nt) {
            pn = pn * n[i - 1];
            f[i] = pn * sd[i];
            num = num + f[i];
        }
    }
    if (num > 0.0 && num <= 1.0e300) {
        const double inv = 1.0 / num;
#pragma unroll
        for (int i = 0; i < kMaxSt; ++i) f[i] = f[i] * inv;
        return;
    }
    // the ratio form (metal_chain) where the products leave the double range
    double s = 1.0, prod = 1.0, r[kMaxSt - 1];
#pragma unroll
    for (int t = 0; t < E; ++t) {
        r[t] = t < nt ? n[t] / d[t] : 0.0;
        if (t < nt) {
            prod = prod * r[t];
            s = s + prod;
        }
    }
    f[0] = 1.0 / s;
#pragma unroll
    for (int i = 1; i < kMaxSt; ++i) f[i] = i <= nt ? f[i - 1] * r[i - 1] : 0.0;
}

// species_metal_sums: metal electrons and the two CX rates hydrogen sees,
// over the elements e0, e0 + estep, ...  The sums accumulate in registers
// and are stored once at the end (the outputs live in the caller's frame).
__device__ __noinline__ void lane_sums(const LaneCache c, double nH, double ne, double nHI, double nHII, double& nem_out,
                                       double& rin_out, double& rout_out, int e0 = 0, int estep = 1) {
    const int nel = c.nel;
    const MetalEl* __restrict__ els = c.el;
    double nem = 0.0, rin = 0.0, rout = 0.0;
    for (int ie = e0; ie < nel; ie += estep) {
        const MetalEl e = els[ie];
        double n[kMaxSt - 1], d[kMaxSt - 1], xi[kMaxSt - 1], xr[kMaxSt - 1], f[kMaxSt];
        lane_rates(c, e, ne, nHI, nHII, n, d, xi, xr);
        lane_fracs(e.nstage, n, d, f);
        const double nX = e.abund * nH;
        if (e.nstage > 1) rin = rin + xi[0] * nX * f[0];
#pragma unroll
        for (int i = 2; i <= kMaxSt; ++i)
            if (i <= e.nstage) {
                nem = nem + e.abund * nH * f[i - 1] * (double)(i - 1);
                rout = rout + xr[i - 2] * nX * f[i - 1];
                if (i < e.nstage) rin = rin + xi[i - 1] * nX * f[i - 1];
            }
    }
    nem_out = nem;
    rin_out = rin;
    rout_out = rout;
}

// The cascade sums of every lane with `need`, computed by the whole warp
// (every lane enters): with k such lanes, each is served by G = 8, 4, 2 or 1
// lanes (k <= 4, 8, 16, more), which split its elements (group lane s takes
// elements s, s + G, ...; the caches are in shared memory, so any lane can
// read them) and add their parts by shuffles within the group.  A search's
// tail, where a few lanes are still iterating, then runs on all 32 lanes.
__device__ __forceinline__ void warp_sums(const LaneCache& c, bool need, double nH, double ne, double nHI, double nHII,
                                          double& em, double& rin, double& rout) {
    const unsigned mask = __ballot_sync(kFull, need);
    const int k = __popc(mask);
    const int lane = threadIdx.x & 31;
    const int G = k <= 4 ? 8 : k <= 8 ? 4 : k <= 16 ? 2 : 1;
    if (G == 1) {
        if (need) lane_sums(c, nH, ne, nHI, nHII, em, rin, rout);
        return;
    }
    const int g = lane / G, sub = lane - g * G;
    int owner = lane;
    if (g < k) {   // the g-th lane of the mask
        unsigned m = mask;
        for (int t = 0; t < g; ++t) m &= m - 1u;
        owner = __ffs(m) - 1;
    }
    const double oH = __shfl_sync(kFull, nH, owner), oNe = __shfl_sync(kFull, ne, owner);
    const double oHI = __shfl_sync(kFull, nHI, owner), oHII = __shfl_sync(kFull, nHII, owner);
    double a = 0.0, b = 0.0, d = 0.0;
    if (g < k) {
        LaneCache co = c;
        co.S = c.S + (owner - lane);
        lane_sums(co, oH, oNe, oHI, oHII, a, b, d, sub, G);
    }
    for (int o = 1; o < G; o <<= 1) {
        a = a + __shfl_xor_sync(kFull, a, o);
        b = b + __shfl_xor_sync(kFull, b, o);
        d = d + __shfl_xor_sync(kFull, d, o);
    }
    const int src = need ? __popc(mask & ((1u << lane) - 1u)) * G : lane;
    const double ta = __shfl_sync(kFull, a, src), tb = __shfl_sync(kFull, b, src), td = __shfl_sync(kFull, d, src);
    if (need) {
        em = ta;
        rin = tb;
        rout = td;
    }
}

// The metal terms of net_rate (as metal_thermal) from the shared cache.
__device__ __noinline__ MetalThermalTerms lane_thermal(const LaneCache c, const ThermalDev& td, long long il, double T,
                                                      double nH, double ne, double nHI, double nHII) {
    const MetalDev& m = *c.m;
    const double A_CII = 2.321e-6, A_OI = 8.865e-5;
    MetalThermalTerms o = {0.0, 0.0, 0.0, 0.0};
    double g[4];
    for (int z = 1; z <= 4; ++z) g[z - 1] = gbar_ff(td.gff, T, z);
    const double rsT = 1.0 / sqrt(T);
    double ff = 0.0;
    const NlAt at = nl_at(td.tinv, T, ne);
    const TNode tn = m.ctab ? t_node(m, T) : TNode{-1, 0.0, 0.0, 0.0, 0.0};
    for (int ie = 0; ie < m.nel; ++ie) {
        const MetalEl e = m.el[ie];
        double n[kMaxSt - 1], d[kMaxSt - 1], xi[kMaxSt - 1], xr[kMaxSt - 1], frac[kMaxSt];
        lane_rates(c, e, ne, nHI, nHII, n, d, xi, xr);
        lane_fracs(e.nstage, n, d, frac);
        const double nel = e.abund * nH;
#pragma unroll
        for (int i = 1; i <= kMaxSt; ++i) {
            if (i > e.nstage) continue;
            const MetalStage& st = m.st[e.st0 + i - 1];
            if (!st.has_cool) continue;
            double fit = 0.0;
            if (tn.i0 >= 0) {   // the fit from its ln T table
                const double* Lt = m.ctab + (size_t)(e.st0 + i - 1) * m.tnt + tn.i0;
                fit = exp(tn.w0 * Lt[0] + tn.w1 * Lt[1] + tn.w2 * Lt[2] + tn.w3 * Lt[3]);
            } else {
                for (int q = 0; q < st.nterm; ++q) fit = fit + st.A[q] * exp(-st.Ti[q] / T);
                fit = fit * rsT;
            }
            const double lam = st.table >= 0 ? nl_apply(m.lamref + (size_t)st.table * kNlNT,
                                                        m.Ssup + (size_t)st.table * kNlNT * kNlNNE,
                                                        m.lnL + (size_t)st.table * kNlNT * kNlNNE, at, fit)
                                             : fit;
            o.cool = o.cool + ne * nel * frac[i - 1] * lam;
        }
        if (e.kind == 1 && e.nstage >= 2) {   // [C II] 158 um, H impact
            const double nion = e.abund * nH * frac[1];
            const double qul = 7.6e-10 * pow(T / 100.0, 0.14);
            const double qlu = 2.0 * qul * exp(-91.25 / T);
            o.cool_H = o.cool_H + nion * nHI * qlu * (91.25 * kKboltz) / (1.0 + nHI * (qul + qlu) / A_CII);
        } else if (e.kind == 2) {             // [O I] 63 um
            const double nion = e.abund * nH * frac[0];
            const double qul = 9.2e-11 * pow(T / 100.0, 0.67);
            const double qlu = 0.6 * qul * exp(-227.7 / T);
            o.cool_H = o.cool_H + nion * nHI * qlu * (227.7 * kKboltz) / (1.0 + nHI * (qul + qlu) / A_OI);
        }
#pragma unroll
        for (int j = 2; j <= kMaxSt; ++j)
            if (j <= e.nstage) {
                const int zion = j - 1;
                ff = ff + e.abund * frac[j - 1] * (double)(zion * zion) * g[min(zion, 4) - 1];
            }
#pragma unroll
        for (int i = 1; i <= kMaxSt - 1; ++i)
            if (i <= e.nstage - 1) o.heat = o.heat + e.abund * nH * frac[i - 1] * m.eheat[il * m.ntr + e.tr0 + i - 1];
    }
    o.freefree = 1.42554e-27 * sqrt(T) * ne * nH * ff;
    return o;
}

// species_stage_cache_refresh from the shared cache (as metal_opacity_fill).
template <typename R>
__device__ __noinline__ void lane_opacity_fill(const LaneCache c, long long il, double nH, double ne, double xHI,
                                               double colscale) {
    const MetalDev& m = *c.m;
    R* op = static_cast<R*>(m.opac) + il * m.ntrp;
    const double nHI = nH * xHI, nHII = nH * (1.0 - xHI);
    for (int ie = 0; ie < m.nel; ++ie) {
        const MetalEl e = m.el[ie];
        double n[kMaxSt - 1], d[kMaxSt - 1], xi[kMaxSt - 1], xr[kMaxSt - 1], f[kMaxSt];
        lane_rates(c, e, ne, nHI, nHII, n, d, xi, xr);
        lane_fracs(e.nstage, n, d, f);
#pragma unroll
        for (int it = 1; it <= kMaxSt - 1; ++it)
            if (it <= e.nstage - 1) op[m.tr[e.tr0 + it - 1].flat] = (R)(nH * (e.abund * f[it - 1]) * colscale);
    }
}

// ---- the per-lane root searches ---------------------------------------------

// solve_cell_fast with the H root of every n_e evaluation
// (hydrogen_neutral_fraction_warm, falling back to the Illinois iteration)
// as one machine that asks for one cascade sum at a time.
struct CellSolve {
    Coef k;
    double g0, g1, g2, nH, yHe, floor, top;
    int with_ne, with_cx;
    // n_e root (solve_cell_ls): ph 0 first point, 1 search, 2 false position, 9 done
    int ph, nev, side, it;
    double a, fa, b, fb, c, fac, la, lb;
    CellState ea, eb, ec;
    // H root of the evaluation at c: hph 0 substitution, 1-2 Illinois end
    // points, 3 Illinois steps, 4 the sums at the root, 5 done
    int hph, hk, hkk;
    double hx, hprev, xa, xb, Ra, Rb, hscale, A, B, hnem;
    // the last two evaluations (n_e, x) of this solve: the H root's start is
    // their linear extrapolation to the next n_e
    double pc1, px1, pc2, px2;
    int npv;

    // the x at which the pending sum is taken
    __device__ __forceinline__ double xe() const { return hph == 1 ? 0.0 : hph == 2 ? 1.0 : hx; }

    __device__ __forceinline__ void h_begin() {
        A = k.aH * c;
        B = g0 + (k.cH + k.aH) * c;
        hnem = 0.0;
        if (with_cx) {
            hph = 0; hk = 0; hkk = 0;
            double xg = ec.x;
            if (npv >= 2 && pc1 != pc2) xg = px1 + (px1 - px2) * ((c - pc1) / (pc1 - pc2));
            hx = fmin(fmax(xg, 0.0), 1.0);
            hprev = 1.0e300;
            xa = 0.0; xb = 1.0; Ra = 0.0; Rb = 0.0; hscale = 0.0;
        } else {
            hx = B > 0.0 ? A / B : 1.0;
            hph = with_ne ? 4 : 5;
        }
    }

    // one cascade sum (em, rin, rout) at (c, xe())
    __device__ __forceinline__ void h_feed(double em, double rin, double rout) {
        if (hph == 0) {
            const double Rx = hx * (B + rin + rout) - (A + rin);
            const double sc = A + B + fabs(A + rin) + fabs(B + rout);
            const double xn = fmin(fmax((A + rin) / (B + rin + rout), 0.0), 1.0);
            const int v = h_subst_verdict(hx, xn, Rx, sc, hprev);
            if (v == 1) {
                hnem = em;
                hph = 5;
            } else if (v == 2 || ++hk >= 8) {
                hph = 1;
            } else {
                hprev = fabs(Rx);
                hx = xn;
            }
        } else if (hph == 1) {
            Ra = -(A + rin);
            hph = 2;
        } else if (hph == 2) {
            Rb = B + rout;
            hscale = A + B + fabs(Ra) + fabs(Rb);
            hx = xb;
            hkk = 0;
            hph = 3;
        } else if (hph == 3) {
            const double Rx = hx * (B + rin + rout) - (A + rin);
            if (fabs(Rx) <= 1.0e-15 * hscale || fabs(xb - xa) <= 1.0e-15) {
                hph = 4;
            } else {
                if (Rx * Rb < 0.0) {
                    xa = xb;
                    Ra = Rb;
                } else {
                    Ra = 0.5 * Ra;
                }
                xb = hx;
                Rb = Rx;
            }
        } else {   // hph == 4
            hnem = em;
            hph = 5;
        }
        if (hph == 3) {   // the next Illinois point
            if (++hkk > 80 || Rb == Ra) {
                hph = 4;
            } else {
                hx = xb - Rb * (xb - xa) / (Rb - Ra);
                hx = fmin(fmax(hx, fmin(xa, xb)), fmax(xa, xb));
            }
        }
    }

    // cell_electrons at c is complete: one step of the n_e root
    __device__ __forceinline__ void eval_done() {
        const double r1 = fmin((g1 + k.cHe1 * c) / (k.aHe2 * c), 1.0e150);
        const double r2 = fmin((g2 + k.cHe2 * c) / (k.aHe3 * c), 1.0e150);
        ec.x = hx;
        pc2 = pc1; px2 = px1;
        pc1 = c; px1 = hx;
        ++npv;
        ec.h1 = 1.0 / (1.0 + r1 + r1 * r2);
        ec.h2 = ec.h1 * r1;
        const double h3 = ec.h2 * r2;
        double nen = nH * ((1.0 - ec.x) + yHe * (ec.h2 + 2.0 * h3));
        if (with_ne) nen = nen + hnem;
        const double fc = nen - c;
        ++nev;
        bool to_fp = false;
        if (ph == 0) {
            fa = fc; ea = ec; b = a; fb = fa; eb = ea;
            if (fabs(fa) <= 2.0e-10 * a) {
                ph = 9;
            } else {
                c = fa > 0.0 ? fmin(a + fa, top) : fmax(a + fa, floor);
                if (!(c > 0.0)) c = floor;
                ph = 1;
            }
        } else if (ph == 1) {
            b = c; fb = fc; eb = ec;
            if (fabs(fc) <= 2.0e-10 * c || fc == 0.0) {
                ph = 9;
            } else if ((fc > 0.0) != (fa > 0.0)) {
                to_fp = true;
            } else if (c >= top || c <= floor) {
                ph = 9;
            } else {
                const double lA = log(a), lC = log(c);
                double ld = lC - fc * (lC - lA) / (fc - fa);
                const bool ahead = fc > 0.0 ? ld > lC : ld < lC;
                const double lim = log(fac);
                if (!(fabs(fc) < fabs(fa)) || !ahead || !(fabs(ld - lC) <= lim)) ld = fc > 0.0 ? lC + lim : lC - lim;
                a = c; fa = fc; ea = ec;
                c = fc > 0.0 ? fmin(exp(ld), top) : fmax(exp(ld), floor);
                fac = fac * fac;
                if (nev >= 60) to_fp = true;
            }
        } else {   // ph == 2: Anderson-Bjorck step at c
            b = c;
            eb = ec;
            ++it;
            const double lc = log(c);
            if (fabs(fc) <= 2.0e-10 * c || fc == 0.0) {
                ph = 9;
            } else if ((fc > 0.0) == (fb > 0.0)) {
                if (side == -1) {
                    const double mm = 1.0 - fc / fb;
                    fa = fa * (mm > 0.0 ? mm : 0.5);
                }
                lb = lc; fb = fc; side = -1;
            } else {
                if (side == +1) {
                    const double mm = 1.0 - fc / fa;
                    fb = fb * (mm > 0.0 ? mm : 0.5);
                }
                la = lc; fa = fc; side = +1;
            }
        }
        if (to_fp) {
            la = log(a);
            lb = log(b);
            side = 0;
            it = 0;
            ph = 2;
        }
        if (ph == 2) {   // the next false-position point, or the end of the search
            const double width = fabs(lb - la);
            if (width <= 1.0e-13 || it >= 100 || nev >= 160) {
                ph = 9;
            } else {
                double lc = (la * fb - lb * fa) / (fb - fa);
                if (!(fabs(lc - la) > 1.0e-3 * width && fabs(lc - lb) > 1.0e-3 * width)) lc = 0.5 * (la + lb);
                c = exp(lc);
            }
        }
        if (ph != 9) h_begin();
    }

    // advance until a cascade sum is pending (true) or the root is found
    __device__ __forceinline__ bool settle() {
        for (int guard = 0; guard < 512 && ph != 9; ++guard) {
            if (hph != 5) return true;
            eval_done();
        }
        ph = 9;
        return false;
    }

    __device__ __forceinline__ void begin(double xHI, double xHeI, double xHeII, double ne, double nemax) {
        floor = 1.0e-12 * nH;
        top = nemax * nH;
        ph = 0; nev = 0; side = 0; it = 0;
        fa = 0.0; b = 0.0; fb = 0.0; fac = 4.0; la = 0.0; lb = 0.0;
        npv = 0; pc1 = pc2 = px1 = px2 = 0.0;
        ea = {xHI, xHeI, xHeII};
        eb = ea;
        ec = ea;
        const double xHeIII = fmax(0.0, 1.0 - xHeI - xHeII);
        a = ne > floor ? ne : fmax(nH * ((1.0 - xHI) + yHe * (xHeII + 2.0 * xHeIII)), floor);
        a = fmin(a, top);
        c = a;
        h_begin();
    }
};

// thermal_bracketed's temperature search for one lane: TRoot.
using TempSearch = TRoot;

// Solver trips between the block barriers of lane_solve: one (measured on
// the 128^3 metals update: 133 ms, against 148 ms with a barrier every
// second trip and 164 ms every fourth).
constexpr int kLaneSyncTrips = 1;

// One lane's leaf.
struct LaneLeaf {
    long long il;
    bool has;
    double nH, x0, h10, h20, T0;
    double xHI, xHeI, xHeII, ne;
    int passes, nsum, nev;
    TempSearch ts;
    // the last two solved (ln T, ln n_e) of this leaf: the next trial's n_e
    // root starts from their linear extrapolation
    double lt1, ln1, lt2, ln2;
    int ntr;
};

// Leaf number q of the work order (the most work first).
__device__ __forceinline__ long long lane_leaf_of(const ThArgs& a, long long q) {
    return a.order ? (long long)a.order[a.b.nleaf - 1 - q] : q;
}

// Claims leaves for the lanes without one until each has an active leaf or
// the order is exhausted; leaves without gas are written as they are met.
__device__ __forceinline__ void lane_claim(const ThArgs& a, unsigned long long* next, LaneLeaf& L, bool& exhausted,
                                           int lane) {
    const BalArgs& b = a.b;
    for (;;) {
        const bool want = !L.has && !exhausted;
        const unsigned mask = __ballot_sync(kFull, want);
        if (!mask) return;
        unsigned long long base = 0;
        if (lane == __ffs(mask) - 1) base = atomicAdd(next, (unsigned long long)__popc(mask));
        base = __shfl_sync(kFull, base, __ffs(mask) - 1);
        if (want) {
            const long long q = (long long)base + __popc(mask & ((1u << lane) - 1u));
            if (q >= b.nleaf) {
                exhausted = true;
            } else {
                const long long il = lane_leaf_of(a, q);
                const double nH = b.nH[il];
                L.il = il;
                L.nH = nH;
                L.x0 = b.xHI[il];
                L.h10 = b.xHeI[il];
                L.h20 = b.xHeII[il];
                L.T0 = b.Te[il];
                if (nH > 0.0) {
                    L.has = true;
                    L.xHI = L.x0; L.xHeI = L.h10; L.xHeII = L.h20;
                    L.ne = b.ne[il];
                    L.passes = 0; L.nsum = 0; L.nev = 0; L.ntr = 0;
                    L.ts.begin(a.Twarm ? a.Twarm[il] : L.T0, a.te_min, a.te_max, a.tfac0, a.Twarm ? a.gate : 0.0);
                } else {
                    b.ne[il] = 0.0;
                    write_columns(b.col, il, b.nabs, b.fp32, nH, b.yHe, L.x0, L.h10, L.h20, b.colscale,
                                  b.rhokap ? b.rhokap[il] : 0.0);
                    if (a.work) a.work[il] = 0u;
                }
            }
        }
    }
}

// The written state of a solved leaf (thermal_mod.f90:191-203): relaxation,
// charge neutrality with the cache at the final temperature, the opacity
// weights and columns; every lane enters, `fin` marks the lanes that write.
__device__ __noinline__ void lane_finish(const ThArgs& a, const LaneCache& cache, LaneLeaf& L, bool fin,
                                         ThermalAcc& acc) {
    const BalArgs& b = a.b;
    const double w = b.relax;
    const double nH = L.nH;
    const double te = L.ts.tr;
    const double xn = (1.0 - w) * L.x0 + w * L.xHI;
    const double h1n = (1.0 - w) * L.h10 + w * L.xHeI;
    const double h2n = (1.0 - w) * L.h20 + w * L.xHeII;
    const double h3n = fmax(0.0, 1.0 - h1n - h2n);
    double nen = nH * ((1.0 - xn) + b.yHe * (h2n + 2.0 * h3n));
    if (b.metal_ne) {   // charge_neutrality_ne, lanes in step
        const double nHI = nH * xn, nHII = nH * (1.0 - xn), ne_HHe = nen;
        double ne = fmax(L.ne, 1.0e-12 * nH);
        int itn = 0;
        bool run = fin;
        while (__any_sync(kFull, run)) {
            const double ne_old = ne;
            double nem = 0.0, rin, rout;
            warp_sums(cache, run, nH, ne_old, nHI, nHII, nem, rin, rout);
            if (!run) continue;
            ne = ne_HHe + nem;
            ne = fmax(0.5 * (ne + ne_old), 1.0e-12 * nH);
            if (fabs(ne - ne_old) <= 1.0e-10 * ne || ++itn >= 200) run = false;
        }
        nen = ne;
    }
    if (!fin) return;
    const long long il = L.il;
    if (b.fp32) lane_opacity_fill<float>(cache, il, nH, nen, xn, b.colscale);
    else lane_opacity_fill<double>(cache, il, nH, nen, xn, b.colscale);
    ++acc.solved;
    acc.tpass += (unsigned long long)L.passes;
    acc.tsums += (unsigned long long)L.nsum;
    acc.nevals += (unsigned long long)L.nev;
    if (L.ts.accepted) ++acc.accepted;
    if (a.work) a.work[il] = (unsigned)min(L.nsum, 65535);
    b.xHI[il] = xn;
    b.xHeI[il] = h1n;
    b.xHeII[il] = h2n;
    b.ne[il] = nen;
    b.Te[il] = te;
    write_columns(b.col, il, b.nabs, b.fp32, nH, b.yHe, xn, h1n, h2n, b.colscale, b.rhokap ? b.rhokap[il] : 0.0);
    const double dx = fabs(xn - L.x0);
    acc.mdx = fmax(acc.mdx, dx);
    acc.mdt = fmax(acc.mdt, fabs(te - L.T0) / L.T0);
    const double vol = leaf_vol(b, il);
    acc.s1 = acc.s1 + vol * dx;
    acc.s2 = acc.s2 + vol * (1.0 - xn);
    acc.s3 = acc.s3 + vol * nen * fabs(te - L.T0);
    acc.s4 = acc.s4 + vol * nen * te;
    L.has = false;
}

// The leaves of one nebula by the warps of one block until its work order is
// exhausted (every thread of the block calls it).
__device__ __noinline__ void lane_solve(const ThArgs& a, unsigned long long* next, const LaneCache& cache,
                                        ThermalAcc& acc, int lane) {
    const BalArgs& b = a.b;
    const long long n = b.nleaf;
    LaneLeaf L = {};
    bool exhausted = false;
    CellSolve cs;
    cs.yHe = b.yHe;
    cs.with_ne = b.metal_ne;
    cs.with_cx = b.two_way;
    for (int trip = 0;; ++trip) {
        lane_claim(a, next, L, exhausted, lane);
        // every warp of the block takes the same trips, with a barrier every
        // kLaneSyncTrips of them: the block's warps stay near the same point
        // of the solver's code, which then stays in the instruction cache.
        // Only a barrier trip ends the loop, for every warp at once.
        if (trip % kLaneSyncTrips == 0 && !__syncthreads_or(L.has ? 1 : 0)) return;
        const bool ev = L.has;   // every lane with a leaf evaluates its net rate at ts.t
        const double T = L.ts.t;
        bool need = false;
        if (ev) {
            lane_prepare(cache, L.il, T);
            cs.k = coef_at_call(b.rs, b.caseA, T);
            cs.g0 = b.rates[L.il];
            cs.g1 = b.rates[n + L.il];
            cs.g2 = b.rates[2 * n + L.il];
            cs.nH = L.nH;
            double ne0 = L.ne;   // the n_e root's first point
            if (L.ntr >= 2 && L.lt1 != L.lt2 && L.ne > 0.0) {
                const double lnT = log(T);
                double d = (L.ln1 - L.ln2) / (L.lt1 - L.lt2) * (lnT - L.lt1);
                d = fmin(fmax(d, -0.7), 0.7);   // within a factor of two of the last root
                ne0 = exp(L.ln1 + d);
            }
            cs.begin(L.xHI, L.xHeI, L.xHeII, ne0, b.nemax);
            need = cs.settle();
        }
        int nsum = 0;
        while (__any_sync(kFull, need)) {   // one cascade sum per searching lane per trip
            double em = 0.0, rin = 0.0, rout = 0.0;
            const double x = need ? cs.xe() : 0.0;
            const double cnH = need ? cs.nH : 0.0, cc = need ? cs.c : 0.0;
            warp_sums(cache, need, cnH, cc, cnH * x, cnH * (1.0 - x), em, rin, rout);
            if (!need) continue;
            ++nsum;
            cs.h_feed(em, rin, rout);
            need = cs.settle();
        }
        L.nsum += nsum;
        bool fin = false;
        if (ev) {
            L.passes += cs.nev;
            L.ne = cs.b;
            if (L.ne > 0.0) {
                L.lt2 = L.lt1; L.ln2 = L.ln1;
                L.lt1 = log(T); L.ln1 = log(L.ne);
                ++L.ntr;
            }
            L.xHI = cs.eb.x;
            L.xHeI = cs.eb.h1;
            L.xHeII = cs.eb.h2;
            const double nH = L.nH;
            const long long il = L.il;
            const double heat = nH * (L.xHI * b.rates[3 * n + il] +
                                      b.yHe * (L.xHeI * b.rates[4 * n + il] + L.xHeII * b.rates[5 * n + il]));
            const double cool = cooling_total(a.td, b.rs, b.caseA, b.yHe, T, nH, L.ne, L.xHI, L.xHeI, L.xHeII);
            double net = heat - cool;
            const MetalThermalTerms mt = lane_thermal(cache, a.td, il, T, nH, L.ne, nH * L.xHI, nH * (1.0 - L.xHI));
            net = net - mt.cool;
            net = net - mt.cool_H;
            if (b.metal_ff) net = net - mt.freefree;
            if (b.metal_heat) net = net + mt.heat;
            // heating plus cooling: the scale of the learned warm start's residual gate
            const double scale = fabs(heat) + fabs(cool) + fabs(mt.cool) + fabs(mt.cool_H) +
                                 (b.metal_ff ? fabs(mt.freefree) : 0.0) + (b.metal_heat ? fabs(mt.heat) : 0.0);
            ++L.nev;
            L.ts.feed(net, a.te_min, a.te_max, scale);
            fin = L.ts.ph == 9;
        }
        lane_finish(a, cache, L, fin, acc);
    }
}

// Shared memory of the lane kernels: the layout, then the cache.
__host__ __device__ __forceinline__ size_t lane_cache_offset() { return (sizeof(LaneLayout) + 255) & ~(size_t)255; }

__global__ void __launch_bounds__(kBThreads, 1) k_thermal_lane(const ThArgs a) {
    extern __shared__ __align__(16) unsigned char lane_smem[];
    __shared__ double red[6][kBThreads / 32];
    LaneLayout* L = reinterpret_cast<LaneLayout*>(lane_smem);
    double* S = reinterpret_cast<double*>(lane_smem + lane_cache_offset());
    if (threadIdx.x == 0) lane_layout_build(a.b.m, *L);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    LaneCache cache{S + threadIdx.x, (int)blockDim.x, L, &a.b.m, a.b.m.el, a.b.m.nel};
    ThermalAcc acc;
    lane_solve(a, a.next, cache, acc, lane);
    // block sums into partial[6 x block], counters
    double v[6] = {acc.mdx, acc.mdt, acc.s1, acc.s2, acc.s3, acc.s4};
    unsigned long long cnt[5] = {acc.solved, acc.tpass, acc.tsums, acc.nevals, acc.accepted};
    for (int o = 16; o > 0; o >>= 1) {
        v[0] = fmax(v[0], __shfl_down_sync(kFull, v[0], o));
        v[1] = fmax(v[1], __shfl_down_sync(kFull, v[1], o));
        for (int k = 2; k < 6; ++k) v[k] += __shfl_down_sync(kFull, v[k], o);
        for (int k = 0; k < 5; ++k) cnt[k] += __shfl_down_sync(kFull, cnt[k], o);
    }
    const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane == 0) {
        for (int k = 0; k < 6; ++k) red[k][w] = v[k];
        if (cnt[0]) atomicAdd(a.b.counters + 0, cnt[0]);
        if (cnt[1]) atomicAdd(a.b.counters + 2, cnt[1]);
        if (cnt[2]) atomicAdd(a.b.counters + 3, cnt[2]);
        if (cnt[3]) atomicAdd(a.b.counters + 4, cnt[3]);
        if (cnt[4]) atomicAdd(a.b.counters + 5, cnt[4]);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double r[6] = {red[0][0], red[1][0], red[2][0], red[3][0], red[4][0], red[5][0]};
        for (int q = 1; q < nw; ++q) {
            r[0] = fmax(r[0], red[0][q]);
            r[1] = fmax(r[1], red[1][q]);
            for (int k = 2; k < 6; ++k) r[k] = r[k] + red[k][q];
        }
        for (int k = 0; k < 6; ++k) a.b.partial[6 * blockIdx.x + k] = r[k];
    }
}
