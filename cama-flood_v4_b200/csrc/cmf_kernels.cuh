// cmf_kernels.cuh -- sm_100a device code of the CaMa-Flood physics time step (FP64).
//
// One outer step (CMF_PHYSICS_ADVANCE, src/cmf_ctrl_physics_mod.F90:21-153) is
//   k_stage   stage scheme at the start of the step + CFL minimum      (:54-59, :161-210)
//   k_ntdt    NT/DT per member, loop bound of the device-side sub-step loop (:205-206)
//   NT x { k_flux  outflow + dam + bifurcation flux         (CMF_CALC_OUTFLW, CMF_DAMOUT_CALC,
//                                                            CMF_CALC_PTHOUT / CMF_LEVEE_OPT_PTHOUT)
//          k_rate  storage-out gather and outflow limiter rate (LSPAMAT steps 1-2); advances the
//                  sub-step counter and the loop condition
//          k_store rescale + inflow gather + dam balance + CALC_VARS_PRE + CMF_CALC_STONXT +
//                  stage scheme + sub-step diagnostics        (LSPAMAT steps 2-3, :101-135)
//        }
//   k_budget  deterministic budget reduction of every member's last sub-step
// Three grid-wide dependencies per sub-step remain (outflow needs the downstream stage; the rate
// needs the upstream outflows; the inflow needs the downstream and upstream rates), so each
// phase is one kernel and the phases are ordered by the graph.
//
// Arithmetic follows the reference statement by statement, compiled with -fmad=false so no
// multiply-add is fused: x**(-1) is 1/x, x**2 is x*x, x**0.5 is an IEEE square root, the depth
// powers of the flux formulas are correctly rounded (pow_depth) and every other non-integral power
// is pow().  Default-real literals of the reference are promoted float values
// (F(...) below).  All gathers sum in the reference's loop order (ascending upstream sequence);
// there are no atomics on state, so results are independent of block size and timing.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define CMF_F(x) ((double)(float)(x))

namespace cmf {

// Occupancy of the latency-bound cell kernels: at most kCellThreads threads per block and the
// minimum resident blocks per SM (caps registers at 65536 / (threads x blocks)).  k_flux and
// k_store come in two profiles, one of the dimensions the engine's autotuner searches: with many
// cell-members in flight more resident warps beat the spills they cost (`wide`: 40/48 registers;
// 16 config-1 members 22.2 vs 24.4 ms per coupling step), while a grid of about two waves runs
// best with few spills (`small`: 64/64 registers, k_flux spill-free; one config-1 member 1.91 ms
// vs 1.95 ms with k_flux at 48).  Both profiles execute the same arithmetic; only the register
// allocation differs.
constexpr int kFluxMinBlocksWide = 6, kStoreMinBlocksWide = 5;
constexpr int kFluxMinBlocksSmall = 4, kStoreMinBlocksSmall = 4;
constexpr size_t kSmallCellMembers = size_t(1) << 19;   // untuned start: `small` up to this many cell-members
#ifndef CMF_STAGE_MINB
#define CMF_STAGE_MINB 6
#endif
constexpr int kCellThreads = 256;
constexpr int kUpSlots = 4;        // upstream cells per cell held in Net::up_ell

constexpr int kBudgets = 12;       // stopre stonxt stonew rivinf rivout stopre2 stonew2 rivsto fldsto fldare levsto dammiss
// dynamic shared memory of k_store: the last sub-step's budget terms, kBudgets per thread
inline size_t store_smem(int block) { return (size_t)kBudgets * block * sizeof(double); }
constexpr int kNtCap = 10000;      // bound of the device-side sub-step loop
// MemberCtl.err codes (mapped to the ABI's positive statuses by the engine)
constexpr int kErrNtCap = 2;       // DT_MIN non-finite or NT above kNtCap: no sub-step ran
constexpr int kErrNonFinite = 3;   // a sub-step produced a non-finite storage

struct MemberCtl {
    double dt_def;                 // DT at entry (DT_DEF)
    double dt;                     // sub-step DT
    double dt_min;                 // CFL minimum of this outer step
    double nadd;                   // NADD_adp before the current sub-step
    unsigned long long dtmin_bits; // atomicMin target (positive doubles order like their bit patterns)
    int nt;                        // sub-steps of this outer step
    int it;                        // index of the next sub-step
    int err;
    int pad;
    double budget[kBudgets];       // last finished sub-step
};

constexpr int kNtHist = 64;       // NT histogram bins (the last one holds NT >= kNtHist-1)

struct LoopCtl {
    int k;            // sub-step counter of the device-side loop (advanced by k_rate)
    int kcur;         // the sub-step the running k_flux/k_rate/k_store work on (set by k_flux)
    int ntmax;        // max NT over members
    int err;
    int split;        // 1 until the first sub-step after a host state upload: D2RIVOUT /= D2RIVOUT_PRE
    long long member_substeps;   // sum over outer steps and members of NT (throughput accounting)
    long long loop_iters;        // sum over outer steps of NTmax (kernel-launch accounting)
    long long outer_steps;
    long long near_int;          // (outer step, member) pairs whose DT_DEF/DT_MIN-0.01 lay within
                                 // 1e-12 (relative) of an integer: NT there hangs on DT_MIN's last bits
    long long nt_hist[kNtHist];  // (outer step, member) pairs by NT
    unsigned bar;                // grid-barrier arrival count of the persistent kernel (zeroed per launch)
    int bar_err;                 // set when a bounded wait of the persistent kernel ran out
};

// Static data shared by all members (device pointers).
struct Net {
    int N, R, L, P, Lp, M;
    const int *__restrict__ next;       // [N] 0-based downstream (river cells)
    const int *__restrict__ up_ptr;     // [N+1] upstream CSR, ascending sequence (I1UPST order)
    const int *__restrict__ up_idx;
    // [kUpSlots][N] the first upstream cells of each cell in I1UPST order, -1 past the last; with
    // more than kUpSlots of them the last slot holds -2 - (CSR position of the kUpSlots-th), and the
    // walk goes on in up_idx.  All slots of a cell are read at once, so the upstream values are
    // gathered one dependent load after the cell's own reads instead of two (pointer, index, value).
    const int *__restrict__ up_ell;
    const int *__restrict__ i2mask;     // [N]
    const double *__restrict__ rivelv, *__restrict__ elevtn, *__restrict__ nxtdst, *__restrict__ rivwth;
    const double *__restrict__ rivhgt, *__restrict__ rivlen, *__restrict__ rivman, *__restrict__ grarea;
    const double *__restrict__ rivstomax, *__restrict__ dwnelv;
    // D2NXTDST**(-1), D2RIVWTH**(-1), D2RIVLEN**(-1) of the outflow formulas, computed once at init
    // (the same correctly rounded reciprocal the reference evaluates every time)
    const double *__restrict__ inv_nxtdst, *__restrict__ inv_rivwth, *__restrict__ inv_rivlen;
    const double *__restrict__ fldstomax, *__restrict__ fldgrd, *__restrict__ fldhgt;   // [L][N]
    // bifurcation paths
    const int *__restrict__ pth_up, *__restrict__ pth_dn;   // [P] 0-based, -1 outside domain
    const int *__restrict__ pth_skip;                        // [P] bit0 plain/LSPAMAT skip, bit1 levee skip
    const double *__restrict__ pth_dst, *__restrict__ pth_elv, *__restrict__ pth_wth, *__restrict__ pth_man;
    const int *__restrict__ pout_ptr, *__restrict__ pout_idx, *__restrict__ pinf_ptr, *__restrict__ pinf_idx;
    // levee (compact per levee cell)
    const int *__restrict__ lev_id;     // [N] -1 when the cell carries the no-levee sentinels
    const double *__restrict__ levhgt, *__restrict__ levfrc, *__restrict__ bashgt, *__restrict__ levdst;
    const double *__restrict__ levbassto, *__restrict__ levtopsto, *__restrict__ levfilsto;
    // dams
    const int *__restrict__ i1dam;      // [N]
    const int *__restrict__ dam_id;     // [N] compact dam of the cell or -1
    const int *__restrict__ dam_stat;   // [D]
    const double *__restrict__ qn, *__restrict__ qf, *__restrict__ qa, *__restrict__ convol;
    const double *__restrict__ emevol, *__restrict__ norvol, *__restrict__ adjvol, *__restrict__ r_volupa;
    double pgrv, pmanfld, pdstmth, pcadp, pminslp, dfrcinc;
    int ladpstp, lfldout, lpthout, ldamout, llevee, ldamh22, ldiag;
    int ldiag_out;   // CMF_DIAG_AVEMAX_OUTPUT after every outer step, fused into its last sub-step
};

// Per-member state, member-major [M][N] (paths [M][Lp][P] / [M][P]).
struct State {
    double *rivsto, *fldsto, *levsto, *damsto, *daminf;
    double *rivout_raw, *fldout_raw;          // outflow before the LSPAMAT rescale (phase A -> C)
    double *rivout_pre, *fldout_pre;          // D2RIVOUT_PRE / D2FLDOUT_PRE (== D2RIVOUT / D2FLDOUT after a step)
    double *rivout_cur, *fldout_cur;          // host-set D2RIVOUT / D2FLDOUT while LoopCtl.split
    double *rivdph_pre, *fldsto_pre;
    double *rivdph, *flddph, *fldfrc, *fldare, *sfcelv, *storge, *levdph, *rivvel;
    double *rivinf, *fldinf, *pthout, *outflw, *rate;
    double *pthflw_raw, *pthflw_pre, *pthsum_raw, *pthsum;
    double *runoff;
    // sub-step diagnostics
    double *a_rivout, *a_fldout, *a_outflw, *a_rivvel, *a_pthout, *a_runoff, *a_daminf;
    double *m_storge, *m_outflw, *m_rivdph, *a_pthflw, *a_pthsum;
    // output-interval averages and maxima (D2*_oAVG, D2*_oMAX, D1PTHFLW_oAVG, NADD_out per member)
    double *o_rivout, *o_fldout, *o_outflw, *o_rivvel, *o_pthout, *o_runoff, *o_daminf;
    double *om_storge, *om_outflw, *om_rivdph, *o_pthflw, *o_nadd;
    MemberCtl *ctl;
    LoopCtl *loop;
    double *partials;                         // [M][nblk][kBudgets]
};

__device__ __forceinline__ double dmax(double a, double b) { return (a > b) ? a : b; }
__device__ __forceinline__ double dmin(double a, double b) { return (a < b) ? a : b; }

// Own-cell reads of the per-cell code go through an accessor (OwnG: the arrays in global memory,
// static maps through the read-only path), so that a kernel could stage a cell's own values
// elsewhere without touching the arithmetic.  Static maps are indexed by the cell i, member state
// by g = m*N + i; reads of another cell (downstream, upstream, path ends) go to global memory
// through Net/State.
#define CMF_OWN_STATIC(name) \
    __device__ __forceinline__ double name(int i) const { return __ldg(&n.name[i]); }
#define CMF_OWN_STATE(name) \
    __device__ __forceinline__ double name(size_t g) const { return s.name[g]; }
struct OwnG {
    const Net &n;
    const State &s;
    CMF_OWN_STATIC(rivelv) CMF_OWN_STATIC(elevtn) CMF_OWN_STATIC(nxtdst) CMF_OWN_STATIC(rivwth)
    CMF_OWN_STATIC(rivhgt) CMF_OWN_STATIC(rivlen) CMF_OWN_STATIC(rivman) CMF_OWN_STATIC(grarea)
    CMF_OWN_STATIC(rivstomax) CMF_OWN_STATIC(inv_nxtdst) CMF_OWN_STATIC(inv_rivwth) CMF_OWN_STATIC(inv_rivlen)
    __device__ __forceinline__ int next(int i) const { return __ldg(&n.next[i]); }
    __device__ __forceinline__ int up_lo(int i) const { return __ldg(&n.up_ptr[i]); }
    __device__ __forceinline__ int up_hi(int i) const { return __ldg(&n.up_ptr[i + 1]); }
    __device__ __forceinline__ int up_slot(int k, int i) const { return __ldg(&n.up_ell[(size_t)k * n.N + i]); }
    __device__ __forceinline__ int i1dam(int i) const { return __ldg(&n.i1dam[i]); }
    CMF_OWN_STATE(rivsto) CMF_OWN_STATE(fldsto) CMF_OWN_STATE(levsto) CMF_OWN_STATE(rivdph)
    CMF_OWN_STATE(rivdph_pre) CMF_OWN_STATE(rivout_pre) CMF_OWN_STATE(fldout_pre) CMF_OWN_STATE(fldsto_pre)
    CMF_OWN_STATE(flddph) CMF_OWN_STATE(fldfrc) CMF_OWN_STATE(storge) CMF_OWN_STATE(runoff)
    CMF_OWN_STATE(rivout_raw) CMF_OWN_STATE(fldout_raw) CMF_OWN_STATE(rate)
    CMF_OWN_STATE(a_rivvel) CMF_OWN_STATE(a_rivout) CMF_OWN_STATE(a_fldout) CMF_OWN_STATE(a_outflw)
    CMF_OWN_STATE(a_pthout) CMF_OWN_STATE(m_outflw) CMF_OWN_STATE(m_rivdph) CMF_OWN_STATE(m_storge)
};
#undef CMF_OWN_STATIC
#undef CMF_OWN_STATE

// f(j) for every upstream cell j of cell i, in I1UPST order (the order of every upstream sum)
template <class Own, class F>
__device__ __forceinline__ void for_each_upstream(const Net &n, const Own &w, int i, F f) {
    int slot[kUpSlots];
#pragma unroll
    for (int k = 0; k < kUpSlots; k++) slot[k] = w.up_slot(k, i);
#pragma unroll
    for (int k = 0; k < kUpSlots - 1; k++) {
        if (slot[k] < 0) return;
        f(slot[k]);
    }
    const int last = slot[kUpSlots - 1];
    if (last >= 0) {
        f(last);
    } else if (last < -1) {                       // more than kUpSlots upstream cells
        const int k1 = __ldg(&n.up_ptr[i + 1]);
        for (int k = -2 - last; k < k1; k++) f(__ldg(&n.up_idx[k]));
    }
}


// x**(-7._JPRB/3._JPRB) and x**(-4._JPRB/3._JPRB) of the local-inertial flux formulas
// (src/cmf_calc_outflw_mod.F90:74,106,133,162; src/cmf_calc_pthout_mod.F90:67;
// src/cmf_ctrl_levee_mod.F90:553,573): pow(x, y) for the
// doubles y nearest -7/3 and -4/3, correctly rounded, for the positive depths these formulas take.
// The exponent is y = -K/3 + d with d its rounding offset (d = -0x1.5555555555555p-53 for K = 7,
// +0x1.5555555555555p-54 for K = 4), so x^y = (x^(-1/3))^K * x^d:
//   c0 = rcbrt(x); one Newton step for the inverse cube root, c = c0 (1 + r/3), r = 1 - x c0^3,
//     with c0^3 formed exactly by Dekker's FMA products (c carried as a double-double);
//   c^K in double-double (Dekker products; relative error about 2^-100);
//   x^d = 1 + d ln x to first order (|d ln x| < 3e-15, so ln x to single precision suffices).
// The sum is rounded once.  Outside (1e-300, 1e300) the general pow is used.
struct DD {
    double hi, lo;
};
__device__ __forceinline__ DD dd_mul(DD a, DD b) {
    const double p = a.hi * b.hi;
    double e = fma(a.hi, b.hi, -p);
    e = e + (a.hi * b.lo + a.lo * b.hi);
    return {p, e};
}
template <int K>
__device__ __forceinline__ double pow_depth(double x) {
    static_assert(K == 7 || K == 4, "exponents -7/3 and -4/3 only");
    constexpr double y = -(double)K / 3.0;
    constexpr double d = (K == 7) ? -0x1.5555555555555p-53 : 0x1.5555555555555p-54;
    if (!(x > 1e-300 && x < 1e300)) return pow(x, y);
    const double c0 = rcbrt(x);
    const double p2 = c0 * c0, e2 = fma(c0, c0, -p2);
    const double p3 = p2 * c0, e3 = fma(p2, c0, -p3);
    const double t = fma(x, p3, -1.0);
    const double r = -(t + x * (e3 + e2 * c0));
    const DD c = {c0, c0 * (r * (1.0 / 3.0))};
    const DD c2 = dd_mul(c, c), c4 = dd_mul(c2, c2);
    const DD v = (K == 7) ? dd_mul(dd_mul(c4, c2), c) : c4;
    const double corr = v.hi * (d * (double)logf((float)x));
    return v.hi + (v.lo + corr);
}

// (PGRV*DDPH)**(-0.5) of CALC_ADPSTP (src/cmf_ctrl_physics_mod.F90:193,201), correctly rounded.
// NT is INT(DT_DEF/DT_MIN - 0.01) + 1, so a last-bit change of the minimum can move NT; the
// oracle's glibc pow is correctly rounded for all but rare arguments, and so is this:
//   r0 = rsqrt(x) (within an ulp or two); the residual e = 1 - x r0^2 from exact FMA products
//   (r0^2 = p + pe exactly, x p - 1 rounded once at ~2^-51 magnitude); then one Newton step with
//   its second-order term, x^-1/2 = r0 (1 + e/2 + 3e^2/8 + O(e^3)), added to r0 and rounded once.
// Relative error before the final rounding is about 2^-100.  Outside (1e-300, 1e300) pow is used.
__device__ __forceinline__ double rsqrt_cr(double x) {
    if (!(x > 1e-300 && x < 1e300)) return pow(x, -0.5);
    const double r0 = rsqrt(x);
    const double p = r0 * r0, pe = fma(r0, r0, -p);
    const double t = fma(x, p, -1.0);
    const double e = -(t + x * pe);
    return r0 + r0 * (e * (0.5 + 0.375 * e));
}

// CFL key of one cell, PCADP*DDST*(PGRV*DDPH)**(-0.5) (src/cmf_ctrl_physics_mod.F90:190-202)
__device__ __forceinline__ double cfl_key(double pcadp, double ddst, double pgrv, double rivdph) {
    const double ddph = (rivdph > 0.01) ? rivdph : 0.01;
    return (pcadp * ddst) * rsqrt_cr(pgrv * ddph);
}

// ------------------------------------------------------------------------------------------
// stage schemes (one cell)
// ------------------------------------------------------------------------------------------
struct StageOut {
    double rivsto, fldsto, levsto, rivdph, flddph, fldfrc, fldare, levdph;
};

// CMF_CALC_FLDSTG_DEF body, src/cmf_calc_fldstg_mod.F90:46-97
template <class Own>
__device__ __forceinline__ StageOut stage_def(const Net &n, const Own &w, int i, double rivsto, double fldsto) {
    StageOut o;
    const int N = n.N, L = n.L;
    const double pstoall = rivsto + fldsto;
    const double rsm = w.rivstomax(i);
    o.levsto = 0.0;
    o.levdph = 0.0;
    if (pstoall > rsm) {
        const double len = w.rivlen(i), wth = w.rivwth(i);
        const double inc = (w.grarea(i) / len) * n.dfrcinc;
        int I = 0;   // 0-based layer
        double sfil = rsm, wfil = wth, dfil = 0.0;
        while (I < L) {
            const double smax = __ldg(&n.fldstomax[(size_t)I * N + i]);
            if (!(pstoall > smax)) break;
            sfil = smax;
            wfil = wfil + inc;
            dfil = dfil + __ldg(&n.fldgrd[(size_t)I * N + i]) * inc;
            I++;
        }
        double wadd;
        if (I >= L) {
            wadd = 0.0;
            o.flddph = dfil + ((pstoall - sfil) / wfil) / len;
        } else {
            const double gr = __ldg(&n.fldgrd[(size_t)I * N + i]);
            const double sadd = pstoall - sfil;
            wadd = -wfil + sqrt(wfil * wfil + ((2.0 * sadd) / len) / gr);
            o.flddph = dfil + gr * wadd;
        }
        double rs = rsm + (len * wth) * o.flddph;
        rs = dmin(rs, pstoall);
        o.rivsto = rs;
        o.rivdph = (rs / len) / wth;
        o.fldsto = dmax(pstoall - rs, 0.0);
        double frc = ((-wth + wfil) + wadd) / (inc * (double)L);
        frc = dmax(frc, 0.0);
        frc = dmin(frc, 1.0);
        o.fldfrc = frc;
        o.fldare = w.grarea(i) * frc;
    } else {
        o.rivsto = pstoall;
        o.rivdph = dmax((pstoall / w.rivlen(i)) / w.rivwth(i), 0.0);
        o.fldsto = 0.0;
        o.flddph = 0.0;
        o.fldfrc = 0.0;
        o.fldare = 0.0;
    }
    return o;
}

// CMF_LEVEE_FLDSTG body, src/cmf_ctrl_levee_mod.F90:301-461
template <class Own>
__device__ __forceinline__ StageOut stage_levee(const Net &n, const Own &w, int i, double rivsto, double fldsto,
                                                double levsto) {
    StageOut o;
    const int N = n.N, L = n.L;
    const double pstoall = (rivsto + fldsto) + levsto;
    const double rsm = w.rivstomax(i);
    const double len = w.rivlen(i), wth = w.rivwth(i);
    const double inc = (w.grarea(i) / len) * n.dfrcinc;
    const double grarea = w.grarea(i);
    const int lv = __ldg(&n.lev_id[i]);
    const double lbas = lv >= 0 ? __ldg(&n.levbassto[lv]) : 1.E18;
    if (pstoall > rsm) {
        if (pstoall < lbas) {                                                       // case 1
            int I = 0;
            double sfil = rsm, wfil = wth, dfil = 0.0, wadd;
            while (I < L) {
                const double smax = __ldg(&n.fldstomax[(size_t)I * N + i]);
                if (!(pstoall > smax)) break;
                sfil = smax; wfil = wfil + inc; dfil = dfil + __ldg(&n.fldgrd[(size_t)I * N + i]) * inc;
                I++;
            }
            if (I < L) {
                const double gr = __ldg(&n.fldgrd[(size_t)I * N + i]);
                wadd = -wfil + sqrt(wfil * wfil + ((2.0 * (pstoall - sfil)) / len) / gr);
                o.flddph = dfil + gr * wadd;
            } else {
                wadd = 0.0;
                o.flddph = dfil + ((pstoall - sfil) / wfil) / len;
            }
            o.rivsto = rsm + (len * wth) * o.flddph;
            o.rivdph = (o.rivsto / len) / wth;
            o.fldsto = dmax(pstoall - o.rivsto, 0.0);
            double frc = ((-wth + wfil) + wadd) / (inc * (double)L);
            frc = dmax(frc, 0.0);
            frc = dmin(frc, 1.0);
            o.fldfrc = frc;
            o.fldare = grarea * frc;
            o.levsto = 0.0;
            o.levdph = 0.0;
        } else {
            const double lhgt = __ldg(&n.levhgt[lv]), lfrc = __ldg(&n.levfrc[lv]), bhgt = __ldg(&n.bashgt[lv]), ldst = __ldg(&n.levdst[lv]);
            const double ltop = __ldg(&n.levtopsto[lv]), lfil = __ldg(&n.levfilsto[lv]);
            if (pstoall < ltop) {                                                   // case 2
                const double sadd = pstoall - lbas;
                const double wadd = ldst + wth;
                o.flddph = bhgt + (sadd / wadd) / len;
                o.rivsto = rsm + (len * wth) * o.flddph;
                o.rivdph = (o.rivsto / len) / wth;
                o.fldsto = dmax(pstoall - o.rivsto, 0.0);
                o.fldfrc = lfrc;
                o.fldare = grarea * lfrc;
                o.levsto = 0.0;
                o.levdph = 0.0;
            } else if (pstoall < lfil) {                                            // case 3
                o.flddph = lhgt;
                o.rivsto = rsm + (len * wth) * o.flddph;
                o.rivdph = (o.rivsto / len) / wth;
                o.fldsto = dmax(ltop - o.rivsto, 0.0);
                o.levsto = dmax((pstoall - o.rivsto) - o.fldsto, 0.0);
                const int ilev = (int)(lfrc * (double)L) + 1;   // 1-based layer with the levee
                double sfil = ltop, wfil = 0.0, dfil = 0.0, sadd;
                int I = ilev;                                   // 1-based
                while (I <= L) {
                    sadd = ((ldst + wth) * (lhgt - __ldg(&n.fldhgt[(size_t)(I - 1) * N + i]))) * len;
                    if (pstoall < __ldg(&n.fldstomax[(size_t)(I - 1) * N + i]) + sadd) break;
                    sfil = __ldg(&n.fldstomax[(size_t)(I - 1) * N + i]) + sadd;
                    wfil = inc * (double)I - ldst;
                    dfil = __ldg(&n.fldhgt[(size_t)(I - 1) * N + i]) - bhgt;
                    I++;
                }
                if (I <= L) {
                    const double gr = __ldg(&n.fldgrd[(size_t)(I - 1) * N + i]);
                    const double wadd = -wfil + sqrt(wfil * wfil + ((2.0 * (pstoall - sfil)) / len) / gr);
                    const double dadd = wadd * gr;
                    o.levdph = (bhgt + dfil) + dadd;
                    double frc = (wfil + ldst) / (inc * (double)L);
                    frc = dmax(frc, 0.0);
                    frc = dmin(frc, 1.0);
                    o.fldfrc = frc;
                    o.fldare = grarea * frc;
                } else {
                    const double dadd = ((pstoall - sfil) / wfil) / len;
                    o.levdph = (bhgt + dfil) + dadd;
                    o.fldfrc = 1.0;
                    o.fldare = grarea * 1.0;
                }
            } else {                                                                // case 4
                int I = 0;
                double sfil = rsm, wfil = wth, dfil = 0.0, wadd;
                while (I < L) {
                    const double smax = __ldg(&n.fldstomax[(size_t)I * N + i]);
                    if (!(pstoall > smax)) break;
                    sfil = smax; wfil = wfil + inc; dfil = dfil + __ldg(&n.fldgrd[(size_t)I * N + i]) * inc;
                    I++;
                }
                if (I < L) {
                    const double gr = __ldg(&n.fldgrd[(size_t)I * N + i]);
                    wadd = -wfil + sqrt(wfil * wfil + ((2.0 * (pstoall - sfil)) / len) / gr);
                    o.flddph = dfil + gr * wadd;
                } else {
                    wadd = 0.0;
                    o.flddph = dfil + ((pstoall - sfil) / wfil) / len;
                }
                o.fldfrc = ((-wth + wfil) + wadd) / (inc * (double)L);
                o.fldare = grarea * o.fldfrc;
                o.rivsto = rsm + (len * wth) * o.flddph;
                o.rivdph = (o.rivsto / len) / wth;
                const double sadd = ((o.flddph - lhgt) * (ldst + wth)) * len;
                o.fldsto = dmax((ltop + sadd) - o.rivsto, 0.0);
                o.levsto = dmax((pstoall - o.rivsto) - o.fldsto, 0.0);
                o.levdph = o.flddph;
            }
        }
    } else {                                                                        // case 0
        o.rivsto = pstoall;
        o.rivdph = dmax((pstoall / len) / wth, 0.0);
        o.fldsto = 0.0; o.flddph = 0.0; o.fldfrc = 0.0; o.fldare = 0.0; o.levsto = 0.0; o.levdph = 0.0;
    }
    return o;
}

// diag_only: D2FLDARE and D2SFCELV are read by nothing inside the sub-step loop, so the sub-steps
// write them on the last sub-step only (the values the caller observes are the same)
__device__ __forceinline__ void store_stage(const Net &n, const State &s, size_t gi, int i, const StageOut &o,
                                            bool diag_out = true) {
    s.rivsto[gi] = o.rivsto;
    s.fldsto[gi] = o.fldsto;
    s.rivdph[gi] = o.rivdph;
    s.flddph[gi] = o.flddph;
    s.fldfrc[gi] = o.fldfrc;
    if (diag_out) {
        s.fldare[gi] = o.fldare;
        s.sfcelv[gi] = __ldg(&n.rivelv[i]) + o.rivdph;
    }
    if (n.llevee) {
        s.levsto[gi] = o.levsto;
        s.levdph[gi] = o.levdph;
        s.storge[gi] = (o.rivsto + o.fldsto) + o.levsto;
    } else {
        s.storge[gi] = o.rivsto + o.fldsto;
    }
}

template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *smem /* [32*NV] */) {
    // fixed-shape tree: warp butterfly, then warp 0 over the warp partials -> deterministic
#pragma unroll
    for (int k = 0; k < NV; k++)
        for (int o = 16; o > 0; o >>= 1) v[k] = v[k] + __shfl_down_sync(0xffffffffu, v[k], o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; k++) smem[warp * NV + k] = v[k];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) {
            double x = lane < nw ? smem[lane * NV + k] : 0.0;
            for (int o = 16; o > 0; o >>= 1) x = x + __shfl_down_sync(0xffffffffu, x, o);
            v[k] = x;
        }
    }
}

// ------------------------------------------------------------------------------------------
// k_stage: stage scheme at the top of CMF_PHYSICS_ADVANCE + CALC_ADPSTP minimum
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kCellThreads, CMF_STAGE_MINB) k_stage(Net n, State s) {
    const int m = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double key = 1.0e308;
    if (i < n.N) {
        const size_t gi = (size_t)m * n.N + i;
        const OwnG w{n, s};
        const StageOut o = n.llevee ? stage_levee(n, w, i, s.rivsto[gi], s.fldsto[gi], s.levsto[gi])
                                    : stage_def(n, w, i, s.rivsto[gi], s.fldsto[gi]);
        store_stage(n, s, gi, i, o);
        if (n.ladpstp && __ldg(&n.i2mask[i]) == 0) key = cfl_key(n.pcadp, (i < n.R) ? __ldg(&n.nxtdst[i]) : n.pdstmth, n.pgrv, o.rivdph);
    }
    if (n.ladpstp) {
        for (int o = 16; o > 0; o >>= 1) key = dmin(key, __shfl_down_sync(0xffffffffu, key, o));
        __shared__ double wmin[32];
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
        if (lane == 0) wmin[warp] = key;
        __syncthreads();
        if (warp == 0) {
            double x = lane < nw ? wmin[lane] : 1.0e308;
            for (int o = 16; o > 0; o >>= 1) x = dmin(x, __shfl_down_sync(0xffffffffu, x, o));
            if (lane == 0 && x < 1.0e308) atomicMin(&s.ctl[m].dtmin_bits, (unsigned long long)__double_as_longlong(x));
        }
    }
}

// ------------------------------------------------------------------------------------------
// k_ntdt: NT and DT per member (src/cmf_ctrl_physics_mod.F90:205-206) and the loop bound
// ------------------------------------------------------------------------------------------
__global__ void k_ntdt(Net n, State s, cudaGraphConditionalHandle h, int use_cond) {
    __shared__ int smax[32];
    int ntmax = 1;
    long long ntsum = 0, near = 0;
    for (int m = threadIdx.x; m < n.M; m += blockDim.x) {
        MemberCtl &c = s.ctl[m];
        const double dt_def = c.dt_def;
        int nt = 1;
        double dt = dt_def;
        if (n.ladpstp) {
            const double dt_min = dmin(dt_def, __longlong_as_double((long long)c.dtmin_bits));
            c.dt_min = dt_min;
            const double x = dt_def * (1.0 / dt_min) - CMF_F(0.01);
            if (!(x >= 0.0) || x > (double)(kNtCap - 1)) {
                c.err = kErrNtCap;   // non-finite or oversized NT: refuse to loop
                nt = 0;
            } else {
                nt = (int)x + 1;
                dt = dt_def * (double)(1.0f / (float)nt);
                if (fabs(x - rint(x)) <= 1e-12 * dmax(x, 1.0)) near++;
            }
            c.dtmin_bits = (unsigned long long)__double_as_longlong(dt_def);
        } else {
            c.dt_min = dt_def;
        }
        c.nt = nt;
        c.dt = dt;
        c.it = 0;
        c.nadd = 0.0;
        ntmax = max(ntmax, nt);
        ntsum += nt;
        atomicAdd((unsigned long long *)&s.loop->nt_hist[min(nt, kNtHist - 1)], 1ull);
    }
    __shared__ long long ssum[32], snear[32];
    for (int o = 16; o > 0; o >>= 1) {
        ntmax = max(ntmax, __shfl_down_sync(0xffffffffu, ntmax, o));
        ntsum += __shfl_down_sync(0xffffffffu, ntsum, o);
        near += __shfl_down_sync(0xffffffffu, near, o);
    }
    if ((threadIdx.x & 31) == 0) { smax[threadIdx.x >> 5] = ntmax; ssum[threadIdx.x >> 5] = ntsum; snear[threadIdx.x >> 5] = near; }
    __syncthreads();
    if (threadIdx.x == 0) {
        int v = 1;
        long long tot = 0, nr = 0;
        for (int w = 0; w < (int)((blockDim.x + 31) >> 5); w++) { v = max(v, smax[w]); tot += ssum[w]; nr += snear[w]; }
        v = min(v, kNtCap);
        s.loop->k = 0;
        s.loop->ntmax = v;
        s.loop->near_int += nr;
        s.loop->member_substeps += tot;
        s.loop->loop_iters += v;
        s.loop->outer_steps += 1;
        if (use_cond) cudaGraphSetConditional(h, 1u);
    }
}

// ------------------------------------------------------------------------------------------
// phase A: outflow + dam + bifurcation flux
// ------------------------------------------------------------------------------------------
// CMF_CALC_OUTFLW river/floodplain/mouth discharge and limiter, src/cmf_calc_outflw_mod.F90:44-182
// NADD_adp before sub-step k: the running sum of DT over the sub-steps already done (the same
// additions CMF_DIAG_AVEMAX_ADPSTP performs, so the averages divide by the same value)
__device__ __forceinline__ double nadd_before(int k, double dt) {
    double a = 0.0;
    for (int j = 0; j < k; j++) a = a + dt;
    return a;
}

// Exact shortcuts (the same bits as evaluating every expression):
//  - merge(DOUT, 0, Mask) discards DOUT when Mask is false, so the floodplain flux is evaluated only
//    where its area term passes the mask (most cells carry no floodplain water);
//  - min(a/b, 1) with b > 0 is 1 whenever a >= b (a correctly rounded quotient of a >= b is >= 1),
//    so the limiter rates skip the division in the common case; a NaN a still takes the division.
__device__ __forceinline__ double rate_min1(double a, double b) { return (a >= b) ? 1.0 : dmin(a / b, 1.0); }

// CMF_DIAG_AVEMAX_ADPSTP (src/cmf_calc_diag_mod.F90:104-161) of the sub-step before this one,
// carried into this sub-step's phase A, which reads that sub-step's results anyway: its D2RIVOUT and
// D2FLDOUT are this sub-step's D2*OUT_PRE, its D2RIVDPH and D2STORGE the state it left, its D2DAMINF
// the inflow phase A is about to replace.  Every addition and maximum is the reference's, in its
// order, so each accumulator holds the bits phase C of that sub-step would have stored.  Phase C
// still forms the last sub-step's terms (and the division by NADD), and D2PTHOUT_aAVG, whose
// per-cell path sum phase A does not see.  The accumulators are read after phase A's own stores:
// read at its top they would hold 16 registers across the outflow arithmetic and spill (measured
// slower).
struct DiagPrev {
    double rivout, fldout, outflw, daminf, dinf, mout, mdph, msto;
};
// `daminf` is the previous sub-step's D2DAMINF (phase A captures it before replacing it)
__device__ __forceinline__ DiagPrev diag_carry_load(const Net &n, const State &s, size_t gi, bool first,
                                                    double daminf) {
    DiagPrev p;
    p.rivout = first ? 0.0 : s.a_rivout[gi];
    p.fldout = first ? 0.0 : s.a_fldout[gi];
    p.outflw = first ? 0.0 : s.a_outflw[gi];
    p.mout = first ? 0.0 : s.m_outflw[gi];
    p.mdph = first ? 0.0 : s.m_rivdph[gi];
    p.msto = first ? 0.0 : s.m_storge[gi];
    p.dinf = daminf;
    p.daminf = (first || !n.ldamout) ? 0.0 : s.a_daminf[gi];
    return p;
}
__device__ __forceinline__ bool same_bits(double a, double b) {
    return __double_as_longlong(a) == __double_as_longlong(b);
}
__device__ __forceinline__ void diag_carry_store(const Net &n, const State &s, size_t gi, double DT, bool first,
                                                 const DiagPrev &p, double rivout, double fldout, double rivdph,
                                                 double storge) {
    // a store is skipped when the sub-step leaves the accumulator's bits unchanged (a zero discharge
    // added to a running sum, a maximum that did not move): the array holds the same bits either way
    auto acc = [&](double prev, double *a, double v) {
        const double x = first ? v * DT : prev + v * DT;
        if (first || !same_bits(x, prev)) a[gi] = x;
    };
    const double outflw = rivout + fldout;
    acc(p.rivout, s.a_rivout, rivout);
    acc(p.fldout, s.a_fldout, fldout);
    acc(p.outflw, s.a_outflw, outflw);
    if (n.ldamout) acc(p.daminf, s.a_daminf, p.dinf);
    const double mo = dmax(p.mout, fabs(outflw));
    const double md = dmax(p.mdph, rivdph);
    const double ms = dmax(p.msto, storge);
    if (first || !same_bits(mo, p.mout)) s.m_outflw[gi] = mo;
    if (first || !same_bits(md, p.mdph)) s.m_rivdph[gi] = md;
    if (first || !same_bits(ms, p.msto)) s.m_storge[gi] = ms;
}

template <class Own>
__device__ __forceinline__ void cell_outflow(const Net &n, const State &s, const Own &w, int m, int i, double DT,
                                             const MemberCtl &c, int k, bool split) {
    const size_t base = (size_t)m * n.N, gi = base + i;
    const double gdt = n.pgrv * DT;
    const double rivelv = w.rivelv(i);
    const double rivdph = w.rivdph(gi), rivdph_pre = w.rivdph_pre(gi);
    const double sfc = rivelv + rivdph;
    const double sfc_pre = rivelv + rivdph_pre;
    const double wth = w.rivwth(i);
    const double inv_wth = w.inv_rivwth(i);
    const double man = w.rivman(i);
    const double rivout_pre = w.rivout_pre(gi);
    const double rivout_old = split ? s.rivout_cur[gi] : rivout_pre;
    const double fldout_pre = w.fldout_pre(gi), storge = w.storge(gi);
    const bool carry = n.ldiag && k > 0;   // diagnostics of sub-step k-1 (diag_carry_store)
    bool dinf_taken = false;                 // D2DAMINF of sub-step k-1 read before the dam code replaced it
    double dinf_prev = 0.0;
    double rout, fout = 0.0, rvel;
    if (i < n.R) {
        const int j = w.next(i);
        const size_t gj = base + j;
        const double rj = __ldg(&n.rivelv[j]);
        const double dwn = rj + s.rivdph[gj];
        const double dwn_pre = rj + s.rivdph_pre[gj];
        const double inv_dst = w.inv_nxtdst(i);
        // river
        {
            const double dsfc = dmax(sfc, dwn);
            const double dslp = (sfc - dwn) * inv_dst;
            const double dflw = dsfc - rivelv;
            const double dare = dmax(wth * dflw, 1.E-10);
            const double dflw_pr = dmax(sfc_pre, dwn_pre) - rivelv;
            const double dflw_im = dmax(sqrt(dflw * dflw_pr), 1.E-6);
            const double dout_pr = rivout_pre * inv_wth;
            const double dout = (wth * (dout_pr + (gdt * dflw_im) * dslp))
                              * (1.0 / (1.0 + ((gdt * (man * man)) * fabs(dout_pr)) * pow_depth<7>(dflw_im)));
            const double dvel = rivout_old * (1.0 / dare);
            const bool mask = (dflw_im > CMF_F(1.E-5) && dare > CMF_F(1.E-5));
            rout = mask ? dout : 0.0;
            rvel = mask ? dvel : 0.0;
        }
        if (n.lfldout) {
            const double inv_len = w.inv_rivlen(i);
            double dare = w.fldsto(gi) * inv_len;
            dare = dmax(dare - w.flddph(gi) * wth, 0.0);
            if (dare > 1.E-5) {
                const double elv = w.elevtn(i);
                const double dsfc = dmax(sfc, dwn);
                double dslp = (sfc - dwn) * inv_dst;
                dslp = dmax(-0.005, dmin(0.005, dslp));
                const double dflw = dmax(dsfc - elv, 0.0);
                const double dflw_pr = dmax(sfc_pre, dwn_pre) - elv;
                const double dflw_im = dmax(sqrt(dmax(dflw * dflw_pr, 0.0)), 1.E-6);
                const double flddph_pre = dmax(rivdph_pre - w.rivhgt(i), 0.0);
                double dare_pr = w.fldsto_pre(gi) * inv_len;
                dare_pr = dmax(dare_pr - flddph_pre * wth, 1.E-6);
                const double dare_im = dmax(sqrt(dare * dare_pr), 1.E-6);
                const double dout_pr = fldout_pre;
                const double dout = (dout_pr + (gdt * dare_im) * dslp)
                    * (1.0 / (1.0 + (((gdt * (n.pmanfld * n.pmanfld)) * fabs(dout_pr)) * pow_depth<4>(dflw_im)) * (1.0 / dare_im)));
                fout = (dflw_im > 1.E-5) ? dout : 0.0;
                if (!(fout * rout > 0.0)) fout = 0.0;
            }
        }
        // storage-change limiter (v423), :176-182
        const double dlim = dmax((-rout - fout) * DT, CMF_F(1.E-10));
        const double rate = rate_min1(0.05 * storge, dlim);
        rout = rout * rate;
        fout = fout * rate;
    } else {
        const double inv_dst = 1.0 / n.pdstmth;
        const double dwn = __ldg(&n.dwnelv[i]);
        {
            const double dslp = (sfc - dwn) * inv_dst;
            const double dare = dmax(wth * rivdph, 1.E-10);
            const double dflw_im = dmax(sqrt(rivdph * rivdph_pre), 1.E-6);
            const double dout_pr = rivout_pre * inv_wth;
            const double dout = (wth * (dout_pr + (gdt * dflw_im) * dslp))
                              * (1.0 / (1.0 + ((gdt * (man * man)) * fabs(dout_pr)) * pow_depth<7>(dflw_im)));
            const double dvel = rivout_old * (1.0 / dare);
            const bool mask = (dflw_im > CMF_F(1.E-5) && dare > CMF_F(1.E-5));
            rout = mask ? dout : 0.0;
            rvel = mask ? dvel : 0.0;
        }
        if (n.lfldout) {
            const double inv_len = w.inv_rivlen(i);
            const double dare = dmax(w.fldsto(gi) * inv_len - w.flddph(gi) * wth, 0.0);
            if (dare > CMF_F(1.E-5)) {
                const double elv = w.elevtn(i);
                double dslp = (sfc - dwn) * inv_dst;
                dslp = dmax(-0.005, dmin(0.005, dslp));
                const double dflw = sfc - elv;
                const double dflw_pr = sfc_pre - elv;
                const double dflw_im = dmax(sqrt(dmax(dflw * dflw_pr, 0.0)), 1.E-6);
                const double flddph_pre = dmax(rivdph_pre - w.rivhgt(i), 0.0);
                const double dare_pr = dmax(w.fldsto_pre(gi) * inv_len - flddph_pre * wth, 1.E-6);
                const double dare_im = dmax(sqrt(dare * dare_pr), 1.E-6);
                const double dout_pr = fldout_pre;
                const double dout = (dout_pr + (gdt * dare_im) * dslp)
                    * (1.0 / (1.0 + (((gdt * (n.pmanfld * n.pmanfld)) * fabs(dout_pr)) * pow_depth<4>(dflw_im)) * (1.0 / dare_im)));
                fout = (dflw_im > CMF_F(1.E-5)) ? dout : 0.0;
                if (!(fout * rout > 0.0)) fout = 0.0;
            }
        }
    }
    // reservoir operation, CMF_DAMOUT_CALC (src/cmf_ctrl_damout_mod.F90:316-498)
    if (n.ldamout) {
        const int code = w.i1dam(i);
        if (code > 0) {
            rout = 0.0;
            fout = 0.0;
            double dinf = s.runoff[gi];
            const int d = __ldg(&n.dam_id[i]);
            if (d >= 0) {
                // UPDATE_INFLOW 1b: inflow from the dam's upstream cells, in ascending sequence
                for (int k = __ldg(&n.up_ptr[i]); k < __ldg(&n.up_ptr[i + 1]); k++) {
                    const int j = __ldg(&n.up_idx[k]);
                    const int cj = __ldg(&n.i1dam[j]);
                    if (cj == 10 || cj == 11) {
                        const double fpre = n.lfldout ? s.fldout_pre[base + j] : 0.0;
                        dinf = (dinf + s.rivout_pre[base + j]) + fpre;
                    }
                }
            }
            if (carry) {
                dinf_prev = s.daminf[gi];
                dinf_taken = true;
            }
            s.daminf[gi] = dinf;
            if (code == 10 && i < n.R) {
                // UPDATE_INFLOW 1c: kinematic outflow upstream of a dam
                const int j = __ldg(&n.next[i]);
                const double p23 = CMF_F(2. / 3.);
                double dslope = (__ldg(&n.elevtn[i]) - __ldg(&n.elevtn[j])) * (1.0 / __ldg(&n.nxtdst[i]));
                dslope = dmax(dslope, n.pminslp);
                const double dph = rivdph;
                const double dvel = ((1.0 / man) * sqrt(dslope)) * pow(dph, p23);
                const double darea = wth * dph;
                rvel = dvel;
                rout = dmin(darea * dvel, s.rivsto[gi] / DT);
                const double slope_f = dmin(0.005, dslope);
                const double fdph = s.flddph[gi];
                const double dvel_f = ((1.0 / n.pmanfld) * sqrt(slope_f)) * pow(fdph, p23);
                double dare_f = s.fldsto[gi] * (1.0 / __ldg(&n.rivlen[i]));
                dare_f = dmax(dare_f - fdph * wth, 0.0);
                fout = dmin(dare_f * dvel_f, s.fldsto[gi] / DT);
            }
            if (d >= 0 && __ldg(&n.dam_stat[d]) > 0) {
                const double vol = s.damsto[gi];
                const double qn = __ldg(&n.qn[d]), qf = __ldg(&n.qf[d]), qa = __ldg(&n.qa[d]), con = __ldg(&n.convol[d]), eme = __ldg(&n.emevol[d]);
                double q = 0.0;
                if (n.ldamh22) {
                    const double nor = __ldg(&n.norvol[d]);
                    if (vol <= nor) q = qn * (vol / con);
                    else if (nor < vol && vol <= con) {
                        if (qf <= dinf) q = qn * CMF_F(0.5) + ((vol - nor) / (con - nor)) * (qf - qn);
                        else { const double r = (vol - nor) / (eme - nor); q = qn * CMF_F(0.5) + (r * r) * (qf - qn); }
                    } else if (con < vol && vol < eme) {
                        if (qf <= dinf)
                            q = qf + ((dmax(CMF_F(1.) - __ldg(&n.r_volupa[d]) / CMF_F(0.2), 0.0) * (vol - con)) / (eme - con)) * (dinf - qf);
                        else { const double r = (vol - nor) / (eme - nor); q = qn * CMF_F(0.5) + (r * r) * (qf - qn); }
                    } else q = dmax(dinf, qf);
                } else {
                    const double adj = __ldg(&n.adjvol[d]);
                    if (vol <= con) q = qn * sqrt(vol / con);
                    else if (vol > con && vol <= adj) q = qn + pow((vol - con) / (adj - con), 3.0) * (qa - qn);
                    else if (vol > adj && vol <= eme) {
                        const double t = qa + pow((vol - adj) / (eme - adj), CMF_F(0.1)) * (qf - qa);
                        if (dinf >= qf) q = dmax(qn + ((vol - con) / (eme - con)) * (dinf - qn), t);
                        else q = t;
                    } else if (vol > eme) q = (dinf >= qf) ? dinf : qf;
                }
                q = dmin(dmin(q, vol / DT), (s.rivsto[gi] + s.fldsto[gi]) / DT);
                q = dmax(q, 0.0);
                rout = q;
                fout = 0.0;
            }
        }
    }
    s.rivout_raw[gi] = rout;
    s.fldout_raw[gi] = fout;
    if (carry) {
        const double dinf = dinf_taken ? dinf_prev : (n.ldamout ? s.daminf[gi] : 0.0);
        diag_carry_store(n, s, gi, DT, k == 1, diag_carry_load(n, s, gi, k == 1, dinf), rivout_pre, fldout_pre,
                         rivdph, storge);
    }
    // D2RIVVEL is observed after the last sub-step; its sub-step average is accumulated here
    // (CMF_DIAG_AVEMAX_ADPSTP, src/cmf_calc_diag_mod.F90:104-161) instead of in phase C
    const bool first = (k == 0), last = (k == c.nt - 1);
    if (last) s.rivvel[gi] = rvel;
    if (n.ldiag) {
        const double prev = first ? 0.0 : w.a_rivvel(gi);
        double a = first ? rvel * DT : prev + rvel * DT;
        if (last) {
            a = a / (nadd_before(k, DT) + DT);
            if (n.ldiag_out) s.o_rivvel[gi] = s.o_rivvel[gi] + a * c.dt_def;   // CMF_DIAG_AVEMAX_OUTPUT
        }
        // unchanged bits (a dry cell adds +0): no store needed
        if (first || last || __double_as_longlong(a) != __double_as_longlong(prev)) s.a_rivvel[gi] = a;
    }
}

// CMF_CALC_PTHOUT (src/cmf_calc_pthout_mod.F90:34-94) / CMF_LEVEE_OPT_PTHOUT (src/cmf_ctrl_levee_mod.F90:508-601)
__device__ __forceinline__ double path_flux(double wth, double pre, double gdt, double dflw_im, double dslp, double man,
                                           bool recip) {
    const double dout_pr = recip ? pre * (1.0 / wth) : pre / wth;
    return (wth * (dout_pr + (gdt * dflw_im) * dslp)) / (1.0 + ((gdt * (man * man)) * fabs(dout_pr)) * pow_depth<7>(dflw_im));
}

__device__ __forceinline__ void path_outflow(const Net &n, const State &s, int m, int p, double DT) {
    const int P = n.P, Lp = n.Lp;
    const size_t pb = (size_t)m * Lp * P;
    const size_t base = (size_t)m * n.N;
    const double gdt = n.pgrv * DT;
    const int skip = __ldg(&n.pth_skip[p]);
    double sum = 0.0;
    double flw[8];
    const bool skipped = n.llevee ? (skip & 2) : (skip & 1);
    if (skipped) {
        for (int l = 0; l < Lp; l++) s.pthflw_raw[pb + (size_t)l * P + p] = 0.0;
        s.pthsum_raw[(size_t)m * P + p] = 0.0;
        return;
    }
    const int u = __ldg(&n.pth_up[p]), d = __ldg(&n.pth_dn[p]);
    const double su = __ldg(&n.rivelv[u]) + s.rivdph[base + u], sd = __ldg(&n.rivelv[d]) + s.rivdph[base + d];
    const double spu = __ldg(&n.rivelv[u]) + s.rivdph_pre[base + u], spd = __ldg(&n.rivelv[d]) + s.rivdph_pre[base + d];
    double dslp = (su - sd) / __ldg(&n.pth_dst[p]);
    dslp = dmax(-0.005, dmin(0.005, dslp));
    if (!n.llevee) {
        for (int l = 0; l < Lp; l++) {
            const size_t o = (size_t)l * P + p;
            const double elv = __ldg(&n.pth_elv[o]);
            const double dflw = dmax(dmax(su, sd) - elv, 0.0);
            const double dflw_pr = dmax(dmax(spu, spd) - elv, 0.0);
            double dflw_im = sqrt(dflw * dflw_pr);
            dflw_im = dmax(dflw_im, sqrt(dflw * 0.01));
            const double f = (dflw_im > 1.E-5) ? path_flux(__ldg(&n.pth_wth[o]), s.pthflw_pre[pb + o], gdt, dflw_im, dslp, __ldg(&n.pth_man[l]), false) : 0.0;
            if (l < 8) flw[l] = f;
            s.pthflw_raw[pb + o] = f;
        }
    } else {
        // level 1: river channel, semi-implicit depth
        {
            const double elv = __ldg(&n.pth_elv[p]);
            const double dflw = dmax(dmax(su, sd) - elv, 0.0);
            const double dflw_pr = dmax(dmax(spu, spd) - elv, 0.0);
            double dflw_im = sqrt(dflw * dflw_pr);
            if (dflw_im <= 0.0) dflw_im = dflw;
            const double f = (dflw_im > 1.E-5) ? path_flux(__ldg(&n.pth_wth[p]), s.pthflw_pre[pb + p], gdt, dflw_im, dslp, __ldg(&n.pth_man[0]), false) : 0.0;
            flw[0] = f;
            s.pthflw_raw[pb + p] = f;
        }
        if (Lp > 1) {
            const int lu = __ldg(&n.lev_id[u]), ld = __ldg(&n.lev_id[d]);
            double slu = su, sld = sd;
            if (lu >= 0 && __ldg(&n.levfrc[lu]) < 1.0) slu = dmin(__ldg(&n.elevtn[u]) + s.levdph[base + u], su);
            if (ld >= 0 && __ldg(&n.levfrc[ld]) < 1.0) sld = dmin(__ldg(&n.elevtn[d]) + s.levdph[base + d], sd);
            for (int l = 1; l < Lp; l++) {
                const size_t o = (size_t)l * P + p;
                const double dflw = dmax(dmax(slu, sld) - __ldg(&n.pth_elv[o]), 0.0);
                const double f = (dflw > 1.E-5) ? path_flux(__ldg(&n.pth_wth[o]), s.pthflw_pre[pb + o], gdt, dflw, dslp, __ldg(&n.pth_man[l]), true) : 0.0;
                if (l < 8) flw[l] = f;
                s.pthflw_raw[pb + o] = f;
            }
        }
    }
    for (int l = 0; l < Lp; l++) sum = sum + (l < 8 ? flw[l] : s.pthflw_raw[pb + (size_t)l * P + p]);
    if (sum != 0.0) {
        const double rate = rate_min1(0.05 * dmin(s.storge[base + u], s.storge[base + d]), fabs(sum * DT));
        for (int l = 0; l < Lp; l++) {
            const size_t o = pb + (size_t)l * P + p;
            s.pthflw_raw[o] = (l < 8 ? flw[l] : s.pthflw_raw[o]) * rate;
        }
        sum = sum * rate;
    }
    s.pthsum_raw[(size_t)m * P + p] = sum;
}

template <int MinBlocks>
__global__ void __launch_bounds__(kCellThreads, MinBlocks) k_flux(Net n, State s, int ncell_blocks) {
    const int m = blockIdx.y;
    const MemberCtl &c = s.ctl[m];
    const int k = s.loop->k;
    if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) s.loop->kcur = k;   // for k_rate and k_store
    if (k >= c.nt) return;
    const double DT = c.dt;
    if ((int)blockIdx.x < ncell_blocks) {
        const int i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i < n.N) cell_outflow(n, s, OwnG{n, s}, m, i, DT, c, k, s.loop->split != 0);
    } else {
        const int p = (blockIdx.x - ncell_blocks) * blockDim.x + threadIdx.x;
        if (p < n.P) path_outflow(n, s, m, p, DT);
    }
}

// ------------------------------------------------------------------------------------------
// phase B: P2STOOUT and D2RATE, src/cmf_calc_outflw_mod.F90:410-451
// ------------------------------------------------------------------------------------------
template <class Own>
__device__ __forceinline__ void cell_rate(const Net &n, const State &s, const Own &w, int m, int i, double DT) {
    const size_t base = (size_t)m * n.N, gi = base + i;
    double so = dmax(w.rivout_raw(gi), 0.0) + dmax(w.fldout_raw(gi), 0.0);
    // the CSR walk: at full occupancy the slot table's 16 B per cell cost more than its saved round
    const int u1 = w.up_hi(i);
    for (int k = w.up_lo(i); k < u1; k++) {
        const int j = __ldg(&n.up_idx[k]);
        so = (so + dmax(-s.rivout_raw[base + j], 0.0)) + dmax(-s.fldout_raw[base + j], 0.0);
    }
    so = so * DT;
    if (n.lpthout) {
        const double *sum = s.pthsum_raw + (size_t)m * n.P;
        for (int k = __ldg(&n.pout_ptr[i]); k < __ldg(&n.pout_ptr[i + 1]); k++) so = so + dmax(sum[__ldg(&n.pout_idx[k])], 0.0) * DT;
        for (int k = __ldg(&n.pinf_ptr[i]); k < __ldg(&n.pinf_ptr[i + 1]); k++) so = so + dmax(-sum[__ldg(&n.pinf_idx[k])], 0.0) * DT;
    }
    const double dout = dmax(so, 1.E-10);
    const double dsto = w.rivsto(gi) + w.fldsto(gi);
    s.rate[gi] = rate_min1(dsto, dout);
}

// advance != 0: block (0,0) also moves the loop counter to the next sub-step and sets the WHILE
// condition (every k_flux block has read the counter; k_rate and k_store read `kcur`)
__global__ void k_rate(Net n, State s, int advance, cudaGraphConditionalHandle h, int use_cond) {
    const int m = blockIdx.y;
    const MemberCtl &c = s.ctl[m];
    const int k = s.loop->kcur;
    if (advance && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) {
        const int kn = k + 1;
        s.loop->k = kn;
        s.loop->split = 0;
        if (use_cond) cudaGraphSetConditional(h, (kn < s.loop->ntmax && kn < kNtCap) ? 1u : 0u);
    }
    if (k >= c.nt) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n.N) return;
    cell_rate(n, s, OwnG{n, s}, m, i, c.dt);
}

// ------------------------------------------------------------------------------------------
// phase C: rescale + inflow + dam balance + VARS_PRE + STONXT + stage + diagnostics
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ double scaled_pathsum(const Net &n, const double *sum_raw, const double *rate_m, int p) {
    const double v = sum_raw[p];
    if (__ldg(&n.pth_skip[p]) & 1) return v;
    return v >= 0.0 ? v * rate_m[__ldg(&n.pth_up[p])] : v * rate_m[__ldg(&n.pth_dn[p])];
}

// bifurcation paths in phase C: LSPAMAT path rescale (:494-517), CALC_VARS_PRE copy, diagnostics
__device__ __forceinline__ void path_rescale(const Net &n, const State &s, int m, int p, double DT, bool first, bool last,
                                             double nadd, double dt_def) {
    const int P = n.P, Lp = n.Lp;
    const size_t base = (size_t)m * n.N;
    const size_t pb = (size_t)m * Lp * P;
    const double *rate_m = s.rate + base;
    const bool sk = __ldg(&n.pth_skip[p]) & 1;
    const int u = __ldg(&n.pth_up[p]), d = __ldg(&n.pth_dn[p]);
    double asum = 0.0;
    for (int l = 0; l < Lp; l++) {
        const size_t o = pb + (size_t)l * P + p;
        double f = s.pthflw_raw[o];
        if (!sk) f = (f >= 0.0) ? f * rate_m[u] : f * rate_m[d];
        s.pthflw_pre[o] = f;
        if (n.ldiag) {
            double a = first ? f * DT : s.a_pthflw[o] + f * DT;
            if (last) {
                a = a / (nadd + DT);
                asum = asum + a;
                if (n.ldiag_out) s.o_pthflw[o] = s.o_pthflw[o] + a * dt_def;
            }
            s.a_pthflw[o] = a;
        }
    }
    s.pthsum[(size_t)m * P + p] = scaled_pathsum(n, s.pthsum_raw + (size_t)m * P, rate_m, p);
    if (n.ldiag && last) s.a_pthsum[(size_t)m * P + p] = asum;
}

// one cell in phase C; `bput(k, v)` receives the last sub-step's budget term k
template <class Own, class BPut>
__device__ __forceinline__ void cell_store(const Net &n, const State &s, const Own &w, int m, int i, double DT,
                                           bool first, bool last, double nadd, const MemberCtl &c, BPut bput) {
    const size_t base = (size_t)m * n.N;
    const size_t gi = base + i;
    const double *rate_m = s.rate + base;
    // the cell's own state is read up front, before anything is stored: in the compiler's view a
    // store may alias any later load of another state array and would hold that load back
    const double rate_i = w.rate(gi);
    double rout = w.rivout_raw(gi), fout = w.fldout_raw(gi);
    const double runoff = w.runoff(gi);
    const double rivsto0 = w.rivsto(gi), fldsto0 = w.fldsto(gi), rivdph0 = w.rivdph(gi);
    const double frc = w.fldfrc(gi);
    const double levsto = n.llevee ? w.levsto(gi) : 0.0;
    // own outflow after the LSPAMAT rescale (:456-473)
    if (i < n.R) {
        const double r = (rout > 0.0) ? rate_i : rate_m[w.next(i)];
        rout = rout * r;
        fout = fout * r;
    } else {
        rout = rout * rate_i;
        fout = fout * rate_i;
    }
    // inflow from the upstream cells, rescaled on the fly (:481-489); next(j) == i
    double rinf = 0.0, finf = 0.0;
    for_each_upstream(n, w, i, [&](int j) {
        const double rj = s.rivout_raw[base + j], fj = s.fldout_raw[base + j];
        const double r = (rj > 0.0) ? rate_m[j] : rate_i;
        rinf = rinf + rj * r;
        finf = finf + fj * r;
    });
    double pout = 0.0;
    bool has_path = false;
    if (n.lpthout) {
        const double *sum = s.pthsum_raw + (size_t)m * n.P;
        const int o0 = __ldg(&n.pout_ptr[i]), o1 = __ldg(&n.pout_ptr[i + 1]), f0 = __ldg(&n.pinf_ptr[i]), f1 = __ldg(&n.pinf_ptr[i + 1]);
        has_path = (o1 > o0) || (f1 > f0);
        for (int k = o0; k < o1; k++) pout = pout + scaled_pathsum(n, sum, rate_m, __ldg(&n.pout_idx[k]));
        for (int k = f0; k < f1; k++) pout = pout - scaled_pathsum(n, sum, rate_m, __ldg(&n.pinf_idx[k]));
    }
    // CMF_DAMOUT_WATBAL, src/cmf_ctrl_damout_mod.F90:516-535 (the new dam storage is stored below)
    double dmiss = 0.0, damsto1 = 0.0;
    const int dam = n.ldamout ? __ldg(&n.dam_id[i]) : -1;
    if (dam >= 0) {
        const double inflow = (rinf + finf) + runoff;
        const double outflw = rout + fout;
        const double s0 = s.damsto[gi];
        damsto1 = (s0 + inflow * DT) - outflw * DT;
        dmiss = ((s0 - damsto1) + inflow * DT) - outflw * DT;
    }
    bput(11, dmiss);
    // CMF_CALC_STONXT, src/cmf_calc_stonxt_mod.F90:53-100
    bput(0, rivsto0 + fldsto0);
    bput(3, rinf * DT + finf * DT);
    bput(4, (rout * DT + fout * DT) + pout * DT);
    double rs = (rivsto0 + rinf * DT) - rout * DT;
    double fs = fldsto0;
    if (rs < 0.0) { fs = fs + rs; rs = 0.0; }
    fs = ((fs + finf * DT) - fout * DT) - pout * DT;
    if (fs < 0.0) { rs = dmax(rs + fs, 0.0); fs = 0.0; }
    bput(1, rs + fs);
    const double outflw = rout + fout;
    rs = rs + (runoff * (1.0 - frc)) * DT;       // D2GDWRTN is zero without groundwater delay
    fs = fs + (runoff * frc) * DT;
    bput(2, n.llevee ? (rs + fs) + levsto : rs + fs);
    // stage scheme, :125
    const StageOut o = n.llevee ? stage_levee(n, w, i, rs, fs, levsto) : stage_def(n, w, i, rs, fs);
    // CALC_VARS_PRE, src/cmf_ctrl_physics_mod.F90:254-277, and the dam storage
    s.rivout_pre[gi] = rout;
    s.fldout_pre[gi] = fout;
    s.rivdph_pre[gi] = rivdph0;
    s.fldsto_pre[gi] = fldsto0;
    if (dam >= 0) s.damsto[gi] = damsto1;
    // CMF_CheckNanB-style probe (src/cmf_utils_mod.F90:807-815) on the new storage: a NaN or
    // infinite runoff or state surfaces as a positive status instead of a silent NaN state
    if (!isfinite((o.rivsto + o.fldsto) + o.levsto)) s.ctl[m].err = kErrNonFinite;
    store_stage(n, s, gi, i, o, last);
    bput(5, n.llevee ? (rs + fs) + levsto : rs + fs);
    bput(6, n.llevee ? (o.rivsto + o.fldsto) + o.levsto : o.rivsto + o.fldsto);
    bput(7, o.rivsto);
    bput(8, o.fldsto);
    bput(9, o.fldare);
    bput(10, o.levsto);
    if (last) {   // diagnostics read by nothing inside the sub-step loop
        s.rivinf[gi] = rinf;
        s.fldinf[gi] = finf;
        s.pthout[gi] = pout;
        s.outflw[gi] = outflw;
    }
    // CMF_DIAG_AVEMAX_ADPSTP / GETAVE_ADPSTP, src/cmf_calc_diag_mod.F90:104-221.  The sub-steps
    // before the last one are accumulated by the next sub-step's phase A (diag_carry_store), except
    // D2PTHOUT_aAVG: D2PTHINF is never written by the reference (always 0), and a cell without
    // bifurcation channels adds +0 every sub-step, so its average (and output average) stays at the
    // +0 the arrays were created with; cells with channels accumulate it here every sub-step.
    if (n.ldiag && (last || has_path)) {
        const double na = nadd + DT;
        // CMF_DIAG_AVEMAX_OUTPUT (src/cmf_calc_diag_mod.F90:272-318) on the last sub-step: the
        // output interval accumulates the finished sub-step average times DT_DEF
        const bool out = last && n.ldiag_out;
        const double ddef = c.dt_def;
        auto acc = [&](double prev, double *a, double *oa, double v) {
            double x = first ? v * DT : prev + v * DT;
            if (last) x = x / na;
            if (first || last || !same_bits(x, prev)) a[gi] = x;
            if (out) oa[gi] = oa[gi] + x * ddef;
        };
        if (has_path) acc(first ? 0.0 : w.a_pthout(gi), s.a_pthout, s.o_pthout, pout);
        if (last) {
            // every previous accumulator is read before the first of them is stored
            const double pro = first ? 0.0 : w.a_rivout(gi), pfo = first ? 0.0 : w.a_fldout(gi);
            const double pof = first ? 0.0 : w.a_outflw(gi);
            const double pmo = first ? 0.0 : w.m_outflw(gi), pmd = first ? 0.0 : w.m_rivdph(gi);
            const double pms = first ? 0.0 : w.m_storge(gi);
            const double dinf = n.ldamout ? s.daminf[gi] : 0.0, pdi = (first || !n.ldamout) ? 0.0 : s.a_daminf[gi];
            acc(pro, s.a_rivout, s.o_rivout, rout);
            acc(pfo, s.a_fldout, s.o_fldout, fout);
            acc(pof, s.a_outflw, s.o_outflw, outflw);
            // runoff and DT are constant over the outer step: the same running sum of
            // runoff*DT the accumulator would hold, rebuilt in registers on the last sub-step
            const double rdt = runoff * DT;
            double a = rdt;
            for (int k = 1; k < c.nt; k++) a = a + rdt;
            a = a / na;
            s.a_runoff[gi] = a;
            if (out) s.o_runoff[gi] = s.o_runoff[gi] + a * ddef;
            if (n.ldamout) acc(pdi, s.a_daminf, s.o_daminf, dinf);
            const double stg = n.llevee ? (o.rivsto + o.fldsto) + o.levsto : o.rivsto + o.fldsto;
            const double mo = dmax(pmo, fabs(outflw));
            const double md = dmax(pmd, o.rivdph);
            const double ms = dmax(pms, stg);
            s.m_outflw[gi] = mo;
            s.m_rivdph[gi] = md;
            s.m_storge[gi] = ms;
            if (out) {
                s.om_outflw[gi] = dmax(s.om_outflw[gi], fabs(mo));
                s.om_rivdph[gi] = dmax(s.om_rivdph[gi], md);
                s.om_storge[gi] = dmax(s.om_storge[gi], ms);
            }
        }
    }
}

// Budget partials of the last sub-step (the only one the caller observes), one per warp of 32
// consecutive cells: a fixed butterfly over the warp, so the partials -- and the budgets k_budget
// sums from them in a fixed order -- are the same whatever block size or schedule ran the cells.
// Layout [m][k][warp] for a coalesced final reduction.  Every lane of the warp calls it.
__device__ __forceinline__ void warp_budget_partials(const State &s, int m, int warp, int nwarps, double (&b)[kBudgets]) {
#pragma unroll
    for (int k = 0; k < kBudgets; k++)
        for (int o = 16; o > 0; o >>= 1) b[k] = b[k] + __shfl_down_sync(0xffffffffu, b[k], o);
    if ((threadIdx.x & 31) == 0 && warp < nwarps) {     // warps past the last cell hold no cells
        double *dst = s.partials + (size_t)m * kBudgets * nwarps + warp;
#pragma unroll
        for (int k = 0; k < kBudgets; k++) dst[(size_t)k * nwarps] = b[k];
    }
}
__host__ __device__ inline int budget_warps(int N) { return (N + 31) / 32; }

template <int MinBlocks>
__global__ void __launch_bounds__(kCellThreads, MinBlocks) k_store(Net n, State s, int ncell_blocks) {
    const int m = blockIdx.y;
    const MemberCtl &c = s.ctl[m];
    const int kk = s.loop->kcur;
    const bool active = kk < c.nt;
    if (!active) return;   // uniform per block (blockIdx.y), no barrier is skipped divergently
    const double DT = c.dt;
    const bool first = (kk == 0);
    const bool last = (kk == c.nt - 1);
    const double nadd = last ? nadd_before(kk, DT) : 0.0;   // only the averages of the last sub-step need it
    if ((int)blockIdx.x >= ncell_blocks) {
        const int p = (blockIdx.x - ncell_blocks) * blockDim.x + threadIdx.x;
        if (p < n.P) path_rescale(n, s, m, p, DT, first, last, nadd, c.dt_def);
        return;
    }
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    // budget terms of the last sub-step go to shared memory where they are computed (dynamic
    // shared memory, kBudgets x blockDim doubles), so they hold no registers across the stage scheme
    extern __shared__ double sbud[];
    double *bt = sbud + threadIdx.x;
    const int bstride = blockDim.x;
    auto bput = [&](int k, double v) { if (last) bt[k * bstride] = v; };
    if (last && i >= n.N)
#pragma unroll
        for (int k = 0; k < kBudgets; k++) bt[k * bstride] = 0.0;
    if (i < n.N) cell_store(n, s, OwnG{n, s}, m, i, DT, first, last, nadd, c, bput);
    if (last) {
        double b[kBudgets];
#pragma unroll
        for (int k = 0; k < kBudgets; k++) b[k] = bt[k * bstride];
        warp_budget_partials(s, m, i >> 5, budget_warps(n.N), b);
    }
}

// ------------------------------------------------------------------------------------------
// k_budget: after the sub-step loop, the budgets of every member's last sub-step
// ------------------------------------------------------------------------------------------
// grid (members, kBudgets), kBudgetThreads threads: block (m, k) reduces budget k of member m over
// the warp partials its last sub-step wrote -- thread t sums partials t, t+T, ... in order, then a
// fixed warp tree and a fixed tree over the warps: the same sums whatever the timing
constexpr int kBudgetThreads = 256;
__global__ void __launch_bounds__(kBudgetThreads) k_budget(Net n, State s) {
    const int m = blockIdx.x, k = blockIdx.y;
    if (s.ctl[m].nt < 1) return;                        // refused step (NT cap): no sub-step ran
    const int nw = budget_warps(n.N);
    const double *src = s.partials + ((size_t)m * kBudgets + k) * nw;
    double x = 0.0;
    for (int b = threadIdx.x; b < nw; b += kBudgetThreads) x = x + src[b];
    for (int o = 16; o > 0; o >>= 1) x = x + __shfl_down_sync(0xffffffffu, x, o);
    __shared__ double w[kBudgetThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) w[warp] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int j = 0; j < kBudgetThreads / 32; j++) t = t + w[j];
        s.ctl[m].budget[k] = t;
        if (k == 0 && n.ldiag_out) s.o_nadd[m] = s.o_nadd[m] + s.ctl[m].dt_def;   // NADD_out = NADD_out + DT
    }
}

// CMF_DIAG_GETAVE_OUTPUT (src/cmf_calc_diag_mod.F90:324-356): the output-interval sums divided by
// NADD_out in place (maxima untouched).  Cells on blocks [0, ncell_blocks), path levels after them.
__global__ void k_diag_getave_output(Net n, State s, int ncell_blocks) {
    const int m = blockIdx.y;
    const double na = s.o_nadd[m];
    if ((int)blockIdx.x < ncell_blocks) {
        const int i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= n.N) return;
        const size_t gi = (size_t)m * n.N + i;
        s.o_rivout[gi] = s.o_rivout[gi] / na;
        s.o_fldout[gi] = s.o_fldout[gi] / na;
        s.o_outflw[gi] = s.o_outflw[gi] / na;
        s.o_rivvel[gi] = s.o_rivvel[gi] / na;
        s.o_pthout[gi] = s.o_pthout[gi] / na;
        s.o_runoff[gi] = s.o_runoff[gi] / na;
        if (n.ldamout) s.o_daminf[gi] = s.o_daminf[gi] / na;
    } else {
        const int q = (blockIdx.x - ncell_blocks) * blockDim.x + threadIdx.x;
        const size_t PL = (size_t)n.P * n.Lp;
        if ((size_t)q >= PL) return;
        const size_t o = (size_t)m * PL + q;
        s.o_pthflw[o] = s.o_pthflw[o] / na;
    }
}

// ------------------------------------------------------------------------------------------
// k_outpre: CMF_CALC_OUTPRE (src/cmf_opt_outflw_mod.F90:308-421) -- previous-step discharge by the
// diffusive (Manning) wave, after a storage-only restart and the stage scheme.  Cells on blocks
// [0, ncell_blocks), bifurcation paths on the blocks after them; the downstream surface elevation
// is recomputed from the depth (the same sum the reference stores in D2SFCELV first).
// ------------------------------------------------------------------------------------------
__global__ void k_outpre(Net n, State s, int ncell_blocks) {
    const int m = blockIdx.y;
    const size_t base = (size_t)m * n.N;
    const double p23 = CMF_F(2. / 3.);
    if ((int)blockIdx.x < ncell_blocks) {
        const int i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= n.N) return;
        const size_t gi = base + i;
        const double rivdph = s.rivdph[gi];
        const double sfc = __ldg(&n.rivelv[i]) + rivdph;
        s.sfcelv[gi] = sfc;
        s.rivdph_pre[gi] = rivdph;
        double dslope, dsfcmax, dflw;
        if (i < n.R) {
            const int j = __ldg(&n.next[i]);
            const double sfcj = __ldg(&n.rivelv[j]) + s.rivdph[base + j];
            dsfcmax = dmax(sfc, sfcj);
            dslope = (sfc - sfcj) * (1.0 / __ldg(&n.nxtdst[i]));
            dflw = dsfcmax - __ldg(&n.rivelv[i]);
        } else {
            dsfcmax = sfc;
            dslope = (sfc - __ldg(&n.dwnelv[i])) * (1.0 / n.pdstmth);
            dflw = rivdph;
        }
        const double dslope_f = dmax(-0.005, dmin(0.005, dslope));
        const double darea = __ldg(&n.rivwth[i]) * dflw;
        double rout = 0.0;
        if (darea > CMF_F(1.E-5)) {
            rout = darea * (((1.0 / __ldg(&n.rivman[i])) * pow(dflw, p23)) * sqrt(fabs(dslope)));
            if (dslope < 0.0) rout = -rout;
        }
        const double dflw_f = dmax(dsfcmax - __ldg(&n.elevtn[i]), 0.0);
        double dare_f = s.fldsto[gi] * (1.0 / __ldg(&n.rivlen[i]));
        dare_f = dmax(dare_f - s.flddph[gi] * __ldg(&n.rivwth[i]), 0.0);
        double fout = 0.0;
        if (dare_f > CMF_F(1.E-5)) {
            fout = dare_f * (((1.0 / n.pmanfld) * pow(dflw_f, p23)) * sqrt(fabs(dslope_f)));
            if (dslope_f < 0.0) fout = -fout;
        }
        s.rivout_pre[gi] = rout;
        s.fldout_pre[gi] = n.lfldout ? fout : 0.0;
    } else {
        const int p = (blockIdx.x - ncell_blocks) * blockDim.x + threadIdx.x;
        if (p >= n.P) return;
        const int u = __ldg(&n.pth_up[p]), d = __ldg(&n.pth_dn[p]);
        if (u < 0 || d < 0) return;                    // path leaves the domain
        const size_t pb = (size_t)m * n.Lp * n.P;
        const double su = __ldg(&n.rivelv[u]) + s.rivdph[base + u], sd = __ldg(&n.rivelv[d]) + s.rivdph[base + d];
        const double dslope = (su - sd) * (1.0 / __ldg(&n.pth_dst[p]));
        for (int l = 0; l < n.Lp; l++) {
            const size_t o = (size_t)l * n.P + p;
            const double dflw = dmax(dmax(su, sd) - __ldg(&n.pth_elv[o]), 0.0);
            double f = 0.0;
            if (dflw > CMF_F(1.E-5)) {
                f = (__ldg(&n.pth_wth[o]) * dflw) * (((1.0 / __ldg(&n.pth_man[l])) * pow(dflw, p23)) * sqrt(fabs(dslope)));
                if (dslope < 0.0) f = -f;
            }
            s.pthflw_pre[pb + o] = f;
        }
    }
}

// ------------------------------------------------------------------------------------------
// k_runoff_map: CMF_FORCING_PUT on the device (src/cmf_ctrl_forcing_mod.F90:716-831) for every
// member: the runoff field PBUFF(NXIN,NYIN) of member m is grid[m][NYIN][NXIN] (fp64, or fp32
// promoted exactly).  linterp: ROFF_INTERP over the input matrix (inpx/inpy/inpa [INPN][N]);
// else CONV_RESOL at (inpx, inpy) = (I1SEQX, I1SEQY) with the cell area.  clean applies
// CMF_FORCING_GET's NaN -> RMIS and max(., 0) (:486-494) to every value read.
// ------------------------------------------------------------------------------------------
struct RunoffMap {
    int linterp, nxin, nyin, inpn, clean;
    const int *__restrict__ inpx, *__restrict__ inpy;
    const double *__restrict__ inpa;
    double drofunit;
};

__global__ void k_runoff_map(Net n, State s, RunoffMap r, const double *__restrict__ gridd, const float *__restrict__ gridf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n.N) return;
    const int m = blockIdx.y;
    const size_t g0 = (size_t)m * r.nxin * r.nyin;
    const double rmis = CMF_F(1.E20);
    auto val = [&](int ix, int iy) -> double {
        const size_t k = g0 + (size_t)(iy - 1) * r.nxin + (ix - 1);
        double v = gridd ? gridd[k] : (double)gridf[k];
        if (r.clean) {
            if (isnan(v)) v = rmis;
            v = dmax(v, 0.0);
        }
        return v;
    };
    double out = 0.0;
    if (r.linterp) {
        for (int k = 0; k < r.inpn; k++) {
            const int ix = r.inpx[(size_t)k * n.N + i], iy = r.inpy[(size_t)k * n.N + i];
            if (ix > 0) {
                if (ix > r.nxin || iy > r.nyin || iy < 1) continue;   // the reference logs and skips
                const double v = val(ix, iy);
                if (v != rmis) out = out + (v * r.inpa[(size_t)k * n.N + i]) / r.drofunit;
            }
        }
    } else {
        const double v = val(r.inpx[i], r.inpy[i]);
        if (v != rmis) out = dmax((v * __ldg(&n.grarea[i])) / r.drofunit, 0.0);
    }
    s.runoff[(size_t)m * n.N + i] = out;
}

// k_boundary: CMF_BOUNDARY_UPDATE (src/cmf_ctrl_boundary_mod.F90:267-304): downstream boundary
// elevation D2DWNELV = D2ELEVTN (+ D2MEANSL) (+ D2SEALEV); only the mouths read it.
__global__ void k_boundary(int N, const double *__restrict__ elevtn, const double *__restrict__ meansl,
                           const double *__restrict__ sealev, double *dwnelv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double v = meansl ? elevtn[i] + meansl[i] : elevtn[i];
    if (sealev) v = v + sealev[i];
    dwnelv[i] = v;
}

}  // namespace cmf
