// cmf_engine.cu -- device context, graph construction, autotuner and the C ABI of cmf_gpu.h.
//
// A context owns the device copy of one river network (maps, CSR tables) and the state of
// `nmembers` ensemble members.  One outer step is one CUDA graph launch:
//   k_stage -> k_ntdt -> while (k < NTmax) { k_flux -> k_rate -> k_store } -> k_budget
// The loop is a conditional WHILE node whose condition the device sets (k_ntdt, k_rate), so the
// adaptive sub-step count never travels to the host.  launch_mode 1 replaces the conditional node
// by a host loop (reads NTmax back), which tests use to cross-check the graph path.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <map>
#include <mutex>
#include <tuple>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cmf_gpu.h"
#include "cmf_kernels.cuh"
#include "cmf_persist.cuh"

namespace {

thread_local std::string g_last_error;

int set_err(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

#define CUDA_TRY(expr)                                                                          \
    do {                                                                                        \
        cudaError_t e_ = (expr);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            return set_err(CMF_E_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_));     \
    } while (0)

constexpr int kImis = -9999;

}  // namespace

// Launch schedule of one outer step: the graph of phase kernels with a block size per kernel and
// an occupancy profile (wide: more resident warps, fewer registers; small: fewer spills), or the
// persistent kernel.  Every schedule computes the same bits (no atomics on state, budgets from
// per-warp partials), so the autotuner may switch between them at any outer step.
struct Sched {
    int mode = 0;               // 0 graph of phase kernels, 2 persistent kernel
    int bf = 256, br = 256, bs = 256;
    int prof = 0;               // 0 wide, 1 small
    bool operator==(const Sched &o) const {
        return mode == o.mode && bf == o.bf && br == o.br && bs == o.bs && prof == o.prof;
    }
};
inline int nblk(int n, int b) { return n > 0 ? (n + b - 1) / b : 0; }

// Online autotuner: after `warm` outer steps on the starting schedule (so that the state is
// spun up: flooded cells, levees and dams active), every candidate runs `reps` real outer steps,
// timed with CUDA events and normalised by the sub-step count; the fastest is kept for good and
// cached per network shape for later contexts.  The trajectory is not affected (same bits).
struct Tuner {
    bool active = false;
    int warm = 0, reps = 2, cand = 0, rep = 0;
    std::vector<Sched> cands;
    std::vector<double> ms, sub;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    long long iters0 = 0;
    double best_us = 0.0, worst_us = 0.0;
    int timed = 0;              // candidates timed (0: the schedule was fixed by the caller or the cache)
};

struct cmf_gpu_ctx {
    cmf_dims dims{};
    cmf_params params{};
    cmf_opts opts{};
    cmf::Net net{};
    cmf::State st{};
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<void *> allocs;
    Sched sched;                // the launch schedule of the outer step
    int persist_grid = 0;       // co-resident CTAs of the persistent kernel (0: it cannot run here)
    bool l2_window = false;     // the hot maps sit under a persisting L2 access-policy window
    bool persist = false;       // outer steps run as one persistent cooperative launch
    Tuner tune;                 // online autotuner state
    int nlev = 0, ndam_placed = 0;
    size_t E = 0;
    // graph
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraphConditionalHandle cond{};
    double dt_def_dev = -1.0;
    // pipelined host I/O (created on first use): copy streams for uploads (io) and read-backs
    // (io_out; separate, so that an upload never queues behind a read-back that waits for a step),
    // the runoff staging buffer, the staging of diagnostics read back while the next step runs,
    // and their events
    cudaStream_t io = nullptr, io_out = nullptr;
    cudaEvent_t ev_in = nullptr, ev_stage_free = nullptr, ev_out_staged = nullptr, ev_out_done = nullptr;
    double *rstage = nullptr;
    bool in_pending = false;    // a runoff field waits in rstage for the next advance
    // outer steps launched by advance_async and not yet waited for (at most two): each launch
    // copies the control blocks after its step into its own pinned ring slot
    int inflight = 0, head = 0;
    cmf::MemberCtl *ring[2] = {nullptr, nullptr};
    cudaEvent_t ev_ctl[2] = {nullptr, nullptr};
    std::vector<double *> ostage;   // per diagnostic field (DIAG order), allocated on first request
    int64_t launches = 0;
    // host staging for the per-member control block
    std::vector<cmf::MemberCtl> hctl;
    cmf::MemberCtl *hctl_pin = nullptr;   // pinned landing buffer of the per-step read-back
    // sea-level boundary inputs (allocated on first use)
    double *bnd_sealev = nullptr, *bnd_meansl = nullptr;
    // runoff interpolation (input matrix or nearest cell) and the staging of runoff fields
    cmf::RunoffMap rmap{};
    bool rmap_set = false;
    void *rgrid = nullptr;
    size_t rgrid_bytes = 0;

    template <class T>
    int alloc(T **p, size_t n) {
        void *q = nullptr;
        if (n == 0) n = 1;
        CUDA_TRY(cudaMalloc(&q, n * sizeof(T)));
        CUDA_TRY(cudaMemsetAsync(q, 0, n * sizeof(T), stream));
        allocs.push_back(q);
        *p = static_cast<T *>(q);
        return CMF_OK;
    }
    template <class P, class T>
    int upload(P *p, const std::vector<T> &h) {
        T *q = nullptr;
        int rc = alloc(&q, h.size());
        if (rc) return rc;
        if (!h.empty()) CUDA_TRY(cudaMemcpyAsync(q, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, stream));
        *p = q;
        return CMF_OK;
    }
    template <class P, class T>
    int upload_raw(P *p, const T *h, size_t n) {
        T *q = nullptr;
        int rc = alloc(&q, n);
        if (rc) return rc;
        if (h && n) CUDA_TRY(cudaMemcpyAsync(q, h, n * sizeof(T), cudaMemcpyHostToDevice, stream));
        *p = q;
        return CMF_OK;
    }
};

// Several contexts (regional domains of uneven size, each with its own members) advanced by ONE
// graph launch per coupling step: every context's outer step is an independent branch of the
// batch graph with its own WHILE node, so each domain loops over its own sub-step count while the
// branches run concurrently on the device.
struct cmf_gpu_batch {
    std::vector<cmf_gpu_ctx *> ctx;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<cudaEvent_t> ready;
    cudaEvent_t done = nullptr;
    int64_t launches = 0;
};

namespace {

int check_opts(const cmf_opts &o) {
    if (o.lkine) return set_err(CMF_E_UNSUPPORTED, "LKINE (kinematic outflow) is not on the GPU path");
    if (o.lslpmix) return set_err(CMF_E_UNSUPPORTED, "LSLPMIX is not on the GPU path");
    if (o.lstg_es) return set_err(CMF_E_UNSUPPORTED, "LSTG_ES: the GPU path implements the default stage scheme");
    if (o.lgdwdly) return set_err(CMF_E_UNSUPPORTED, "LGDWDLY (groundwater delay) is not on the GPU path");
    if (o.lrosplit) return set_err(CMF_E_UNSUPPORTED, "LROSPLIT is not on the GPU path");
    if (o.lwevap) return set_err(CMF_E_UNSUPPORTED, "LWEVAP is not on the GPU path");
    if (o.lupsinf) return set_err(CMF_E_UNSUPPORTED, "LUPSINF is not on the GPU path");
    if (o.lheatlink) return set_err(CMF_E_UNSUPPORTED, "LHEATLINK hooks run inside the sub-step loop on the host");
    if (o.ltrace) return set_err(CMF_E_UNSUPPORTED, "LTRACE is not on the GPU path");
    if (o.lslopemouth) return set_err(CMF_E_UNSUPPORTED, "LSLOPEMOUTH is not on the GPU path");
    if (o.ldamyby) return set_err(CMF_E_UNSUPPORTED, "LDAMYBY is not on the GPU path");
    if (!o.lspamat) return set_err(CMF_E_UNSUPPORTED, "the GPU path implements the LSPAMAT inflow gather");
    return CMF_OK;
}

int build_net(cmf_gpu_ctx *c, const cmf_map_ptrs *mp) {
    const cmf_dims &d = c->dims;
    const int N = d.nseqall, R = d.nseqriv, L = d.nlfp;
    cmf::Net &n = c->net;
    n.N = N; n.R = R; n.L = L; n.M = d.nmembers;
    n.P = c->opts.lpthout ? d.npthout : 0;
    n.Lp = c->opts.lpthout ? d.npthlev : 0;
    n.pgrv = c->params.pgrv; n.pmanfld = c->params.pmanfld; n.pdstmth = c->params.pdstmth;
    n.pcadp = c->params.pcadp; n.pminslp = c->params.pminslp; n.dfrcinc = c->params.dfrcinc;
    n.ladpstp = c->opts.ladpstp; n.lfldout = c->opts.lfldout; n.lpthout = c->opts.lpthout;
    n.ldamout = c->opts.ldamout; n.llevee = c->opts.llevee; n.ldamh22 = c->opts.ldamh22; n.ldiag = c->opts.ldiag;
    n.ldiag_out = c->opts.ldiag && c->opts.ldiag_output;
    // ---- network
    std::vector<int> next(N, -1);
    for (int i = 0; i < R; i++) {
        const int j = mp->i1next[i] - 1;
        if (j <= i || j >= N) return set_err(CMF_E_ARG, "I1NEXT is not a topological order (I1NEXT(i) <= i)");
        next[i] = j;
    }
    for (int i = R; i < N; i++)
        if (mp->i1next[i] > 0) return set_err(CMF_E_ARG, "a river mouth has a downstream cell");
    std::vector<int> up_ptr(N + 1, 0), up_idx;
    up_idx.reserve(R);
    for (int i = 0; i < N; i++) {
        const int nu = mp->i1upn[i];
        if (nu < 0 || nu > d.upnmax) return set_err(CMF_E_ARG, "I1UPN out of range");
        for (int k = 0; k < nu; k++) {
            const int j = mp->i1upst[(size_t)k * d.nseqmax + i] - 1;
            if (j < 0 || j >= N || next[j] != i) return set_err(CMF_E_ARG, "I1UPST inconsistent with I1NEXT");
            up_idx.push_back(j);
        }
        up_ptr[i + 1] = (int)up_idx.size();
    }
    c->E = up_idx.size();
    constexpr int S = cmf::kUpSlots;
    std::vector<int> up_ell((size_t)S * N, -1);
    for (int i = 0; i < N; i++) {
        const int k0 = up_ptr[i], nu = up_ptr[i + 1] - k0;
        for (int k = 0; k < std::min(nu, S); k++) up_ell[(size_t)k * N + i] = up_idx[k0 + k];
        if (nu > S) up_ell[(size_t)(S - 1) * N + i] = -2 - (k0 + S - 1);
    }
    int rc;
    if ((rc = c->upload(&n.next, next)) || (rc = c->upload(&n.up_ptr, up_ptr)) || (rc = c->upload(&n.up_idx, up_idx)) ||
        (rc = c->upload(&n.up_ell, up_ell)))
        return rc;
    std::vector<int> i2mask(mp->i2mask, mp->i2mask + N);
    if ((rc = c->upload(&n.i2mask, i2mask))) return rc;
    struct { const double *__restrict__ *dst; const double *src; size_t cnt; } arrs[] = {
        {&n.rivelv, mp->rivelv, (size_t)N}, {&n.elevtn, mp->elevtn, (size_t)N}, {&n.nxtdst, mp->nxtdst, (size_t)N},
        {&n.rivwth, mp->rivwth, (size_t)N}, {&n.rivhgt, mp->rivhgt, (size_t)N}, {&n.rivlen, mp->rivlen, (size_t)N},
        {&n.rivman, mp->rivman, (size_t)N}, {&n.grarea, mp->grarea, (size_t)N}, {&n.rivstomax, mp->rivstomax, (size_t)N},
        {&n.dwnelv, mp->dwnelv, (size_t)N}};
    for (auto &a : arrs) {
        if (!a.src) return set_err(CMF_E_ARG, "a required map pointer is NULL");
        if ((rc = c->upload_raw(a.dst, a.src, a.cnt))) return rc;
    }
    // reciprocals the outflow formulas take (x**(-1._JPRB)), correctly rounded once here
    {
        std::vector<double> inv(N);
        struct { const double *__restrict__ *dst; const double *src; } recips[] = {
            {&n.inv_nxtdst, mp->nxtdst}, {&n.inv_rivwth, mp->rivwth}, {&n.inv_rivlen, mp->rivlen}};
        for (auto &r : recips) {
            for (int i = 0; i < N; i++) inv[i] = 1.0 / r.src[i];
            if ((rc = c->upload(r.dst, inv))) return rc;
        }
    }
    // layer tables: (NSEQMAX,1,NLFP) -> [L][N]
    auto layers = [&](const double *src, std::vector<double> &out) {
        out.assign((size_t)L * N, 0.0);
        for (int l = 0; l < L; l++) std::memcpy(&out[(size_t)l * N], src + (size_t)l * d.nseqmax, sizeof(double) * N);
    };
    std::vector<double> tmp;
    if (!mp->fldstomax || !mp->fldgrd) return set_err(CMF_E_ARG, "FLDSTOMAX/FLDGRD missing");
    layers(mp->fldstomax, tmp);
    if ((rc = c->upload(&n.fldstomax, tmp))) return rc;
    layers(mp->fldgrd, tmp);
    if ((rc = c->upload(&n.fldgrd, tmp))) return rc;
    if (c->opts.llevee) {
        if (!mp->fldhgt) return set_err(CMF_E_ARG, "FLDHGT missing (levee scheme)");
        layers(mp->fldhgt, tmp);
        if ((rc = c->upload(&n.fldhgt, tmp))) return rc;
    } else {
        if ((rc = c->upload(&n.fldhgt, std::vector<double>(1, 0.0)))) return rc;
    }
    // ---- bifurcation paths
    {
        const int P = n.P, Lp = n.Lp;
        std::vector<int> pu(std::max(P, 1), -1), pd(std::max(P, 1), -1), skip(std::max(P, 1), 3);
        std::vector<double> dst(std::max(P, 1), 1.0), elv((size_t)std::max(P * Lp, 1), 0.0), wth(elv.size(), 1.0),
            man(std::max(Lp, 1), 0.0);
        std::vector<int> po_ptr(N + 1, 0), po_idx, pi_ptr(N + 1, 0), pi_idx;
        if (P > 0) {
            if (Lp > 64) return set_err(CMF_E_UNSUPPORTED, "NPTHLEV above 64");
            for (int p = 0; p < P; p++) {
                const int u = mp->pth_upst[p], v = mp->pth_down[p];
                pu[p] = (u > 0 && u <= N) ? u - 1 : -1;
                pd[p] = (v > 0 && v <= N) ? v - 1 : -1;
                int s = 0;
                if (pu[p] < 0 || pd[p] < 0) s = 3;
                else {
                    if (i2mask[pu[p]] > 0 || i2mask[pd[p]] > 0) s |= 1;
                    if (i2mask[pu[p]] == 1 || i2mask[pd[p]] == 1) s |= 2;
                }
                skip[p] = s;
                dst[p] = mp->pth_dst[p];
                for (int l = 0; l < Lp; l++) {
                    elv[(size_t)l * P + p] = mp->pth_elv[(size_t)l * P + p];
                    wth[(size_t)l * P + p] = mp->pth_wth[(size_t)l * P + p];
                }
            }
            for (int l = 0; l < Lp; l++) man[l] = mp->pth_man[l];
            for (int i = 0; i < N; i++) {
                for (int k = 0; k < mp->i1p_outn[i]; k++) po_idx.push_back(mp->i1p_out[(size_t)k * d.nseqmax + i] - 1);
                po_ptr[i + 1] = (int)po_idx.size();
                for (int k = 0; k < mp->i1p_infn[i]; k++) pi_idx.push_back(mp->i1p_inf[(size_t)k * d.nseqmax + i] - 1);
                pi_ptr[i + 1] = (int)pi_idx.size();
            }
            for (int p : po_idx) if (p < 0 || p >= P) return set_err(CMF_E_ARG, "I1P_OUT out of range");
            for (int p : pi_idx) if (p < 0 || p >= P) return set_err(CMF_E_ARG, "I1P_INF out of range");
        }
        if (po_idx.empty()) po_idx.push_back(0);
        if (pi_idx.empty()) pi_idx.push_back(0);
        if ((rc = c->upload(&n.pth_up, pu)) || (rc = c->upload(&n.pth_dn, pd)) || (rc = c->upload(&n.pth_skip, skip)) ||
            (rc = c->upload(&n.pth_dst, dst)) || (rc = c->upload(&n.pth_elv, elv)) || (rc = c->upload(&n.pth_wth, wth)) ||
            (rc = c->upload(&n.pth_man, man)) || (rc = c->upload(&n.pout_ptr, po_ptr)) || (rc = c->upload(&n.pout_idx, po_idx)) ||
            (rc = c->upload(&n.pinf_ptr, pi_ptr)) || (rc = c->upload(&n.pinf_idx, pi_idx)))
            return rc;
    }
    // ---- levee: compact the cells that do not carry the no-levee sentinels
    {
        std::vector<int> lev_id(N, -1);
        std::vector<double> lh, lf, bh, ld, lb, lt, lfl;
        if (c->opts.llevee) {
            if (!mp->levhgt || !mp->levfrc || !mp->bashgt || !mp->levdst || !mp->levbassto || !mp->levtopsto || !mp->levfilsto)
                return set_err(CMF_E_ARG, "levee parameter pointer missing");
            for (int i = 0; i < N; i++) {
                const bool sentinel = mp->bashgt[i] == 1.E18 && mp->levdst[i] == 1.E18 && mp->levbassto[i] == 1.E18 &&
                                      mp->levtopsto[i] == 1.E18 && mp->levfilsto[i] == 1.E18 && mp->levfrc[i] == 1.0;
                if (sentinel) continue;
                lev_id[i] = (int)lh.size();
                lh.push_back(mp->levhgt[i]); lf.push_back(mp->levfrc[i]); bh.push_back(mp->bashgt[i]);
                ld.push_back(mp->levdst[i]); lb.push_back(mp->levbassto[i]); lt.push_back(mp->levtopsto[i]);
                lfl.push_back(mp->levfilsto[i]);
            }
        }
        c->nlev = (int)lh.size();
        for (auto *v : {&lh, &lf, &bh, &ld, &lb, &lt, &lfl}) if (v->empty()) v->push_back(0.0);
        if ((rc = c->upload(&n.lev_id, lev_id)) || (rc = c->upload(&n.levhgt, lh)) || (rc = c->upload(&n.levfrc, lf)) ||
            (rc = c->upload(&n.bashgt, bh)) || (rc = c->upload(&n.levdst, ld)) || (rc = c->upload(&n.levbassto, lb)) ||
            (rc = c->upload(&n.levtopsto, lt)) || (rc = c->upload(&n.levfilsto, lfl)))
            return rc;
    }
    // ---- dams
    {
        std::vector<int> i1dam(N, 0), dam_id(N, -1), stat;
        std::vector<double> qn, qf, qa, con, eme, nor, adj, rvu;
        if (c->opts.ldamout) {
            if (!mp->damseq || !mp->damstat || !mp->i1dam) return set_err(CMF_E_ARG, "dam table pointer missing");
            for (int i = 0; i < N; i++) i1dam[i] = mp->i1dam[i];
            for (int k = 0; k < d.ndam; k++) {
                if (mp->damstat[k] == kImis) continue;
                const int s = mp->damseq[k] - 1;
                if (s < 0 || s >= N) return set_err(CMF_E_ARG, "DamSeq out of range");
                if (dam_id[s] >= 0) return set_err(CMF_E_UNSUPPORTED, "two dams on one cell");
                dam_id[s] = (int)stat.size();
                stat.push_back(mp->damstat[k]);
                qn.push_back(mp->dam_qn[k]); qf.push_back(mp->dam_qf[k]); qa.push_back(mp->dam_qa[k]);
                con.push_back(mp->dam_convol[k]); eme.push_back(mp->dam_emevol[k]); nor.push_back(mp->dam_norvol[k]);
                adj.push_back(mp->dam_adjvol[k]); rvu.push_back(mp->dam_r_volupa[k]);
            }
            for (int i = 0; i < N; i++)
                if ((i1dam[i] == 1 || i1dam[i] == 11) && dam_id[i] < 0) return set_err(CMF_E_ARG, "I1DAM marks a dam cell without a dam");
        }
        c->ndam_placed = (int)stat.size();
        if (stat.empty()) stat.push_back(0);
        for (auto *v : {&qn, &qf, &qa, &con, &eme, &nor, &adj, &rvu}) if (v->empty()) v->push_back(0.0);
        if ((rc = c->upload(&n.i1dam, i1dam)) || (rc = c->upload(&n.dam_id, dam_id)) || (rc = c->upload(&n.dam_stat, stat)) ||
            (rc = c->upload(&n.qn, qn)) || (rc = c->upload(&n.qf, qf)) || (rc = c->upload(&n.qa, qa)) ||
            (rc = c->upload(&n.convol, con)) || (rc = c->upload(&n.emevol, eme)) || (rc = c->upload(&n.norvol, nor)) ||
            (rc = c->upload(&n.adjvol, adj)) || (rc = c->upload(&n.r_volupa, rvu)))
            return rc;
    }
    return CMF_OK;
}

// ---- hot maps in L2 ----------------------------------------------------------------------------
// The maps every sub-step reads (about 120 B per cell) are moved into one allocation, and the
// context's stream gets a persisting L2 access-policy window over it (kernels launched or
// captured on that stream carry it), so the member state streaming through L2 does not evict
// them.  Only when the whole allocation fits one window (config 1: 36 MB).  The persisting
// carve-out is a process-wide limit of the CUDA context: raised to the largest window any live
// library context needs, and put back when the last of them is destroyed.  Same bits: the kernels
// read identical copies.  One context at a time holds a window: several windows (the domains of a
// batch) would each claim the carve-out, thrash one another inside it and leave the rest of the
// L2 too small for the neighbour gathers of the member state; a context created while another
// holds the window keeps its maps where they are, as a domain too large for one window does.
std::mutex g_l2_mu;
int g_l2_users = 0;
size_t g_l2_saved = 0, g_l2_limit = 0;

int hot_maps_window(cmf_gpu_ctx *c) {
    {
        std::lock_guard<std::mutex> lk(g_l2_mu);
        if (g_l2_users > 0) return CMF_OK;
    }
    cmf::Net &n = c->net;
    const size_t N = (size_t)c->dims.nseqall;
    struct Item { const void **field; size_t bytes; };
    const Item items[] = {
        {(const void **)&n.rivelv, N * 8}, {(const void **)&n.elevtn, N * 8}, {(const void **)&n.rivwth, N * 8},
        {(const void **)&n.rivhgt, N * 8}, {(const void **)&n.rivlen, N * 8}, {(const void **)&n.rivman, N * 8},
        {(const void **)&n.grarea, N * 8}, {(const void **)&n.rivstomax, N * 8}, {(const void **)&n.inv_nxtdst, N * 8},
        {(const void **)&n.inv_rivwth, N * 8}, {(const void **)&n.inv_rivlen, N * 8},
        {(const void **)&n.next, N * 4}, {(const void **)&n.up_ptr, (N + 1) * 4}, {(const void **)&n.up_idx, c->E * 4},
        {(const void **)&n.up_ell, N * 4 * cmf::kUpSlots},
        {(const void **)&n.i1dam, N * 4}, {(const void **)&n.dam_id, N * 4}, {(const void **)&n.lev_id, N * 4},
        {(const void **)&n.pout_ptr, (N + 1) * 4}, {(const void **)&n.pinf_ptr, (N + 1) * 4}};
    size_t total = 0;
    for (const Item &it : items) total += (it.bytes + 255) & ~(size_t)255;
    int max_persist = 0, max_win = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, c->device));
    CUDA_TRY(cudaDeviceGetAttribute(&max_win, cudaDevAttrMaxAccessPolicyWindowSize, c->device));
    if (max_persist <= 0 || max_win <= 0 || total > (size_t)max_win) return CMF_OK;
    char *arena = nullptr;
    CUDA_TRY(cudaMalloc(&arena, total));
    c->allocs.push_back(arena);
    std::vector<const void *> old;
    size_t off = 0;
    for (const Item &it : items) {
        if (it.bytes) CUDA_TRY(cudaMemcpyAsync(arena + off, *it.field, it.bytes, cudaMemcpyDeviceToDevice, c->stream));
        old.push_back(*it.field);
        *it.field = arena + off;
        off += (it.bytes + 255) & ~(size_t)255;
    }
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    for (const void *p : old) {   // the separate allocations the maps came from
        auto at = std::find(c->allocs.begin(), c->allocs.end(), p);
        if (at != c->allocs.end()) {
            cudaFree(*at);
            c->allocs.erase(at);
        }
    }
    const size_t persist = std::min(total, (size_t)max_persist);
    {
        std::lock_guard<std::mutex> lk(g_l2_mu);
        if (g_l2_users == 0) {
            CUDA_TRY(cudaDeviceGetLimit(&g_l2_saved, cudaLimitPersistingL2CacheSize));
            g_l2_limit = g_l2_saved;
        }
        if (persist > g_l2_limit) {
            CUDA_TRY(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, persist));
            g_l2_limit = persist;
        }
        g_l2_users++;
    }
    c->l2_window = true;
    cudaStreamAttrValue v{};
    v.accessPolicyWindow.base_ptr = arena;
    v.accessPolicyWindow.num_bytes = total;
    v.accessPolicyWindow.hitRatio = (float)std::min(1.0, (double)persist / (double)total);
    v.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    v.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    CUDA_TRY(cudaStreamSetAttribute(c->stream, cudaStreamAttributeAccessPolicyWindow, &v));
    return CMF_OK;
}

int alloc_state(cmf_gpu_ctx *c) {
    cmf::State &s = c->st;
    const size_t MN = (size_t)c->dims.nmembers * c->dims.nseqall;
    const size_t MP = (size_t)c->dims.nmembers * std::max(c->net.P, 1);
    const size_t MPL = (size_t)c->dims.nmembers * std::max(c->net.P * c->net.Lp, 1);
    const bool dg = c->opts.ldiag;
    double **cell[] = {&s.rivsto, &s.fldsto, &s.rivout_raw, &s.fldout_raw, &s.rivout_pre, &s.fldout_pre,
                       &s.rivout_cur, &s.fldout_cur, &s.rivdph_pre, &s.fldsto_pre, &s.rivdph, &s.flddph,
                       &s.fldfrc, &s.fldare, &s.sfcelv, &s.storge, &s.rivvel, &s.rivinf, &s.fldinf, &s.pthout,
                       &s.outflw, &s.rate, &s.runoff};
    int rc;
    for (double **p : cell)
        if ((rc = c->alloc(p, MN))) return rc;
    const size_t opt_cells[] = {c->opts.llevee ? MN : 1, c->opts.ldamout ? MN : 1};
    if ((rc = c->alloc(&s.levsto, opt_cells[0])) || (rc = c->alloc(&s.levdph, opt_cells[0]))) return rc;
    if ((rc = c->alloc(&s.damsto, opt_cells[1])) || (rc = c->alloc(&s.daminf, opt_cells[1]))) return rc;
    if ((rc = c->alloc(&s.pthflw_raw, MPL)) || (rc = c->alloc(&s.pthflw_pre, MPL)) || (rc = c->alloc(&s.pthsum_raw, MP)) ||
        (rc = c->alloc(&s.pthsum, MP)))
        return rc;
    double **diag[] = {&s.a_rivout, &s.a_fldout, &s.a_outflw, &s.a_rivvel, &s.a_pthout, &s.a_runoff,
                       &s.m_storge, &s.m_outflw, &s.m_rivdph};
    for (double **p : diag)
        if ((rc = c->alloc(p, dg ? MN : 1))) return rc;
    if ((rc = c->alloc(&s.a_daminf, (dg && c->opts.ldamout) ? MN : 1))) return rc;
    if ((rc = c->alloc(&s.a_pthflw, dg ? MPL : 1)) || (rc = c->alloc(&s.a_pthsum, dg ? MP : 1))) return rc;
    // output-interval accumulators (zeroed by alloc: CMF_DIAG_INIT leaves them at zero, NADD_out = 0)
    const bool dout = c->net.ldiag_out;
    double **oarr[] = {&s.o_rivout, &s.o_fldout, &s.o_outflw, &s.o_rivvel, &s.o_pthout, &s.o_runoff,
                       &s.om_storge, &s.om_outflw, &s.om_rivdph};
    for (double **p : oarr)
        if ((rc = c->alloc(p, dout ? MN : 1))) return rc;
    if ((rc = c->alloc(&s.o_daminf, (dout && c->opts.ldamout) ? MN : 1)) || (rc = c->alloc(&s.o_pthflw, dout ? MPL : 1)) ||
        (rc = c->alloc(&s.o_nadd, c->dims.nmembers)))
        return rc;
    if ((rc = c->alloc(&s.ctl, c->dims.nmembers)) || (rc = c->alloc(&s.loop, 1))) return rc;
    // budget partials: one per warp of 32 cells, per member and budget
    if ((rc = c->alloc(&s.partials, (size_t)c->dims.nmembers * cmf::budget_warps(c->dims.nseqall) * cmf::kBudgets)))
        return rc;
    return CMF_OK;
}

// phase A and phase C in the schedule's occupancy profile; grids cover the cells of every member,
// then (phases A and C) the bifurcation paths
void launch_flux(cmf_gpu_ctx *c) {
    const Sched &q = c->sched;
    const int nc = nblk(c->dims.nseqall, q.bf);
    const dim3 g(nc + nblk(c->net.P, q.bf), c->dims.nmembers);
    if (q.prof)
        cmf::k_flux<cmf::kFluxMinBlocksSmall><<<g, q.bf, 0, c->stream>>>(c->net, c->st, nc);
    else
        cmf::k_flux<cmf::kFluxMinBlocksWide><<<g, q.bf, 0, c->stream>>>(c->net, c->st, nc);
}
void launch_rate(cmf_gpu_ctx *c, int advance, cudaGraphConditionalHandle cond, int use_cond) {
    const dim3 g(nblk(c->dims.nseqall, c->sched.br), c->dims.nmembers);
    cmf::k_rate<<<g, c->sched.br, 0, c->stream>>>(c->net, c->st, advance, cond, use_cond);
}
void launch_store(cmf_gpu_ctx *c) {
    const Sched &q = c->sched;
    const int nc = nblk(c->dims.nseqall, q.bs);
    const dim3 g(nc + nblk(c->net.P, q.bs), c->dims.nmembers);
    if (q.prof)
        cmf::k_store<cmf::kStoreMinBlocksSmall><<<g, q.bs, cmf::store_smem(q.bs), c->stream>>>(c->net, c->st, nc);
    else
        cmf::k_store<cmf::kStoreMinBlocksWide><<<g, q.bs, cmf::store_smem(q.bs), c->stream>>>(c->net, c->st, nc);
}
constexpr int kStageBlock = 256;   // stage + CFL kernel (once per outer step)
void launch_stage(cmf_gpu_ctx *c) {
    const dim3 g(nblk(c->dims.nseqall, kStageBlock), c->dims.nmembers);
    cmf::k_stage<<<g, kStageBlock, 0, c->stream>>>(c->net, c->st);
}

// Enqueue one sub-step (phases A, B, C).
void enqueue_substep(cmf_gpu_ctx *c, int use_cond, cudaGraphConditionalHandle cond) {
    launch_flux(c);
    launch_rate(c, 1, cond, use_cond);
    launch_store(c);
}
void enqueue_substep(cmf_gpu_ctx *c, int use_cond) { enqueue_substep(c, use_cond, c->cond); }

void enqueue_prologue(cmf_gpu_ctx *c, int use_cond, cudaGraphConditionalHandle cond) {
    launch_stage(c);
    cmf::k_ntdt<<<1, 256, 0, c->stream>>>(c->net, c->st, cond, use_cond);
}
void enqueue_prologue(cmf_gpu_ctx *c, int use_cond) { enqueue_prologue(c, use_cond, c->cond); }

// after the sub-step loop: the budgets of every member's last sub-step
void enqueue_epilogue(cmf_gpu_ctx *c) {
    cmf::k_budget<<<dim3(c->dims.nmembers, cmf::kBudgets), cmf::kBudgetThreads, 0, c->stream>>>(c->net, c->st);
}

// Captures one context's outer step (prologue, then a WHILE node around the sub-step body) into
// `graph` as a branch with no dependencies, using the conditional handle `cond` of that graph.
int capture_outer(cmf_gpu_ctx *c, cudaGraph_t graph, cudaGraphConditionalHandle cond) {
    CUDA_TRY(cudaStreamBeginCaptureToGraph(c->stream, graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    enqueue_prologue(c, 1, cond);
    cudaStreamCaptureStatus status;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    cudaGraph_t captured = nullptr;
    CUDA_TRY(cudaStreamGetCaptureInfo(c->stream, &status, nullptr, &captured, &deps, &ndeps));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t cnode;
    CUDA_TRY(cudaGraphAddNode(&cnode, captured, deps, ndeps, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    CUDA_TRY(cudaStreamUpdateCaptureDependencies(c->stream, &cnode, 1, cudaStreamSetCaptureDependencies));
    enqueue_epilogue(c);
    cudaGraph_t g2 = nullptr;
    CUDA_TRY(cudaStreamEndCapture(c->stream, &g2));
    CUDA_TRY(cudaStreamBeginCaptureToGraph(c->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    enqueue_substep(c, 1, cond);
    cudaGraph_t g3 = nullptr;
    CUDA_TRY(cudaStreamEndCapture(c->stream, &g3));
    return CMF_OK;
}

int build_graph(cmf_gpu_ctx *c) {
    if (c->exec) { cudaGraphExecDestroy(c->exec); c->exec = nullptr; }
    if (c->graph) { cudaGraphDestroy(c->graph); c->graph = nullptr; }
    CUDA_TRY(cudaGraphCreate(&c->graph, 0));
    CUDA_TRY(cudaGraphConditionalHandleCreate(&c->cond, c->graph, 1u, cudaGraphCondAssignDefault));
    int rc = capture_outer(c, c->graph, c->cond);
    if (rc) return rc;
    CUDA_TRY(cudaGraphInstantiate(&c->exec, c->graph, 0));
    return CMF_OK;
}

int sync_dt_def(cmf_gpu_ctx *c, double dt_def) {
    if (!(dt_def > 0.0)) return set_err(CMF_E_ARG, "DT must be positive");
    if (dt_def == c->dt_def_dev) return CMF_OK;
    for (auto &m : c->hctl) {
        m.dt_def = dt_def;
        unsigned long long b;
        std::memcpy(&b, &dt_def, sizeof b);
        m.dtmin_bits = b;
    }
    // only the first two fields and the atomicMin target change; copy the whole block (small)
    CUDA_TRY(cudaMemcpyAsync(c->st.ctl, c->hctl.data(), c->hctl.size() * sizeof(cmf::MemberCtl), cudaMemcpyHostToDevice, c->stream));
    c->dt_def_dev = dt_def;
    return CMF_OK;
}

// ---- persistent schedule: one cooperative launch per outer step --------------------------------
int persist_setup(cmf_gpu_ctx *c) {
    CUDA_TRY(cudaFuncSetAttribute(cmf::k_persist, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cmf::kPersistSmem));
    int per_sm = 0, nsm = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cmf::k_persist, cmf::kTile, cmf::kPersistSmem));
    CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
    int coop = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c->device));
    c->persist_grid = coop ? per_sm * nsm : 0;
    return CMF_OK;
}

cmf::PersistArgs persist_args(const cmf_gpu_ctx *c) {
    cmf::PersistArgs a{};
    a.tpm = (c->dims.nseqall + cmf::kTile - 1) / cmf::kTile;
    a.ppm = c->net.P > 0 ? (c->net.P + cmf::kTile - 1) / cmf::kTile : 0;
    a.wait_ns = cmf::kWaitNsDefault;
    a.selftest = 0;
    return a;
}

int launch_persist(cmf_gpu_ctx *c, cmf::PersistArgs a) {
    if (c->persist_grid < 1) return set_err(CMF_E_UNSUPPORTED, "the persistent kernel cannot be co-resident on this device");
    CUDA_TRY(cudaMemsetAsync(&c->st.loop->bar, 0, sizeof(unsigned), c->stream));
    void *args[] = {&c->net, &c->st, &a};
    CUDA_TRY(cudaLaunchCooperativeKernel((const void *)cmf::k_persist, dim3(c->persist_grid), dim3(cmf::kTile), args,
                                         cmf::kPersistSmem, c->stream));
    c->launches += 1;
    return CMF_OK;
}

int read_loop(cmf_gpu_ctx *c, cmf::LoopCtl *lc) {
    CUDA_TRY(cudaMemcpyAsync(lc, c->st.loop, sizeof *lc, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return CMF_OK;
}

int build_graph(cmf_gpu_ctx *c);

// Installs a schedule: the persistent flag and, for graph launches, the graph of the phase kernels.
int apply_sched(cmf_gpu_ctx *c, const Sched &q) {
    const bool rebuild = c->opts.launch_mode == 0 && q.mode == 0 && (!c->exec || !(q == c->sched) || c->persist);
    c->sched = q;
    c->persist = q.mode == 2;
    if (rebuild) return build_graph(c);
    return CMF_OK;
}

using SchedKey = std::tuple<int, int, int, int, int, int, int>;
std::map<SchedKey, Sched> g_sched_cache;
std::mutex g_sched_mu;
SchedKey sched_key(const cmf_gpu_ctx *c) {
    const int flags = c->opts.llevee | (c->opts.ldamout << 1) | (c->opts.lpthout << 2) | (c->opts.ldiag << 3) |
                      (c->net.ldiag_out << 4) | (c->opts.lfldout << 5);
    return SchedKey{c->device, c->dims.nseqall, c->dims.nseqriv, c->dims.nmembers, c->net.P, c->net.Lp, flags};
}

// before an outer step: the tuner's schedule for it, and the start of its timing
int tune_begin(cmf_gpu_ctx *c, bool &trial) {
    trial = false;
    Tuner &t = c->tune;
    if (!t.active) return CMF_OK;
    if (t.warm > 0) {
        t.warm--;
        return CMF_OK;
    }
    int rc;
    if (t.rep == 0 && (rc = apply_sched(c, t.cands[t.cand]))) return rc;
    cmf::LoopCtl lc;
    if ((rc = read_loop(c, &lc))) return rc;
    t.iters0 = lc.loop_iters;
    CUDA_TRY(cudaEventRecord(t.e0, c->stream));
    trial = true;
    return CMF_OK;
}

// after a timed outer step: time per sub-step of the candidate; after the last candidate, the
// fastest schedule is installed and cached
int tune_end(cmf_gpu_ctx *c, bool trial) {
    if (!trial) return CMF_OK;
    Tuner &t = c->tune;
    CUDA_TRY(cudaEventRecord(t.e1, c->stream));
    CUDA_TRY(cudaEventSynchronize(t.e1));
    float ms = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&ms, t.e0, t.e1));
    cmf::LoopCtl lc;
    int rc;
    if ((rc = read_loop(c, &lc))) return rc;
    const double sub = (double)std::max(1LL, lc.loop_iters - t.iters0);
    const double per = ms / sub;
    if (t.rep == 0 || per < t.ms[t.cand]) t.ms[t.cand] = per;       // best of the repetitions
    if (++t.rep < t.reps) return CMF_OK;
    t.rep = 0;
    if (++t.cand < (int)t.cands.size()) return CMF_OK;
    size_t best = 0, worst = 0;
    for (size_t k = 1; k < t.cands.size(); k++) {
        if (t.ms[k] < t.ms[best]) best = k;
        if (t.ms[k] > t.ms[worst]) worst = k;
    }
    t.best_us = t.ms[best] * 1e3;
    t.worst_us = t.ms[worst] * 1e3;
    t.timed = (int)t.cands.size();
    t.active = false;
    if ((rc = apply_sched(c, t.cands[best]))) return rc;
    std::lock_guard<std::mutex> lk(g_sched_mu);
    g_sched_cache[sched_key(c)] = t.cands[best];
    return CMF_OK;
}

int launch_outer(cmf_gpu_ctx *c) {
    bool trial = false;
    int rc;
    if ((rc = tune_begin(c, trial))) return rc;
    if (c->persist) {
        if ((rc = launch_persist(c, persist_args(c)))) return rc;
    } else if (c->opts.launch_mode == 0) {
        CUDA_TRY(cudaGraphLaunch(c->exec, c->stream));
        c->launches += 3;   // prologue and epilogue; the loop body adds 3 per sub-step (counted on read-back)
    } else {
        enqueue_prologue(c, 0);
        CUDA_TRY(cudaGetLastError());
        cmf::LoopCtl lc;
        if ((rc = read_loop(c, &lc))) return rc;
        for (int k = 0; k < lc.ntmax; k++) enqueue_substep(c, 0);
        enqueue_epilogue(c);
        CUDA_TRY(cudaGetLastError());
        c->launches += 3 + 3LL * lc.ntmax;
    }
    return tune_end(c, trial);
}

// the per-member control blocks after a step, read through a pinned buffer (a direct DMA, no
// staging through pageable memory: this read sits between one outer step and the next launch)
int read_ctl(cmf_gpu_ctx *c) {
    const size_t bytes = c->hctl.size() * sizeof(cmf::MemberCtl);
    if (!c->hctl_pin) CUDA_TRY(cudaMallocHost(&c->hctl_pin, bytes));
    CUDA_TRY(cudaMemcpyAsync(c->hctl_pin, c->st.ctl, bytes, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    std::memcpy(c->hctl.data(), c->hctl_pin, bytes);
    return CMF_OK;
}

int zero_state(cmf_gpu_ctx *c) {
    const size_t MN = (size_t)c->dims.nmembers * c->dims.nseqall;
    cmf::State &s = c->st;
    for (double *p : {s.rivsto, s.fldsto, s.rivout_raw, s.fldout_raw, s.rivout_pre, s.fldout_pre, s.rivout_cur, s.fldout_cur,
                      s.rivdph_pre, s.fldsto_pre, s.rivdph, s.flddph, s.fldfrc, s.fldare, s.sfcelv, s.storge, s.rivvel,
                      s.rivinf, s.fldinf, s.pthout, s.outflw, s.rate})
        CUDA_TRY(cudaMemsetAsync(p, 0, MN * sizeof(double), c->stream));
    if (c->opts.llevee) { CUDA_TRY(cudaMemsetAsync(s.levsto, 0, MN * 8, c->stream)); CUDA_TRY(cudaMemsetAsync(s.levdph, 0, MN * 8, c->stream)); }
    if (c->opts.ldamout) { CUDA_TRY(cudaMemsetAsync(s.damsto, 0, MN * 8, c->stream)); CUDA_TRY(cudaMemsetAsync(s.daminf, 0, MN * 8, c->stream)); }
    const size_t MPL = (size_t)c->dims.nmembers * std::max(c->net.P * c->net.Lp, 1);
    const size_t MP = (size_t)c->dims.nmembers * std::max(c->net.P, 1);
    CUDA_TRY(cudaMemsetAsync(s.pthflw_raw, 0, MPL * 8, c->stream));
    CUDA_TRY(cudaMemsetAsync(s.pthflw_pre, 0, MPL * 8, c->stream));
    CUDA_TRY(cudaMemsetAsync(s.pthsum_raw, 0, MP * 8, c->stream));
    CUDA_TRY(cudaMemsetAsync(s.pthsum, 0, MP * 8, c->stream));
    return CMF_OK;
}

template <class T>
int h2d(cmf_gpu_ctx *c, T *dst, const T *src, size_t n) {
    if (!src) return CMF_OK;
    CUDA_TRY(cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyHostToDevice, c->stream));
    return CMF_OK;
}
template <class T>
int d2h(cmf_gpu_ctx *c, T *dst, const T *src, size_t n) {
    if (!dst) return CMF_OK;
    CUDA_TRY(cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyDeviceToHost, c->stream));
    return CMF_OK;
}

// state arrays of the boundary are [M][NSEQMAX]; the device keeps [M][NSEQALL] (== NSEQMAX here)
// NT, DT, budgets and statuses of the step whose control blocks are in c->hctl
int process_ctl(cmf_gpu_ctx *c, int32_t *nt_out, double *dt_out, cmf_budget *b) {
    if (c->persist) {
        int berr = 0;
        CUDA_TRY(cudaMemcpyAsync(&berr, &c->st.loop->bar_err, sizeof berr, cudaMemcpyDeviceToHost, c->stream));
        CUDA_TRY(cudaStreamSynchronize(c->stream));
        if (berr) {
            CUDA_TRY(cudaMemsetAsync(&c->st.loop->bar_err, 0, sizeof(int), c->stream));
            CUDA_TRY(cudaStreamSynchronize(c->stream));
            return set_err(CMF_E_BARRIER, "persistent kernel: a grid barrier did not complete within its bound");
        }
    }
    int err = 0;
    int ntmax = 0;
    for (size_t m = 0; m < c->hctl.size(); m++) {
        const cmf::MemberCtl &x = c->hctl[m];
        if (x.err) err = x.err;
        ntmax = std::max(ntmax, x.nt);
        if (nt_out) nt_out[m] = x.nt;
        if (dt_out) dt_out[m] = x.dt;
        if (b) {
            b[m].stopre = x.budget[0]; b[m].stonxt = x.budget[1]; b[m].stonew = x.budget[2];
            b[m].rivinf = x.budget[3]; b[m].rivout = x.budget[4]; b[m].stopre2 = x.budget[5];
            b[m].stonew2 = x.budget[6]; b[m].rivsto = x.budget[7]; b[m].fldsto = x.budget[8];
            b[m].fldare = x.budget[9]; b[m].levsto = x.budget[10]; b[m].dam_miss = x.budget[11];
        }
    }
    if (c->opts.launch_mode == 0 && !c->persist) c->launches += 3LL * ntmax;
    if (err) {
        int bad = -1;
        for (size_t m = 0; m < c->hctl.size(); m++)
            if (c->hctl[m].err && bad < 0) bad = (int)m;
        // clear the error words on the device: after every step already launched (drained first),
        // from the control blocks as they stand then
        int rc = read_ctl(c);
        if (rc) return rc;
        for (auto &x : c->hctl) x.err = 0;
        CUDA_TRY(cudaMemcpyAsync(c->st.ctl, c->hctl.data(), c->hctl.size() * sizeof(cmf::MemberCtl), cudaMemcpyHostToDevice, c->stream));
        CUDA_TRY(cudaStreamSynchronize(c->stream));
        if (err == cmf::kErrNonFinite)
            return set_err(CMF_E_NONFINITE, "member " + std::to_string(bad) +
                                                ": a sub-step produced a non-finite storage (NaN or infinite runoff or state)");
        return set_err(CMF_E_NT_CAP, "member " + std::to_string(bad) +
                                         ": adaptive sub-step count is not finite or above the cap (DT_MIN non-finite or tiny)");
    }
    return CMF_OK;
}

int finish_outer(cmf_gpu_ctx *c, int32_t *nt_out, double *dt_out, cmf_budget *b) {
    int rc = read_ctl(c);
    if (rc) return rc;
    return process_ctl(c, nt_out, dt_out, b);
}

cmf_gpu_ctx *g_default = nullptr;
constexpr int kTuneWarm = 4;   // outer steps before the autotuner's first candidate

}  // namespace

// ---- pipelined host I/O ------------------------------------------------------------------------
int io_setup(cmf_gpu_ctx *c) {
    if (c->io) return CMF_OK;
    CUDA_TRY(cudaStreamCreateWithFlags(&c->io, cudaStreamNonBlocking));
    CUDA_TRY(cudaStreamCreateWithFlags(&c->io_out, cudaStreamNonBlocking));
    for (cudaEvent_t *e : {&c->ev_in, &c->ev_stage_free, &c->ev_out_staged, &c->ev_out_done, &c->ev_ctl[0], &c->ev_ctl[1]})
        CUDA_TRY(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    for (auto &r : c->ring) CUDA_TRY(cudaMallocHost(&r, c->hctl.size() * sizeof(cmf::MemberCtl)));
    int rc;
    if ((rc = c->alloc(&c->rstage, (size_t)c->dims.nmembers * c->dims.nseqall))) return rc;
    return CMF_OK;
}

// the runoff field staged by put_runoff_async becomes D2RUNOFF ahead of the next outer step
int apply_staged_runoff(cmf_gpu_ctx *c) {
    if (!c->in_pending) return CMF_OK;
    const size_t MN = (size_t)c->dims.nmembers * c->dims.nseqall;
    CUDA_TRY(cudaStreamWaitEvent(c->stream, c->ev_in, 0));
    CUDA_TRY(cudaMemcpyAsync(c->st.runoff, c->rstage, MN * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    CUDA_TRY(cudaEventRecord(c->ev_stage_free, c->stream));
    c->in_pending = false;
    return CMF_OK;
}

// the device arrays behind the named host buffers of a cmf_diag_ptrs (fields without a device
// array in this configuration are skipped); `slot` numbers the fields for the async staging
struct DiagField { double *dst; const double *src; size_t n; int slot; };
std::vector<DiagField> diag_fields(const cmf_gpu_ctx *c, const cmf_diag_ptrs *p) {
    const size_t MN = (size_t)c->dims.nmembers * c->dims.nseqall;
    const size_t MP = (size_t)c->dims.nmembers * c->net.P;
    const size_t MPL = MP * c->net.Lp;
    const cmf::State &s = c->st;
    const bool dg = c->opts.ldiag != 0;
    const DiagField t[] = {
        {p->rivdph, s.rivdph, MN, 0}, {p->flddph, s.flddph, MN, 1}, {p->fldfrc, s.fldfrc, MN, 2}, {p->fldare, s.fldare, MN, 3},
        {p->sfcelv, s.sfcelv, MN, 4}, {p->storge, s.storge, MN, 5}, {p->rivvel, s.rivvel, MN, 6}, {p->rivinf, s.rivinf, MN, 7},
        {p->fldinf, s.fldinf, MN, 8}, {p->pthout, s.pthout, MN, 9}, {p->outflw, s.outflw, MN, 10},
        {p->pthflwsum, s.pthsum, MP, 11}, {p->levdph, c->opts.llevee ? s.levdph : nullptr, MN, 12},
        {p->rivout_aavg, dg ? s.a_rivout : nullptr, MN, 13}, {p->fldout_aavg, dg ? s.a_fldout : nullptr, MN, 14},
        {p->outflw_aavg, dg ? s.a_outflw : nullptr, MN, 15}, {p->rivvel_aavg, dg ? s.a_rivvel : nullptr, MN, 16},
        {p->pthout_aavg, dg ? s.a_pthout : nullptr, MN, 17}, {p->runoff_aavg, dg ? s.a_runoff : nullptr, MN, 18},
        {p->daminf_aavg, dg && c->opts.ldamout ? s.a_daminf : nullptr, MN, 19},
        {p->storge_amax, dg ? s.m_storge : nullptr, MN, 20}, {p->outflw_amax, dg ? s.m_outflw : nullptr, MN, 21},
        {p->rivdph_amax, dg ? s.m_rivdph : nullptr, MN, 22}, {p->pthflw_aavg, dg ? s.a_pthflw : nullptr, MPL, 23},
        {p->pthflwsum_aavg, dg ? s.a_pthsum : nullptr, MP, 24}};
    std::vector<DiagField> out;
    for (const DiagField &x : t)
        if (x.dst && x.src && x.n) out.push_back(x);
    return out;
}
constexpr int kDiagSlots = 25;

extern "C" {

int cmf_gpu_abi_version(void) { return CMF_GPU_ABI_VERSION; }

namespace {
__global__ void k_depth_powers(const double *x, int n, double *p73, double *p43) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    p73[i] = cmf::pow_depth<7>(x[i]);
    p43[i] = cmf::pow_depth<4>(x[i]);
}
__global__ void k_cfl_keys(const double *rivdph, const double *ddst, int n, double pgrv, double pcadp, double *key) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    key[i] = cmf::cfl_key(pcadp, ddst[i], pgrv, rivdph[i]);
}
}  // namespace

int cmf_gpu_cfl_keys(const double *rivdph, const double *ddst, int32_t n, double pgrv, double pcadp, double *key) {
    if (!rivdph || !ddst || !key || n < 0) return set_err(CMF_E_ARG, "cmf_gpu_cfl_keys: null array or negative count");
    if (n == 0) return CMF_OK;
    double *d = nullptr;
    const size_t bytes = (size_t)n * sizeof(double);
    CUDA_TRY(cudaMalloc(&d, 3 * bytes));
    cudaError_t e = cudaMemcpy(d, rivdph, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d + n, ddst, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_cfl_keys<<<(unsigned)((n + 255) / 256), 256>>>(d, d + n, n, pgrv, pcadp, d + 2 * (size_t)n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(key, d + 2 * (size_t)n, bytes, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return set_err(CMF_E_CUDA, std::string("cmf_gpu_cfl_keys: ") + cudaGetErrorString(e));
    return CMF_OK;
}

int cmf_gpu_depth_powers(const double *x, int32_t n, double *p73, double *p43) {
    if (!x || n < 0) return set_err(CMF_E_ARG, "cmf_gpu_depth_powers: null input or negative count");
    if (n == 0) return CMF_OK;
    double *d = nullptr;
    const size_t bytes = (size_t)n * sizeof(double);
    CUDA_TRY(cudaMalloc(&d, 3 * bytes));
    cudaError_t e = cudaMemcpy(d, x, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_depth_powers<<<(unsigned)((n + 255) / 256), 256>>>(d, n, d + n, d + 2 * (size_t)n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && p73) e = cudaMemcpy(p73, d + n, bytes, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && p43) e = cudaMemcpy(p43, d + 2 * (size_t)n, bytes, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return set_err(CMF_E_CUDA, std::string("cmf_gpu_depth_powers: ") + cudaGetErrorString(e));
    return CMF_OK;
}
const char *cmf_gpu_last_error(void) { return g_last_error.c_str(); }

const char *cmf_gpu_strerror(int status) {
    switch (status) {
        case CMF_OK: return "ok";
        case CMF_E_ARG: return "invalid argument or inconsistent dimensions";
        case CMF_E_UNSUPPORTED: return "option combination not supported by the GPU path";
        case CMF_E_STATE: return "GPU context not initialised";
        case CMF_E_IO: return "cannot read a map, table or namelist";
        case CMF_E_CUDA: return "CUDA runtime error";
        case CMF_E_NT_CAP: return "adaptive sub-step count not finite or above the cap";
        case CMF_E_NO_DEVICE: return "no usable CUDA device (sm_100a required)";
        case CMF_E_NONFINITE: return "non-finite storage after a sub-step";
        case CMF_E_BARRIER: return "a bounded device-side wait ran out";
        default: return "unknown status";
    }
}

int cmf_gpu_create(const cmf_dims *dims, const cmf_params *params, const cmf_map_ptrs *maps, const cmf_opts *opts,
                   cmf_gpu_ctx **out) {
    if (!dims || !params || !maps || !opts || !out) return set_err(CMF_E_ARG, "null argument");
    *out = nullptr;
    if (dims->nseqall <= 0 || dims->nseqriv < 0 || dims->nseqriv > dims->nseqall || dims->nlfp <= 0 || dims->nmembers <= 0)
        return set_err(CMF_E_ARG, "bad dimensions");
    if (dims->nseqmax != dims->nseqall) return set_err(CMF_E_UNSUPPORTED, "NSEQMAX /= NSEQALL (MPI region padding)");
    int rc = check_opts(*opts);
    if (rc) return rc;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= opts->device) return set_err(CMF_E_NO_DEVICE, "no CUDA device");
    cudaDeviceProp prop;
    CUDA_TRY(cudaGetDeviceProperties(&prop, opts->device));
    if (prop.major != 10) return set_err(CMF_E_NO_DEVICE, std::string("kernels are built for sm_100a; device is ") + prop.name);
    CUDA_TRY(cudaSetDevice(opts->device));
    auto *c = new cmf_gpu_ctx();
    c->dims = *dims;
    c->params = *params;
    c->opts = *opts;
    c->device = opts->device;
    c->hctl.assign(dims->nmembers, cmf::MemberCtl{});
    auto fail = [&](int code) {
        cmf_gpu_destroy(c);
        return code;
    };
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(set_err(CMF_E_CUDA, "cudaStreamCreate failed"));
    if ((rc = build_net(c, maps))) return fail(rc);
    if ((rc = hot_maps_window(c))) return fail(rc);
    if ((rc = alloc_state(c))) return fail(rc);
    if ((rc = persist_setup(c))) return fail(rc);
    if (opts->launch_mode < 0 || opts->launch_mode > 2) return fail(set_err(CMF_E_ARG, "launch_mode must be 0, 1 or 2"));
    if (opts->block_size && (opts->block_size % 32 || opts->block_size > cmf::kCellThreads || opts->block_size < 64))
        return fail(set_err(CMF_E_ARG, "block_size must be a multiple of 32 in [64, 256]"));
    // starting schedule: phase kernels at 128 threads, the low-spill profile for grids of about a
    // wave (the rule of thumb the autotuner then checks against the alternatives)
    Sched q;
    q.bf = q.br = q.bs = opts->block_size > 0 ? opts->block_size : 128;
    q.prof = (size_t)dims->nseqall * (size_t)dims->nmembers <= cmf::kSmallCellMembers ? 1 : 0;
    if (opts->launch_mode == 2) {
        if (c->persist_grid < 1) return fail(set_err(CMF_E_UNSUPPORTED, "launch_mode 2: the persistent kernel cannot run here"));
        q.mode = 2;
    }
    if ((rc = zero_state(c))) return fail(rc);
    c->dt_def_dev = -1.0;
    if ((rc = sync_dt_def(c, 86400.0))) return fail(rc);
    if ((rc = apply_sched(c, q))) return fail(rc);
    if (opts->launch_mode == 0 && opts->block_size == 0) {
        bool cached = false;
        {
            std::lock_guard<std::mutex> lk(g_sched_mu);
            auto it = g_sched_cache.find(sched_key(c));
            if (it != g_sched_cache.end()) { q = it->second; cached = true; }
        }
        if (cached) {
            if ((rc = apply_sched(c, q))) return fail(rc);
        } else {
            Tuner &t = c->tune;
            for (int bf : {128, 256})
                for (int bs : {128, 256})
                    for (int prof : {0, 1}) {
                        Sched k;
                        k.bf = k.br = bf;
                        k.bs = bs;
                        k.prof = prof;
                        t.cands.push_back(k);
                    }
            if (c->persist_grid > 0) {
                Sched k;
                k.mode = 2;
                t.cands.push_back(k);
            }
            t.ms.assign(t.cands.size(), 0.0);
            t.warm = kTuneWarm;
            if (cudaEventCreate(&t.e0) != cudaSuccess || cudaEventCreate(&t.e1) != cudaSuccess)
                return fail(set_err(CMF_E_CUDA, "cudaEventCreate failed"));
            t.active = true;
        }
    }
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return fail(set_err(CMF_E_CUDA, cudaGetErrorString(cudaGetLastError())));
    *out = c;
    return CMF_OK;
}

int cmf_gpu_destroy(cmf_gpu_ctx *c) {
    if (!c) return CMF_OK;
    cudaSetDevice(c->device);
    // every stream drained (steps, staged uploads, read-backs) before anything they use is freed
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->io) cudaStreamSynchronize(c->io);
    if (c->io_out) cudaStreamSynchronize(c->io_out);
    if (c->exec) cudaGraphExecDestroy(c->exec);
    if (c->graph) cudaGraphDestroy(c->graph);
    if (c->tune.e0) cudaEventDestroy(c->tune.e0);
    if (c->tune.e1) cudaEventDestroy(c->tune.e1);
    for (void *p : c->allocs) cudaFree(p);
    if (c->rgrid) cudaFree(c->rgrid);
    if (c->hctl_pin) cudaFreeHost(c->hctl_pin);
    for (cudaEvent_t e : {c->ev_in, c->ev_stage_free, c->ev_out_staged, c->ev_out_done, c->ev_ctl[0], c->ev_ctl[1]})
        if (e) cudaEventDestroy(e);
    for (auto *r : c->ring)
        if (r) cudaFreeHost(r);
    if (c->io) cudaStreamDestroy(c->io);
    if (c->io_out) cudaStreamDestroy(c->io_out);
    if (c->stream) cudaStreamDestroy(c->stream);
    if (c->l2_window) {
        std::lock_guard<std::mutex> lk(g_l2_mu);
        if (--g_l2_users == 0) {
            cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, g_l2_saved);
            cudaCtxResetPersistingL2Cache();
            g_l2_limit = g_l2_saved;
        }
    }
    delete c;
    return CMF_OK;
}

int cmf_gpu_ctx_set_state(cmf_gpu_ctx *c, const cmf_state_ptrs *p) {
    if (!c || !p) return set_err(CMF_E_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(c->device));
    const size_t MN = (size_t)c->dims.nmembers * c->dims.nseqall;
    const size_t MPL = (size_t)c->dims.nmembers * c->net.P * c->net.Lp;
    cmf::State &s = c->st;
    int rc;
    if ((rc = h2d(c, s.rivsto, p->rivsto, MN)) || (rc = h2d(c, s.fldsto, p->fldsto, MN)) ||
        (rc = h2d(c, s.rivout_cur, p->rivout, MN)) || (rc = h2d(c, s.fldout_cur, p->fldout, MN)) ||
        (rc = h2d(c, s.rivout_pre, p->rivout_pre, MN)) || (rc = h2d(c, s.fldout_pre, p->fldout_pre, MN)) ||
        (rc = h2d(c, s.rivdph_pre, p->rivdph_pre, MN)) || (rc = h2d(c, s.fldsto_pre, p->fldsto_pre, MN)))
        return rc;
    if (c->opts.lpthout && MPL) {
        if ((rc = h2d(c, s.pthflw_pre, p->pthflw_pre, MPL))) return rc;
    }
    if (c->opts.ldamout) {
        if ((rc = h2d(c, s.damsto, p->damsto, MN)) || (rc = h2d(c, s.daminf, p->daminf, MN))) return rc;
    }
    if (c->opts.llevee) {
        if ((rc = h2d(c, s.levsto, p->levsto, MN))) return rc;
    }
    // D2RIVOUT may differ from D2RIVOUT_PRE (restart): the first sub-step reads the host copy
    cmf::LoopCtl lc{};
    CUDA_TRY(cudaMemcpyAsync(&lc, s.loop, sizeof lc, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    lc.split = 1;
    CUDA_TRY(cudaMemcpyAsync(s.loop, &lc, sizeof lc, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return CMF_OK;
}

int cmf_gpu_ctx_counters(cmf_gpu_ctx *c, int64_t *member_substeps, int64_t *loop_iters, int64_t *outer_steps) {
    if (!c) return set_err(CMF_E_STATE, "no context");
    CUDA_TRY(cudaSetDevice(c->device));
    cmf::LoopCtl lc{};
    CUDA_TRY(cudaMemcpyAsync(&lc, c->st.loop, sizeof lc, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (member_substeps) *member_substeps = lc.member_substeps;
    if (loop_iters) *loop_iters = lc.loop_iters;
    if (outer_steps) *outer_steps = lc.outer_steps;
    return CMF_OK;
}

int cmf_gpu_ctx_diag_output(cmf_gpu_ctx *c, int32_t op) {
    if (!c) return set_err(CMF_E_STATE, "no context");
    if (!c->net.ldiag_out) return set_err(CMF_E_UNSUPPORTED, "output diagnostics need opts.ldiag and opts.ldiag_output");
    CUDA_TRY(cudaSetDevice(c->device));
    const size_t MN = (size_t)c->dims.nmembers * c->dims.nseqall;
    const size_t MPL = (size_t)c->dims.nmembers * c->net.P * c->net.Lp;
    cmf::State &s = c->st;
    if (op == CMF_DIAG_OUT_RESET) {
        // CMF_DIAG_RESET_OUTPUT, src/cmf_calc_diag_mod.F90:222-266
        for (double *p : {s.o_rivout, s.o_fldout, s.o_outflw, s.o_rivvel, s.o_pthout, s.o_runoff, s.om_storge, s.om_outflw,
                          s.om_rivdph})
            CUDA_TRY(cudaMemsetAsync(p, 0, MN * sizeof(double), c->stream));
        if (c->opts.ldamout) CUDA_TRY(cudaMemsetAsync(s.o_daminf, 0, MN * sizeof(double), c->stream));
        if (MPL) CUDA_TRY(cudaMemsetAsync(s.o_pthflw, 0, MPL * sizeof(double), c->stream));
        CUDA_TRY(cudaMemsetAsync(s.o_nadd, 0, (size_t)c->dims.nmembers * sizeof(double), c->stream));
        return CMF_OK;
    }
    if (op == CMF_DIAG_OUT_GETAVE) {
        const int b = 256, nc = nblk(c->dims.nseqall, b);
        const dim3 g(nc + (MPL ? nblk(c->net.P * c->net.Lp, b) : 0), c->dims.nmembers);
        cmf::k_diag_getave_output<<<g, b, 0, c->stream>>>(c->net, c->st, nc);
        CUDA_TRY(cudaGetLastError());
        c->launches += 1;
        return CMF_OK;
    }
    return set_err(CMF_E_ARG, "cmf_gpu_ctx_diag_output: op must be CMF_DIAG_OUT_RESET or CMF_DIAG_OUT_GETAVE "
                              "(AVEMAX runs inside every outer step)");
}

int cmf_gpu_ctx_get_diag_output(cmf_gpu_ctx *c, const cmf_diag_out_ptrs *p) {
    if (!c || !p) return set_err(CMF_E_ARG, "null argument");
    if (!c->net.ldiag_out) return set_err(CMF_E_UNSUPPORTED, "output diagnostics need opts.ldiag and opts.ldiag_output");
    CUDA_TRY(cudaSetDevice(c->device));
    const size_t MN = (size_t)c->dims.nmembers * c->dims.nseqall;
    const size_t MPL = (size_t)c->dims.nmembers * c->net.P * c->net.Lp;
    const cmf::State &s = c->st;
    struct { double *dst; const double *src; size_t n; } t[] = {
        {p->rivout_oavg, s.o_rivout, MN}, {p->fldout_oavg, s.o_fldout, MN}, {p->outflw_oavg, s.o_outflw, MN},
        {p->rivvel_oavg, s.o_rivvel, MN}, {p->pthout_oavg, s.o_pthout, MN}, {p->runoff_oavg, s.o_runoff, MN},
        {p->daminf_oavg, c->opts.ldamout ? s.o_daminf : nullptr, MN}, {p->storge_omax, s.om_storge, MN},
        {p->outflw_omax, s.om_outflw, MN}, {p->rivdph_omax, s.om_rivdph, MN}, {p->pthflw_oavg, s.o_pthflw, MPL},
        {p->nadd_out, s.o_nadd, (size_t)c->dims.nmembers}};
    int rc;
    for (auto &x : t) {
        if (!x.dst || !x.src || !x.n) continue;
        if ((rc = d2h(c, x.dst, x.src, x.n))) return rc;
    }
    // GDWRTN/ROFSUB are zero without groundwater delay or LROSPLIT (both refused)
    if (p->gdwrtn_oavg) std::memset(p->gdwrtn_oavg, 0, MN * sizeof(double));
    if (p->rofsub_oavg) std::memset(p->rofsub_oavg, 0, MN * sizeof(double));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return CMF_OK;
}

int cmf_gpu_ctx_persist_selftest(cmf_gpu_ctx *c, int64_t wait_ns) {
    if (!c) return set_err(CMF_E_STATE, "no context");
    if (wait_ns < 1000 || wait_ns > 2000000000LL) return set_err(CMF_E_ARG, "wait_ns must lie in [1 us, 2 s]");
    CUDA_TRY(cudaSetDevice(c->device));
    cmf::PersistArgs a = persist_args(c);
    a.wait_ns = (unsigned long long)wait_ns;
    a.selftest = 1;
    int rc = launch_persist(c, a);
    if (rc) return rc;
    int berr = 0;
    CUDA_TRY(cudaMemcpyAsync(&berr, &c->st.loop->bar_err, sizeof berr, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    CUDA_TRY(cudaGetLastError());
    if (!berr) return set_err(CMF_E_STATE, "persistent self-test: the barrier completed although it could not");
    CUDA_TRY(cudaMemsetAsync(&c->st.loop->bar_err, 0, sizeof(int), c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return set_err(CMF_E_BARRIER, "persistent self-test: the grid barrier ran out its bound and the kernel returned");
}

int32_t cmf_gpu_ctx_launch_mode(cmf_gpu_ctx *c) { return c ? (c->persist ? 2 : c->opts.launch_mode) : -1; }

int cmf_gpu_ctx_nt_stats(cmf_gpu_ctx *c, int64_t *near_boundary, int64_t *hist, int32_t nbins) {
    if (!c) return set_err(CMF_E_STATE, "no context");
    if (hist && nbins < 1) return set_err(CMF_E_ARG, "cmf_gpu_ctx_nt_stats: nbins must be positive");
    CUDA_TRY(cudaSetDevice(c->device));
    cmf::LoopCtl lc{};
    CUDA_TRY(cudaMemcpyAsync(&lc, c->st.loop, sizeof lc, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (near_boundary) *near_boundary = lc.near_int;
    if (hist) {
        for (int k = 0; k < nbins; k++) hist[k] = 0;
        for (int k = 0; k < cmf::kNtHist; k++) hist[std::min(k, nbins - 1)] += lc.nt_hist[k];
    }
    return CMF_OK;
}

int cmf_gpu_ctx_time_phases(cmf_gpu_ctx *c, double dt_def, int32_t reps, double *ms_out) {
    // Runs `reps` outer steps kernel by kernel (the host-driven schedule) with CUDA events between
    // the kernels on the context's stream, so every sub-step of the step is timed -- first, middle
    // and last alike.  ms_out[0..5] = mean ms per launch of k_stage, k_ntdt (per outer step), of
    // k_flux, k_rate, k_store (per sub-step) and of k_budget (per outer step).  Advances the state
    // like `reps` outer steps.
    if (!c || reps <= 0 || !ms_out) return set_err(CMF_E_ARG, "bad argument");
    CUDA_TRY(cudaSetDevice(c->device));
    int rc;
    if ((rc = sync_dt_def(c, dt_def))) return rc;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    long long nsub = 0;
    std::vector<cudaEvent_t> ev;
    auto need = [&](size_t n) -> int {
        while (ev.size() < n) {
            cudaEvent_t e;
            CUDA_TRY(cudaEventCreate(&e));
            ev.push_back(e);
        }
        return CMF_OK;
    };
    for (int r = 0; r < reps && !rc; r++) {
        if ((rc = need(3))) break;
        CUDA_TRY(cudaEventRecord(ev[0], c->stream));
        launch_stage(c);
        CUDA_TRY(cudaEventRecord(ev[1], c->stream));
        cmf::k_ntdt<<<1, 256, 0, c->stream>>>(c->net, c->st, c->cond, 0);
        CUDA_TRY(cudaEventRecord(ev[2], c->stream));
        cmf::LoopCtl lc;
        CUDA_TRY(cudaMemcpyAsync(&lc, c->st.loop, sizeof lc, cudaMemcpyDeviceToHost, c->stream));
        CUDA_TRY(cudaStreamSynchronize(c->stream));
        float ms = 0.f;
        CUDA_TRY(cudaEventElapsedTime(&ms, ev[0], ev[1]));
        acc[0] += ms;
        CUDA_TRY(cudaEventElapsedTime(&ms, ev[1], ev[2]));
        acc[1] += ms;
        const int nt = lc.ntmax;
        if ((rc = need(3 * (size_t)nt + 2))) break;
        CUDA_TRY(cudaEventRecord(ev[0], c->stream));
        for (int k = 0; k < nt; k++) {
            launch_flux(c);
            CUDA_TRY(cudaEventRecord(ev[3 * k + 1], c->stream));
            launch_rate(c, 1, c->cond, 0);
            CUDA_TRY(cudaEventRecord(ev[3 * k + 2], c->stream));
            launch_store(c);
            CUDA_TRY(cudaEventRecord(ev[3 * k + 3], c->stream));
        }
        enqueue_epilogue(c);
        CUDA_TRY(cudaEventRecord(ev[3 * nt + 1], c->stream));
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaStreamSynchronize(c->stream));
        for (int k = 0; k < 3 * nt; k++) {
            CUDA_TRY(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
            acc[2 + k % 3] += ms;
        }
        CUDA_TRY(cudaEventElapsedTime(&ms, ev[3 * nt], ev[3 * nt + 1]));
        acc[5] += ms;
        nsub += nt;
        c->launches += 3 + 3LL * nt;
    }
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
    if (rc) return rc;
    ms_out[0] = acc[0] / reps;
    ms_out[1] = acc[1] / reps;
    for (int k = 2; k < 5; k++) ms_out[k] = nsub ? acc[k] / (double)nsub : 0.0;
    ms_out[5] = acc[5] / reps;
    return CMF_OK;
}

int cmf_gpu_ctx_get_state(cmf_gpu_ctx *c, const cmf_state_ptrs *p) {
    if (!c || !p) return set_err(CMF_E_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(c->device));
    const size_t MN = (size_t)c->dims.nmembers * c->dims.nseqall;
    const size_t MPL = (size_t)c->dims.nmembers * c->net.P * c->net.Lp;
    cmf::State &s = c->st;
    cmf::LoopCtl lc{};
    CUDA_TRY(cudaMemcpyAsync(&lc, s.loop, sizeof lc, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    int rc;
    if ((rc = d2h(c, p->rivsto, s.rivsto, MN)) || (rc = d2h(c, p->fldsto, s.fldsto, MN)) ||
        (rc = d2h(c, p->rivout, lc.split ? s.rivout_cur : s.rivout_pre, MN)) ||
        (rc = d2h(c, p->fldout, lc.split ? s.fldout_cur : s.fldout_pre, MN)) ||
        (rc = d2h(c, p->rivout_pre, s.rivout_pre, MN)) || (rc = d2h(c, p->fldout_pre, s.fldout_pre, MN)) ||
        (rc = d2h(c, p->rivdph_pre, s.rivdph_pre, MN)) || (rc = d2h(c, p->fldsto_pre, s.fldsto_pre, MN)))
        return rc;
    if (c->opts.lpthout && MPL) {
        if ((rc = d2h(c, p->pthflw_pre, s.pthflw_pre, MPL)) || (rc = d2h(c, p->pthflw, s.pthflw_pre, MPL))) return rc;
    }
    if (c->opts.ldamout) {
        if ((rc = d2h(c, p->damsto, s.damsto, MN)) || (rc = d2h(c, p->daminf, s.daminf, MN))) return rc;
    }
    if (c->opts.llevee) {
        if ((rc = d2h(c, p->levsto, s.levsto, MN))) return rc;
    }
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return CMF_OK;
}

int cmf_gpu_ctx_put_runoff(cmf_gpu_ctx *c, const double *runoff, const double *rofsub) {
    if (!c || !runoff) return set_err(CMF_E_ARG, "null argument");
    (void)rofsub;   // D2ROFSUB only enters the physics through LROSPLIT/LGDWDLY, which are refused
    CUDA_TRY(cudaSetDevice(c->device));
    const size_t MN = (size_t)c->dims.nmembers * c->dims.nseqall;
    CUDA_TRY(cudaMemcpyAsync(c->st.runoff, runoff, MN * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    c->in_pending = false;   // the newest field wins over one staged by put_runoff_async
    return CMF_OK;
}

int cmf_gpu_ctx_physics_advance(cmf_gpu_ctx *c, double dt_def, int32_t *nt_out, double *dt_out, cmf_budget *b) {
    if (!c) return set_err(CMF_E_STATE, "no context");
    CUDA_TRY(cudaSetDevice(c->device));
    int rc;
    if (c->inflight) return set_err(CMF_E_STATE, "physics_advance: steps launched by advance_async are not waited for");
    if ((rc = sync_dt_def(c, dt_def))) return rc;
    if ((rc = apply_staged_runoff(c))) return rc;
    if ((rc = launch_outer(c))) return rc;
    CUDA_TRY(cudaGetLastError());
    return finish_outer(c, nt_out, dt_out, b);
}

int cmf_gpu_ctx_put_runoff_async(cmf_gpu_ctx *c, const double *runoff) {
    if (!c || !runoff) return set_err(CMF_E_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(c->device));
    int rc;
    if ((rc = io_setup(c))) return rc;
    const size_t MN = (size_t)c->dims.nmembers * c->dims.nseqall;
    // the staging buffer is free once the previous staged field was copied into D2RUNOFF
    CUDA_TRY(cudaStreamWaitEvent(c->io, c->ev_stage_free, 0));
    CUDA_TRY(cudaMemcpyAsync(c->rstage, runoff, MN * sizeof(double), cudaMemcpyHostToDevice, c->io));
    CUDA_TRY(cudaEventRecord(c->ev_in, c->io));
    c->in_pending = true;
    return CMF_OK;
}

int cmf_gpu_ctx_advance_async(cmf_gpu_ctx *c, double dt_def) {
    if (!c) return set_err(CMF_E_STATE, "no context");
    if (c->inflight >= 2) return set_err(CMF_E_STATE, "advance_async: two steps are in flight; wait for the oldest first");
    CUDA_TRY(cudaSetDevice(c->device));
    int rc;
    if ((rc = io_setup(c))) return rc;
    if ((rc = sync_dt_def(c, dt_def))) return rc;
    if ((rc = apply_staged_runoff(c))) return rc;
    if ((rc = launch_outer(c))) return rc;
    CUDA_TRY(cudaGetLastError());
    const int slot = (c->head + c->inflight) % 2;
    CUDA_TRY(cudaMemcpyAsync(c->ring[slot], c->st.ctl, c->hctl.size() * sizeof(cmf::MemberCtl), cudaMemcpyDeviceToHost,
                             c->stream));
    CUDA_TRY(cudaEventRecord(c->ev_ctl[slot], c->stream));
    c->inflight++;
    return CMF_OK;
}

int cmf_gpu_ctx_wait(cmf_gpu_ctx *c, int32_t *nt_out, double *dt_out, cmf_budget *b) {
    if (!c) return set_err(CMF_E_STATE, "no context");
    if (!c->inflight) return set_err(CMF_E_STATE, "wait: no outer step was launched by advance_async");
    CUDA_TRY(cudaSetDevice(c->device));
    const int slot = c->head;
    c->head = (c->head + 1) % 2;
    c->inflight--;
    CUDA_TRY(cudaEventSynchronize(c->ev_ctl[slot]));
    std::memcpy(c->hctl.data(), c->ring[slot], c->hctl.size() * sizeof(cmf::MemberCtl));
    return process_ctl(c, nt_out, dt_out, b);
}


int cmf_gpu_ctx_advance_device(cmf_gpu_ctx *c, double dt_def, int32_t ksteps, const double *runoff_dev, int64_t stride) {
    if (!c || ksteps < 0) return set_err(CMF_E_ARG, "bad argument");
    CUDA_TRY(cudaSetDevice(c->device));
    int rc;
    if ((rc = sync_dt_def(c, dt_def))) return rc;
    // a field staged by put_runoff_async: the first step's runoff unless device fields are given
    if (runoff_dev) c->in_pending = false;
    else if (ksteps > 0 && (rc = apply_staged_runoff(c))) return rc;
    const size_t MN = (size_t)c->dims.nmembers * c->dims.nseqall;
    for (int k = 0; k < ksteps; k++) {
        if (runoff_dev)
            CUDA_TRY(cudaMemcpyAsync(c->st.runoff, runoff_dev + (size_t)k * stride, MN * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
        if ((rc = launch_outer(c))) return rc;
    }
    return CMF_OK;
}

void cmf_gpu_batch_destroy(cmf_gpu_batch *b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (cudaEvent_t e : b->ready) if (e) cudaEventDestroy(e);
    if (b->done) cudaEventDestroy(b->done);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

int cmf_gpu_batch_create(cmf_gpu_ctx *const *ctxs, int32_t n, cmf_gpu_batch **out) {
    if (!ctxs || n < 1 || !out) return set_err(CMF_E_ARG, "cmf_gpu_batch_create: null argument or empty batch");
    *out = nullptr;
    for (int k = 0; k < n; k++) {
        if (!ctxs[k]) return set_err(CMF_E_ARG, "cmf_gpu_batch_create: null context");
        if (ctxs[k]->device != ctxs[0]->device) return set_err(CMF_E_ARG, "cmf_gpu_batch_create: contexts on different devices");
        if (ctxs[k]->opts.launch_mode != 0) return set_err(CMF_E_ARG, "cmf_gpu_batch_create: contexts must use launch_mode 0");
        for (int j = 0; j < k; j++)
            if (ctxs[j] == ctxs[k]) return set_err(CMF_E_ARG, "cmf_gpu_batch_create: a context appears twice");
    }
    auto *b = new cmf_gpu_batch();
    b->ctx.assign(ctxs, ctxs + n);
    b->device = ctxs[0]->device;
    auto fail = [&](int code) { cmf_gpu_batch_destroy(b); return code; };
    if (cudaSetDevice(b->device) != cudaSuccess || cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) != cudaSuccess || cudaGraphCreate(&b->graph, 0) != cudaSuccess)
        return fail(set_err(CMF_E_CUDA, "cmf_gpu_batch_create: stream/event/graph creation failed"));
    b->ready.assign(n, nullptr);
    for (int k = 0; k < n; k++) {
        if (cudaEventCreateWithFlags(&b->ready[k], cudaEventDisableTiming) != cudaSuccess)
            return fail(set_err(CMF_E_CUDA, "cmf_gpu_batch_create: event creation failed"));
        cmf_gpu_ctx *c = ctxs[k];
        if (cudaStreamSynchronize(c->stream) != cudaSuccess) return fail(set_err(CMF_E_CUDA, "context stream failed"));
        cudaGraphConditionalHandle h;
        if (cudaGraphConditionalHandleCreate(&h, b->graph, 1u, cudaGraphCondAssignDefault) != cudaSuccess)
            return fail(set_err(CMF_E_CUDA, "cmf_gpu_batch_create: conditional handle"));
        int rc = capture_outer(c, b->graph, h);
        if (rc) return fail(rc);
    }
    if (cudaGraphInstantiate(&b->exec, b->graph, 0) != cudaSuccess)
        return fail(set_err(CMF_E_CUDA, "cmf_gpu_batch_create: graph instantiation failed"));
    *out = b;
    return CMF_OK;
}

int cmf_gpu_batch_launch(cmf_gpu_batch *b, double dt_def) {
    if (!b) return set_err(CMF_E_STATE, "no batch");
    CUDA_TRY(cudaSetDevice(b->device));
    int rc;
    for (size_t k = 0; k < b->ctx.size(); k++) {
        cmf_gpu_ctx *c = b->ctx[k];
        if ((rc = sync_dt_def(c, dt_def))) return rc;
        CUDA_TRY(cudaEventRecord(b->ready[k], c->stream));          // runoff, state uploads, DT
        CUDA_TRY(cudaStreamWaitEvent(b->stream, b->ready[k], 0));
    }
    CUDA_TRY(cudaGraphLaunch(b->exec, b->stream));
    CUDA_TRY(cudaEventRecord(b->done, b->stream));
    for (cmf_gpu_ctx *c : b->ctx) {
        CUDA_TRY(cudaStreamWaitEvent(c->stream, b->done, 0));      // later work of a context follows the step
        c->launches += 3;
    }
    b->launches += 1;
    return CMF_OK;
}

int cmf_gpu_batch_advance(cmf_gpu_batch *b, double dt_def, int32_t *nt_out, double *dt_out, cmf_budget *budget_out) {
    int rc = cmf_gpu_batch_launch(b, dt_def);
    if (rc) return rc;
    size_t off = 0;
    int first_err = CMF_OK;
    for (cmf_gpu_ctx *c : b->ctx) {
        rc = finish_outer(c, nt_out ? nt_out + off : nullptr, dt_out ? dt_out + off : nullptr,
                          budget_out ? budget_out + off : nullptr);
        if (rc && !first_err) first_err = rc;
        off += (size_t)c->dims.nmembers;
    }
    return first_err;
}

int cmf_gpu_batch_synchronize(cmf_gpu_batch *b) {
    if (!b) return set_err(CMF_E_STATE, "no batch");
    CUDA_TRY(cudaSetDevice(b->device));
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    return CMF_OK;
}

void *cmf_gpu_batch_stream(cmf_gpu_batch *b) { return b ? (void *)b->stream : nullptr; }

int cmf_gpu_ctx_synchronize(cmf_gpu_ctx *c) {
    if (!c) return set_err(CMF_E_STATE, "no context");
    CUDA_TRY(cudaSetDevice(c->device));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return CMF_OK;
}

int cmf_gpu_ctx_last_nt(cmf_gpu_ctx *c, int32_t *nt_out, double *dt_out) {
    if (!c) return set_err(CMF_E_STATE, "no context");
    CUDA_TRY(cudaSetDevice(c->device));
    int rc = read_ctl(c);
    if (rc) return rc;
    for (size_t m = 0; m < c->hctl.size(); m++) {
        if (nt_out) nt_out[m] = c->hctl[m].nt;
        if (dt_out) dt_out[m] = c->hctl[m].dt;
    }
    return CMF_OK;
}

int cmf_gpu_ctx_emu_views(cmf_gpu_ctx *c, int32_t m, cmf_emu_net *net, cmf_emu_member *mb) {
    if (!c || m < 0 || m >= c->dims.nmembers) return set_err(CMF_E_ARG, "bad member");
    if (!c->opts.ldiag) return set_err(CMF_E_UNSUPPORTED, "emulator views need ldiag (D2OUTFLW_aAVG)");
    const size_t o = (size_t)m * c->dims.nseqall;
    if (net) {
        net->nseqall = c->net.N; net->nseqriv = c->net.R;
        net->next = c->net.next; net->up_ptr = c->net.up_ptr; net->up_idx = c->net.up_idx;
        net->rivelv = c->net.rivelv; net->elevtn = c->net.elevtn; net->nxtdst = c->net.nxtdst;
        net->rivwth = c->net.rivwth; net->rivhgt = c->net.rivhgt; net->rivlen = c->net.rivlen;
        net->rivstomax = c->net.rivstomax; net->qref = nullptr; net->rivman = c->net.rivman;
        net->pmanfld = c->net.pmanfld;
    }
    if (mb) {
        const cmf::State &s = c->st;
        mb->rivsto = s.rivsto + o; mb->fldsto = s.fldsto + o; mb->levsto = c->opts.llevee ? s.levsto + o : nullptr;
        mb->rivdph = s.rivdph + o; mb->flddph = s.flddph + o; mb->fldfrc = s.fldfrc + o;
        mb->qprev = s.a_outflw + o; mb->runoff = s.runoff + o;
        mb->rivout_pre = s.rivout_pre + o; mb->fldout_pre = s.fldout_pre + o;
    }
    return CMF_OK;
}

int cmf_gpu_ctx_copy_member(cmf_gpu_ctx *d, int32_t dm, cmf_gpu_ctx *s, int32_t sm) {
    if (!d || !s || dm < 0 || sm < 0 || dm >= d->dims.nmembers || sm >= s->dims.nmembers)
        return set_err(CMF_E_ARG, "bad member");
    if (d->dims.nseqall != s->dims.nseqall || d->opts.llevee != s->opts.llevee || d->opts.ldamout != s->opts.ldamout ||
        d->net.P != s->net.P || d->net.Lp != s->net.Lp || d->opts.ldiag != s->opts.ldiag)
        return set_err(CMF_E_ARG, "contexts differ in network or options");
    CUDA_TRY(cudaSetDevice(d->device));
    CUDA_TRY(cudaStreamSynchronize(d->stream));   // nothing of the destination's may still be in flight
    const size_t N = d->dims.nseqall, od = (size_t)dm * N, os = (size_t)sm * N;
    const cmf::State &A = d->st, &B = s->st;
    double *cells_d[] = {A.rivsto, A.fldsto, A.rivout_pre, A.fldout_pre, A.rivdph_pre, A.fldsto_pre, A.rivdph, A.flddph,
                         A.fldfrc, A.fldare, A.sfcelv, A.storge, A.runoff, A.a_outflw};
    double *cells_s[] = {B.rivsto, B.fldsto, B.rivout_pre, B.fldout_pre, B.rivdph_pre, B.fldsto_pre, B.rivdph, B.flddph,
                         B.fldfrc, B.fldare, B.sfcelv, B.storge, B.runoff, B.a_outflw};
    for (size_t k = 0; k < sizeof(cells_d) / sizeof(cells_d[0]); k++) {
        if (!d->opts.ldiag && k == 13) continue;
        CUDA_TRY(cudaMemcpyAsync(cells_d[k] + od, cells_s[k] + os, N * 8, cudaMemcpyDeviceToDevice, s->stream));
    }
    // D2RIVOUT/D2FLDOUT equal the _PRE arrays after a step; keep the destination consistent even
    // if it still reads the host-set copies (first step after an upload)
    CUDA_TRY(cudaMemcpyAsync(A.rivout_cur + od, B.rivout_pre + os, N * 8, cudaMemcpyDeviceToDevice, s->stream));
    CUDA_TRY(cudaMemcpyAsync(A.fldout_cur + od, B.fldout_pre + os, N * 8, cudaMemcpyDeviceToDevice, s->stream));
    if (d->opts.llevee) {
        CUDA_TRY(cudaMemcpyAsync(A.levsto + od, B.levsto + os, N * 8, cudaMemcpyDeviceToDevice, s->stream));
        CUDA_TRY(cudaMemcpyAsync(A.levdph + od, B.levdph + os, N * 8, cudaMemcpyDeviceToDevice, s->stream));
    }
    if (d->opts.ldamout) {
        CUDA_TRY(cudaMemcpyAsync(A.damsto + od, B.damsto + os, N * 8, cudaMemcpyDeviceToDevice, s->stream));
        CUDA_TRY(cudaMemcpyAsync(A.daminf + od, B.daminf + os, N * 8, cudaMemcpyDeviceToDevice, s->stream));
    }
    if (d->net.P > 0) {
        const size_t PL = (size_t)d->net.P * d->net.Lp;
        CUDA_TRY(cudaMemcpyAsync(A.pthflw_pre + dm * PL, B.pthflw_pre + sm * PL, PL * 8, cudaMemcpyDeviceToDevice, s->stream));
    }
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return CMF_OK;
}

int cmf_gpu_ctx_calc_outpre(cmf_gpu_ctx *c) {
    if (!c) return set_err(CMF_E_STATE, "no context");
    // CMF_DRV_INIT (src/cmf_drv_control_mod.F90:273-277): stage scheme, then CMF_CALC_OUTPRE
    const double dt = c->dt_def_dev > 0.0 ? c->dt_def_dev : 86400.0;
    int rc = cmf_gpu_ctx_stage(c, dt, nullptr);
    if (rc) return rc;
    const int b = 256, nc = nblk(c->dims.nseqall, b);
    const dim3 g(nc + nblk(c->net.P, b), c->dims.nmembers);
    cmf::k_outpre<<<g, b, 0, c->stream>>>(c->net, c->st, nc);
    CUDA_TRY(cudaGetLastError());
    c->launches += 1;
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return CMF_OK;
}

int cmf_gpu_ctx_update_boundary(cmf_gpu_ctx *c, const double *sealev, const double *meansl) {
    if (!c) return set_err(CMF_E_STATE, "no context");
    CUDA_TRY(cudaSetDevice(c->device));
    const size_t N = c->dims.nseqall;
    int rc;
    if (sealev) {
        if (!c->bnd_sealev && (rc = c->alloc(&c->bnd_sealev, N))) return rc;
        CUDA_TRY(cudaMemcpyAsync(c->bnd_sealev, sealev, N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    }
    if (meansl) {
        if (!c->bnd_meansl && (rc = c->alloc(&c->bnd_meansl, N))) return rc;
        CUDA_TRY(cudaMemcpyAsync(c->bnd_meansl, meansl, N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    }
    // D2DWNELV is static data of the context (read by the graph's kernels through the same pointer)
    cmf::k_boundary<<<(unsigned)((N + 255) / 256), 256, 0, c->stream>>>((int)N, c->net.elevtn, meansl ? c->bnd_meansl : nullptr,
                                                                        sealev ? c->bnd_sealev : nullptr,
                                                                        const_cast<double *>(c->net.dwnelv));
    CUDA_TRY(cudaGetLastError());
    c->launches += 1;
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return CMF_OK;
}

int cmf_gpu_ctx_set_runoff_map(cmf_gpu_ctx *c, int32_t linterp, int32_t nxin, int32_t nyin, int32_t inpn,
                               const int32_t *inpx, const int32_t *inpy, const double *inpa, double drofunit) {
    if (!c) return set_err(CMF_E_STATE, "no context");
    if (nxin < 1 || nyin < 1 || !inpx || !inpy || !(drofunit > 0.0) || (linterp && (inpn < 1 || !inpa)) ||
        (!linterp && inpn != 1))
        return set_err(CMF_E_ARG, "cmf_gpu_ctx_set_runoff_map: bad arguments (CONV_RESOL takes inpn == 1, the cell grid)");
    CUDA_TRY(cudaSetDevice(c->device));
    const size_t N = c->dims.nseqall, n = (size_t)inpn * N;
    for (size_t k = 0; k < n; k++) {
        if (!linterp && (inpx[k] < 1 || inpx[k] > nxin || inpy[k] < 1 || inpy[k] > nyin))
            return set_err(CMF_E_ARG, "cmf_gpu_ctx_set_runoff_map: a cell lies outside the runoff grid");
    }
    int rc;
    const int32_t *dx, *dy;
    const double *da = nullptr;
    if ((rc = c->upload_raw(&dx, inpx, n)) || (rc = c->upload_raw(&dy, inpy, n))) return rc;
    if (linterp && (rc = c->upload_raw(&da, inpa, n))) return rc;
    c->rmap = cmf::RunoffMap{linterp ? 1 : 0, nxin, nyin, inpn, 0, dx, dy, da, drofunit};
    c->rmap_set = true;
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return CMF_OK;
}

int cmf_gpu_ctx_put_runoff_grid(cmf_gpu_ctx *c, const void *grid, int32_t is_float, int32_t on_device, int32_t clean) {
    if (!c) return set_err(CMF_E_STATE, "no context");
    if (!c->rmap_set) return set_err(CMF_E_STATE, "cmf_gpu_ctx_put_runoff_grid: no runoff map (cmf_gpu_ctx_set_runoff_map)");
    if (!grid) return set_err(CMF_E_ARG, "null runoff field");
    CUDA_TRY(cudaSetDevice(c->device));
    const size_t bytes = (size_t)c->dims.nmembers * c->rmap.nxin * c->rmap.nyin * (is_float ? 4 : 8);
    const void *src = grid;
    if (!on_device) {
        if (c->rgrid_bytes < bytes) {
            if (c->rgrid) { cudaStreamSynchronize(c->stream); cudaFree(c->rgrid); c->rgrid = nullptr; c->rgrid_bytes = 0; }
            CUDA_TRY(cudaMalloc(&c->rgrid, bytes));
            c->rgrid_bytes = bytes;
        }
        CUDA_TRY(cudaMemcpyAsync(c->rgrid, grid, bytes, cudaMemcpyHostToDevice, c->stream));
        src = c->rgrid;
    }
    cmf::RunoffMap r = c->rmap;
    r.clean = clean ? 1 : 0;
    const dim3 g((unsigned)((c->dims.nseqall + 255) / 256), c->dims.nmembers);
    cmf::k_runoff_map<<<g, 256, 0, c->stream>>>(c->net, c->st, r, is_float ? nullptr : (const double *)src,
                                                 is_float ? (const float *)src : nullptr);
    CUDA_TRY(cudaGetLastError());
    c->launches += 1;
    if (!on_device) CUDA_TRY(cudaStreamSynchronize(c->stream));   // the host buffer may be reused on return
    return CMF_OK;
}

void *cmf_gpu_ctx_stream(cmf_gpu_ctx *c) { return c ? (void *)c->stream : nullptr; }
int64_t cmf_gpu_ctx_kernel_launches(cmf_gpu_ctx *c) { return c ? c->launches : 0; }
int32_t cmf_gpu_ctx_block_size(cmf_gpu_ctx *c) { return c ? c->sched.bf : 0; }

int cmf_gpu_ctx_get_schedule(cmf_gpu_ctx *c, cmf_schedule *out) {
    if (!c || !out) return set_err(CMF_E_ARG, "null argument");
    const Sched &q = c->sched;
    out->mode = q.mode;
    out->flux_block = q.bf;
    out->rate_block = q.br;
    out->store_block = q.bs;
    out->profile = q.prof;
    out->tuned = c->tune.active ? -1 : (c->tune.timed > 0 ? 1 : 0);
    out->candidates = c->tune.timed;
    out->best_us_per_substep = c->tune.best_us;
    out->worst_us_per_substep = c->tune.worst_us;
    return CMF_OK;
}

void cmf_gpu_schedule_cache_clear(void) {
    std::lock_guard<std::mutex> lk(g_sched_mu);
    g_sched_cache.clear();
}

int cmf_gpu_ctx_set_schedule(cmf_gpu_ctx *c, const cmf_schedule *q) {
    if (!c || !q) return set_err(CMF_E_ARG, "null argument");
    if (c->opts.launch_mode == 1) return set_err(CMF_E_UNSUPPORTED, "launch_mode 1 contexts run the phase kernels from the host");
    Sched k;
    k.mode = q->mode;
    k.bf = q->flux_block;
    k.br = q->rate_block;
    k.bs = q->store_block;
    k.prof = q->profile;
    if (k.mode != 0 && k.mode != 2) return set_err(CMF_E_ARG, "schedule mode must be 0 (graph) or 2 (persistent)");
    if (k.mode == 2 && c->persist_grid < 1) return set_err(CMF_E_UNSUPPORTED, "the persistent kernel cannot run here");
    for (int b : {k.bf, k.br, k.bs})
        if (b % 32 || b < 64 || b > cmf::kCellThreads) return set_err(CMF_E_ARG, "block sizes must be multiples of 32 in [64, 256]");
    if (k.prof != 0 && k.prof != 1) return set_err(CMF_E_ARG, "profile must be 0 or 1");
    CUDA_TRY(cudaSetDevice(c->device));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->tune.active = false;
    c->tune.timed = 0;
    return apply_sched(c, k);
}

int cmf_gpu_ctx_stage(cmf_gpu_ctx *c, double dt_def, double *dt_min_local) {
    if (!c) return set_err(CMF_E_STATE, "no context");
    CUDA_TRY(cudaSetDevice(c->device));
    int rc;
    if ((rc = sync_dt_def(c, dt_def))) return rc;
    launch_stage(c);
    CUDA_TRY(cudaGetLastError());
    c->launches += 1;
    if ((rc = read_ctl(c))) return rc;
    unsigned long long def_bits;
    std::memcpy(&def_bits, &dt_def, sizeof def_bits);
    for (size_t m = 0; m < c->hctl.size(); m++) {
        double v;
        std::memcpy(&v, &c->hctl[m].dtmin_bits, sizeof v);
        if (dt_min_local) dt_min_local[m] = std::min(v, dt_def);
        c->hctl[m].dtmin_bits = def_bits;   // the next stage starts its minimum from DT again
    }
    CUDA_TRY(cudaMemcpyAsync(c->st.ctl, c->hctl.data(), c->hctl.size() * sizeof(cmf::MemberCtl), cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return CMF_OK;
}

int cmf_gpu_ctx_substeps(cmf_gpu_ctx *c, double dt_def, double dt_min_global, int32_t *nt_out, double *dt_out, cmf_budget *b) {
    if (!c) return set_err(CMF_E_STATE, "no context");
    CUDA_TRY(cudaSetDevice(c->device));
    // install the reduced minimum as the atomicMin result, then run NT/DT and the sub-steps
    for (auto &m : c->hctl) {
        unsigned long long bits;
        std::memcpy(&bits, &dt_min_global, sizeof bits);
        m.dtmin_bits = bits;
        m.dt_def = dt_def;
    }
    CUDA_TRY(cudaMemcpyAsync(c->st.ctl, c->hctl.data(), c->hctl.size() * sizeof(cmf::MemberCtl), cudaMemcpyHostToDevice, c->stream));
    c->dt_def_dev = dt_def;
    cmf::k_ntdt<<<1, 256, 0, c->stream>>>(c->net, c->st, c->cond, 0);
    CUDA_TRY(cudaGetLastError());
    cmf::LoopCtl lc;
    CUDA_TRY(cudaMemcpyAsync(&lc, c->st.loop, sizeof lc, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    for (int k = 0; k < lc.ntmax; k++) enqueue_substep(c, 0);
    enqueue_epilogue(c);
    CUDA_TRY(cudaGetLastError());
    c->launches += 2 + 3LL * lc.ntmax;
    const int saved = c->opts.launch_mode;
    c->opts.launch_mode = 1;
    int rc = finish_outer(c, nt_out, dt_out, b);
    c->opts.launch_mode = saved;
    return rc;
}

int cmf_gpu_ctx_get_diag(cmf_gpu_ctx *c, const cmf_diag_ptrs *p) {
    if (!c || !p) return set_err(CMF_E_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(c->device));
    const size_t MN = (size_t)c->dims.nmembers * c->dims.nseqall;
    int rc;
    for (const DiagField &x : diag_fields(c, p))
        if ((rc = d2h(c, x.dst, x.src, x.n))) return rc;
    // GDWRTN/ROFSUB are zero without groundwater delay or LROSPLIT (both refused)
    if (p->gdwrtn_aavg) std::memset(p->gdwrtn_aavg, 0, MN * sizeof(double));
    if (p->rofsub_aavg) std::memset(p->rofsub_aavg, 0, MN * sizeof(double));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return CMF_OK;
}

// The named diagnostics as they stand after the steps enqueued so far are copied on the device
// into staging buffers (ordered before any later step), then to the host buffers on the copy
// stream, overlapping the next step; cmf_gpu_ctx_io_wait blocks until they landed.
int cmf_gpu_ctx_get_diag_async(cmf_gpu_ctx *c, const cmf_diag_ptrs *p) {
    if (!c || !p) return set_err(CMF_E_ARG, "null argument");
    if (p->gdwrtn_aavg || p->rofsub_aavg) return set_err(CMF_E_ARG, "get_diag_async: GDWRTN/ROFSUB are not staged");
    CUDA_TRY(cudaSetDevice(c->device));
    int rc;
    if ((rc = io_setup(c))) return rc;
    if (c->ostage.empty()) c->ostage.assign(kDiagSlots, nullptr);
    const std::vector<DiagField> fs = diag_fields(c, p);
    // the staging buffers are free once the previous read-back landed
    CUDA_TRY(cudaStreamWaitEvent(c->stream, c->ev_out_done, 0));
    for (const DiagField &x : fs) {
        double *&st = c->ostage[x.slot];
        if (!st && (rc = c->alloc(&st, x.n))) return rc;
        CUDA_TRY(cudaMemcpyAsync(st, x.src, x.n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    }
    CUDA_TRY(cudaEventRecord(c->ev_out_staged, c->stream));
    CUDA_TRY(cudaStreamWaitEvent(c->io_out, c->ev_out_staged, 0));
    for (const DiagField &x : fs)
        CUDA_TRY(cudaMemcpyAsync(x.dst, c->ostage[x.slot], x.n * sizeof(double), cudaMemcpyDeviceToHost, c->io_out));
    CUDA_TRY(cudaEventRecord(c->ev_out_done, c->io_out));
    return CMF_OK;
}

int cmf_gpu_ctx_io_wait(cmf_gpu_ctx *c) {
    if (!c) return set_err(CMF_E_STATE, "no context");
    if (!c->io) return CMF_OK;
    CUDA_TRY(cudaSetDevice(c->device));
    CUDA_TRY(cudaStreamSynchronize(c->io_out));
    return CMF_OK;
}

// ---- default context (the Fortran shim) ----------------------------------------------------
int cmf_gpu_init(const cmf_dims *dims, const cmf_params *params, const cmf_map_ptrs *maps, const cmf_opts *opts) {
    if (g_default) { cmf_gpu_destroy(g_default); g_default = nullptr; }
    return cmf_gpu_create(dims, params, maps, opts, &g_default);
}
int cmf_gpu_set_state(const cmf_state_ptrs *st) {
    return g_default ? cmf_gpu_ctx_set_state(g_default, st) : set_err(CMF_E_STATE, "cmf_gpu_init not called");
}
int cmf_gpu_get_state(const cmf_state_ptrs *st) {
    return g_default ? cmf_gpu_ctx_get_state(g_default, st) : set_err(CMF_E_STATE, "cmf_gpu_init not called");
}
int cmf_gpu_put_runoff(const double *runoff, const double *rofsub) {
    return g_default ? cmf_gpu_ctx_put_runoff(g_default, runoff, rofsub) : set_err(CMF_E_STATE, "cmf_gpu_init not called");
}
int cmf_gpu_physics_advance(double dt_def, int32_t *nt_out, double *dt_out, cmf_budget *b) {
    return g_default ? cmf_gpu_ctx_physics_advance(g_default, dt_def, nt_out, dt_out, b)
                     : set_err(CMF_E_STATE, "cmf_gpu_init not called");
}
int cmf_gpu_get_diag(const cmf_diag_ptrs *dg) {
    return g_default ? cmf_gpu_ctx_get_diag(g_default, dg) : set_err(CMF_E_STATE, "cmf_gpu_init not called");
}
int cmf_gpu_diag_output(int32_t op) {
    return g_default ? cmf_gpu_ctx_diag_output(g_default, op) : set_err(CMF_E_STATE, "cmf_gpu_init not called");
}
int cmf_gpu_get_diag_output(const cmf_diag_out_ptrs *dg) {
    return g_default ? cmf_gpu_ctx_get_diag_output(g_default, dg) : set_err(CMF_E_STATE, "cmf_gpu_init not called");
}
void cmf_gpu_finalize(void) {
    if (g_default) cmf_gpu_destroy(g_default);
    g_default = nullptr;
}

}  // extern "C"

// ============================================================================================
// Stage scheme + CFL minimum without any allocation by the library.
//
// Some hosts cannot let a library call cudaMalloc: couplers that hand every byte of device
// memory to their own pool before the time loop starts, codes that run the physics while a
// stream is being captured (where an allocation would break the capture), or processes whose
// device memory is fully committed to other components.  This entry point serves them: the
// caller passes device pointers for every input and output, and the only global memory the
// library uses beyond those is the file-scope array below, which exists once per GPU for the
// lifetime of the process.
// ============================================================================================
namespace {

constexpr int kNoAllocBlock = 256;
constexpr int kNoAllocMaxBlocks = 8192;   // 8192 x 256 = 2,097,152 cells at most

// per-block CFL minima of the most recent call on this device (64 KiB)
static __device__ __align__(256) double g_noalloc_blockmin[kNoAllocMaxBlocks];

__global__ void k_noalloc_stage(cmf::Net n, cmf::State s, double *blockmin) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double key = 1.0e308;
    if (i < n.N) {
        const cmf::StageOut o = cmf::stage_def(n, cmf::OwnG{n, s}, i, s.rivsto[i], s.fldsto[i]);
        cmf::store_stage(n, s, i, i, o);
        if (n.ladpstp && n.i2mask[i] == 0)
            key = cmf::cfl_key(n.pcadp, (i < n.R) ? n.nxtdst[i] : n.pdstmth, n.pgrv, o.rivdph);
    }
    for (int o = 16; o > 0; o >>= 1) key = cmf::dmin(key, __shfl_down_sync(0xffffffffu, key, o));
    __shared__ double wmin[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if (lane == 0) wmin[warp] = key;
    __syncthreads();
    if (warp == 0) {
        double x = lane < nw ? wmin[lane] : 1.0e308;
        for (int o = 16; o > 0; o >>= 1) x = cmf::dmin(x, __shfl_down_sync(0xffffffffu, x, o));
        if (lane == 0) blockmin[blockIdx.x] = x;   // every block writes its slot on every call
    }
}

__global__ void k_noalloc_min(const double *blockmin, int nblocks, double dt_def, double *dt_min_out) {
    double x = 1.0e308;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) x = cmf::dmin(x, blockmin[b]);
    for (int o = 16; o > 0; o >>= 1) x = cmf::dmin(x, __shfl_down_sync(0xffffffffu, x, o));
    __shared__ double wmin[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if (lane == 0) wmin[warp] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = 1.0e308;
        for (int w = 0; w < nw; w++) v = cmf::dmin(v, wmin[w]);
        *dt_min_out = cmf::dmin(dt_def, v);
    }
}

// device address of g_noalloc_blockmin, looked up once per device
double *g_noalloc_ptr[64] = {};

}  // namespace

extern "C" int cmf_gpu_stage_noalloc(const cmf_stage_dev_args *a) {
    if (!a || !a->rivsto || !a->fldsto || !a->rivstomax || !a->rivlen || !a->rivwth || !a->grarea || !a->rivelv ||
        !a->nxtdst || !a->fldstomax || !a->fldgrd || !a->i2mask || !a->rivdph || !a->flddph || !a->fldfrc ||
        !a->fldare || !a->sfcelv || !a->storge || !a->dt_min_out)
        return set_err(CMF_E_ARG, "cmf_gpu_stage_noalloc: null pointer in arguments");
    if (a->nseqall <= 0 || a->nseqriv < 0 || a->nseqriv > a->nseqall || a->nlfp <= 0 || !(a->dt_def > 0.0))
        return set_err(CMF_E_ARG, "cmf_gpu_stage_noalloc: bad dimensions or DT");
    const int nblocks = (a->nseqall + kNoAllocBlock - 1) / kNoAllocBlock;
    if (nblocks > kNoAllocMaxBlocks)
        return set_err(CMF_E_ARG, "cmf_gpu_stage_noalloc: NSEQALL=" + std::to_string(a->nseqall) +
                                      " exceeds the scratch limit of " + std::to_string(kNoAllocMaxBlocks * kNoAllocBlock) +
                                      " cells; use the context API (cmf_gpu_ctx_stage) for larger domains");
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return set_err(CMF_E_NO_DEVICE, "cmf_gpu_stage_noalloc: device ordinal above 63");
    if (!g_noalloc_ptr[dev]) {
        // set-up on the first call per device (the device must be current); no allocation happens here
        void *p = nullptr;
        CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_blockmin));
        g_noalloc_ptr[dev] = static_cast<double *>(p);
    }
    cmf::Net n{};
    n.N = a->nseqall; n.R = a->nseqriv; n.L = a->nlfp; n.M = 1;
    n.i2mask = a->i2mask; n.rivelv = a->rivelv; n.nxtdst = a->nxtdst; n.rivwth = a->rivwth; n.rivlen = a->rivlen;
    n.grarea = a->grarea; n.rivstomax = a->rivstomax; n.fldstomax = a->fldstomax; n.fldgrd = a->fldgrd;
    n.pgrv = a->pgrv; n.pdstmth = a->pdstmth; n.pcadp = a->pcadp; n.dfrcinc = a->dfrcinc; n.ladpstp = a->ladpstp;
    n.llevee = 0;
    cmf::State s{};
    s.rivsto = a->rivsto; s.fldsto = a->fldsto; s.rivdph = a->rivdph; s.flddph = a->flddph; s.fldfrc = a->fldfrc;
    s.fldare = a->fldare; s.sfcelv = a->sfcelv; s.storge = a->storge;
    cudaStream_t st = static_cast<cudaStream_t>(a->stream);
    k_noalloc_stage<<<nblocks, kNoAllocBlock, 0, st>>>(n, s, g_noalloc_ptr[dev]);
    CUDA_TRY(cudaGetLastError());
    k_noalloc_min<<<1, 256, 0, st>>>(g_noalloc_ptr[dev], nblocks, a->dt_def, a->dt_min_out);
    CUDA_TRY(cudaGetLastError());
    return CMF_OK;
}
