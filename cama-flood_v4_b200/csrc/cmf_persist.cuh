// cmf_persist.cuh -- one persistent, cooperative launch per outer step (CMF_PHYSICS_ADVANCE,
// src/cmf_ctrl_physics_mod.F90:21-153) on sm_100a.
//
// The grid is exactly the set of CTAs that are resident at once (cudaLaunchCooperativeKernel); the
// grid-wide dependencies of the step are software grid barriers:
//   stage + CFL minimum | NT/DT (CTA 0) | NT x { flux | rate | store } | budgets
// Every CTA owns a contiguous range of cell tiles (TILE cells of one member) and path tiles.  In the
// three sub-step phases the own-cell arrays of the next tile are fetched into shared memory by bulk
// asynchronous copies (cp.async.bulk, completion on an mbarrier) while the current tile computes, so
// the latency of the streamed loads overlaps the arithmetic; reads of other cells (downstream,
// upstream, path ends) stay plain loads through L2.  The per-cell arithmetic is the same code as
// the phase kernels (cmf_kernels.cuh) with a shared-memory accessor, so the results are identical
// bit for bit.
//
// Barriers spin on a counter in global memory with a bound: a CTA that waits longer than the bound
// sets LoopCtl.bar_err and every CTA leaves the kernel at its next barrier, so a wait that cannot end
// returns an error status to the host instead of holding the GPU.
#pragma once
#include "cmf_kernels.cuh"

namespace cmf {

constexpr int kTile = 256;                      // cells per tile == threads per CTA
constexpr int kDSlot = kTile + 2;               // doubles per tile slot (alignment slack, 16-byte multiple)
constexpr int kISlot = kTile + 8;               // ints per tile slot (alignment slack + up_ptr's extra entry)
constexpr unsigned long long kWaitNsDefault = 1000000000ull;   // bound of every device-side wait: 1 s

// tile slots of each phase (doubles: member state then static maps; ints)
enum SlotA { A_RIVDPH, A_RIVDPH_PRE, A_RIVOUT_PRE, A_FLDSTO, A_FLDDPH, A_FLDSTO_PRE, A_FLDOUT_PRE, A_STORGE, A_A_RIVVEL,
             A_NSTATE, A_RIVELV = A_NSTATE, A_RIVHGT, A_RIVWTH, A_RIVMAN, A_INV_NXTDST, A_INV_RIVLEN, A_ELEVTN,
             A_INV_RIVWTH, A_ND };
enum SlotAI { AI_NEXT, AI_I1DAM, A_NI };
enum SlotB { B_RIVOUT_RAW, B_FLDOUT_RAW, B_RIVSTO, B_FLDSTO, B_ND, B_NSTATE = B_ND };
enum SlotBI { BI_UP, B_NI };
enum SlotC { C_RATE, C_RIVOUT_RAW, C_FLDOUT_RAW, C_RUNOFF, C_RIVSTO, C_FLDSTO, C_RIVDPH, C_FLDFRC, C_LEVSTO,
             C_A_RIVOUT, C_A_FLDOUT, C_A_OUTFLW, C_A_PTHOUT, C_M_OUTFLW, C_M_RIVDPH, C_M_STORGE,
             C_NSTATE, C_RIVSTOMAX = C_NSTATE, C_RIVLEN, C_RIVWTH, C_GRAREA, C_ND };
enum SlotCI { CI_NEXT, CI_UP, C_NI };
constexpr int kMaxD = ((int)A_ND > (int)C_ND ? (int)A_ND : (int)C_ND);
constexpr int kMaxI = 2;
constexpr size_t kStageBytes = (size_t)kMaxD * kDSlot * 8 + (size_t)kMaxI * kISlot * 4;
constexpr int kStages = 2;
// dynamic shared memory: the stages and their mbarriers (two CTAs fit on an SM)
constexpr size_t kPersistSmem = kStages * kStageBytes + 64;

// ---- PTX helpers -----------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// global -> shared bulk copy (no multicast); dst, src 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async;" ::: "memory"); }
__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Software grid barrier over the `nblocks` co-resident CTAs of a cooperative launch: arrival
// count in LoopCtl.bar (zeroed by the host before each launch), barrier e of the launch completes
// when the count reaches nblocks * e.  The wait is bounded in time (wait_ns); a CTA that gives up
// sets the error word, and every CTA polling a barrier leaves as soon as it sees the word, so all
// CTAs return within about one bound.  Returns false (uniformly across the CTA) on failure.
struct GridBar {
    unsigned *count;
    int *err;
    unsigned nblocks, epoch;
    unsigned long long wait_ns;
    int *sflag;          // shared-memory broadcast of the outcome
    __device__ __forceinline__ bool sync() {
        epoch++;
        // order this thread's global writes before the async-proxy (bulk copy) reads of other CTAs
        fence_proxy_async();
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(count, 1u);
            const unsigned target = nblocks * epoch;
            const unsigned long long t0 = globaltimer_ns();
            int ok = 1;
            while (ld_acquire(count) < target) {
                if (*(volatile int *)err) { ok = 0; break; }
                if (globaltimer_ns() - t0 > wait_ns) {
                    atomicExch(err, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
            __threadfence();
            *sflag = ok;
        }
        __syncthreads();
        return *(volatile int *)sflag != 0;
    }
};

// ---- tiles -----------------------------------------------------------------------------------
struct TileGeom {
    int m, i0, i1;              // member, cells [i0, i1)
    int j;                      // tile index within the member
};
__device__ __forceinline__ TileGeom tile_geom(int t, int tpm, int N) {
    TileGeom g;
    g.m = t / tpm;
    g.j = t - g.m * tpm;
    g.i0 = g.j * kTile;
    g.i1 = min(g.i0 + kTile, N);
    return g;
}

// Shared-memory accessors: element e of slot k lives at slot[k][e - base], with the base the first
// element of the 16-byte aligned range the bulk copy fetched (member state by g = m*N + i, statics
// and ints by i).
struct TileView {
    const double *d;
    const int *iv;
    long long gbase;            // first state element in the slots
    int sbase;                  // first static element
    int ibase;                  // first int element
    __device__ __forceinline__ double st(int k, size_t g) const { return d[k * kDSlot + (long long)g - gbase]; }
    __device__ __forceinline__ double sx(int k, int i) const { return d[k * kDSlot + i - sbase]; }
    __device__ __forceinline__ int ix(int k, int i) const { return iv[k * kISlot + i - ibase]; }
};

struct OwnTA {
    TileView v;
    const Net &n;
    __device__ __forceinline__ double rivelv(int i) const { return v.sx(A_RIVELV, i); }
    __device__ __forceinline__ double rivhgt(int i) const { return v.sx(A_RIVHGT, i); }
    __device__ __forceinline__ double rivwth(int i) const { return v.sx(A_RIVWTH, i); }
    __device__ __forceinline__ double rivman(int i) const { return v.sx(A_RIVMAN, i); }
    __device__ __forceinline__ double inv_nxtdst(int i) const { return v.sx(A_INV_NXTDST, i); }
    __device__ __forceinline__ double inv_rivlen(int i) const { return v.sx(A_INV_RIVLEN, i); }
    __device__ __forceinline__ double inv_rivwth(int i) const { return v.sx(A_INV_RIVWTH, i); }
    __device__ __forceinline__ double elevtn(int i) const { return v.sx(A_ELEVTN, i); }
    __device__ __forceinline__ int next(int i) const { return v.ix(AI_NEXT, i); }
    __device__ __forceinline__ int i1dam(int i) const { return v.ix(AI_I1DAM, i); }
    __device__ __forceinline__ double rivdph(size_t g) const { return v.st(A_RIVDPH, g); }
    __device__ __forceinline__ double rivdph_pre(size_t g) const { return v.st(A_RIVDPH_PRE, g); }
    __device__ __forceinline__ double rivout_pre(size_t g) const { return v.st(A_RIVOUT_PRE, g); }
    __device__ __forceinline__ double fldsto(size_t g) const { return v.st(A_FLDSTO, g); }
    __device__ __forceinline__ double flddph(size_t g) const { return v.st(A_FLDDPH, g); }
    __device__ __forceinline__ double fldsto_pre(size_t g) const { return v.st(A_FLDSTO_PRE, g); }
    __device__ __forceinline__ double fldout_pre(size_t g) const { return v.st(A_FLDOUT_PRE, g); }
    __device__ __forceinline__ double storge(size_t g) const { return v.st(A_STORGE, g); }
    __device__ __forceinline__ double a_rivvel(size_t g) const { return v.st(A_A_RIVVEL, g); }
};
struct OwnTB {
    TileView v;
    __device__ __forceinline__ int up_lo(int i) const { return v.ix(BI_UP, i); }
    __device__ __forceinline__ int up_hi(int i) const { return v.ix(BI_UP, i + 1); }
    __device__ __forceinline__ double rivout_raw(size_t g) const { return v.st(B_RIVOUT_RAW, g); }
    __device__ __forceinline__ double fldout_raw(size_t g) const { return v.st(B_FLDOUT_RAW, g); }
    __device__ __forceinline__ double rivsto(size_t g) const { return v.st(B_RIVSTO, g); }
    __device__ __forceinline__ double fldsto(size_t g) const { return v.st(B_FLDSTO, g); }
};
struct OwnTC {
    TileView v;
    __device__ __forceinline__ double rivstomax(int i) const { return v.sx(C_RIVSTOMAX, i); }
    __device__ __forceinline__ double rivlen(int i) const { return v.sx(C_RIVLEN, i); }
    __device__ __forceinline__ double rivwth(int i) const { return v.sx(C_RIVWTH, i); }
    __device__ __forceinline__ double grarea(int i) const { return v.sx(C_GRAREA, i); }
    __device__ __forceinline__ int next(int i) const { return v.ix(CI_NEXT, i); }
    __device__ __forceinline__ int up_lo(int i) const { return v.ix(CI_UP, i); }
    __device__ __forceinline__ int up_hi(int i) const { return v.ix(CI_UP, i + 1); }
    __device__ __forceinline__ double rate(size_t g) const { return v.st(C_RATE, g); }
    __device__ __forceinline__ double rivout_raw(size_t g) const { return v.st(C_RIVOUT_RAW, g); }
    __device__ __forceinline__ double fldout_raw(size_t g) const { return v.st(C_FLDOUT_RAW, g); }
    __device__ __forceinline__ double runoff(size_t g) const { return v.st(C_RUNOFF, g); }
    __device__ __forceinline__ double rivsto(size_t g) const { return v.st(C_RIVSTO, g); }
    __device__ __forceinline__ double fldsto(size_t g) const { return v.st(C_FLDSTO, g); }
    __device__ __forceinline__ double rivdph(size_t g) const { return v.st(C_RIVDPH, g); }
    __device__ __forceinline__ double fldfrc(size_t g) const { return v.st(C_FLDFRC, g); }
    __device__ __forceinline__ double levsto(size_t g) const { return v.st(C_LEVSTO, g); }
    __device__ __forceinline__ double a_rivout(size_t g) const { return v.st(C_A_RIVOUT, g); }
    __device__ __forceinline__ double a_fldout(size_t g) const { return v.st(C_A_FLDOUT, g); }
    __device__ __forceinline__ double a_outflw(size_t g) const { return v.st(C_A_OUTFLW, g); }
    __device__ __forceinline__ double a_pthout(size_t g) const { return v.st(C_A_PTHOUT, g); }
    __device__ __forceinline__ double m_outflw(size_t g) const { return v.st(C_M_OUTFLW, g); }
    __device__ __forceinline__ double m_rivdph(size_t g) const { return v.st(C_M_RIVDPH, g); }
    __device__ __forceinline__ double m_storge(size_t g) const { return v.st(C_M_STORGE, g); }
};

// The arrays a phase streams, in slot order: member-state arrays [M][N] (index g), static maps [N]
// (index i), int maps.  A null pointer leaves its slot unfetched (an option that is off).
struct PhaseArrays {
    const double *st[C_NSTATE];
    const double *sx[4 + 7];
    const int *iv[kMaxI];
    int nst, nsx, niv;
    int iv_extra;               // extra trailing int element per tile (up_ptr[i1])
};

// Issues the bulk copies of one tile into one stage buffer; called by one thread.
__device__ __forceinline__ void issue_tile(const PhaseArrays &pa, const TileGeom &tg, int N, double *d, int *iv,
                                           unsigned long long *bar) {
    const long long g0 = (long long)tg.m * N + tg.i0, g1 = (long long)tg.m * N + tg.i1;
    const long long ga = g0 & ~1LL, gb = (g1 + 1) & ~1LL;
    const int sa = tg.i0 & ~1, sb = (tg.i1 + 1) & ~1;
    const int ia = tg.i0 & ~3, ib = (tg.i1 + pa.iv_extra + 3) & ~3;
    unsigned bytes = 0;
    for (int k = 0; k < pa.nst; k++)
        if (pa.st[k]) bytes += (unsigned)(gb - ga) * 8u;
    for (int k = 0; k < pa.nsx; k++)
        if (pa.sx[k]) bytes += (unsigned)(sb - sa) * 8u;
    for (int k = 0; k < pa.niv; k++)
        if (pa.iv[k]) bytes += (unsigned)(ib - ia) * 4u;
    mbar_expect_tx(bar, bytes);
    for (int k = 0; k < pa.nst; k++)
        if (pa.st[k]) bulk_g2s(d + k * kDSlot, pa.st[k] + ga, (unsigned)(gb - ga) * 8u, bar);
    for (int k = 0; k < pa.nsx; k++)
        if (pa.sx[k]) bulk_g2s(d + (pa.nst + k) * kDSlot, pa.sx[k] + sa, (unsigned)(sb - sa) * 8u, bar);
    for (int k = 0; k < pa.niv; k++)
        if (pa.iv[k]) bulk_g2s(iv + k * kISlot, pa.iv[k] + ia, (unsigned)(ib - ia) * 4u, bar);
}

__device__ __forceinline__ TileView tile_view(const TileGeom &tg, int N, const double *d, const int *iv) {
    TileView v;
    v.d = d;
    v.iv = iv;
    v.gbase = ((long long)tg.m * N + tg.i0) & ~1LL;
    v.sbase = tg.i0 & ~1;
    v.ibase = tg.i0 & ~3;
    return v;
}

struct PersistArgs {
    int tpm;                    // cell tiles per member (ceil(N / kTile))
    int ppm;                    // path tiles per member (ceil(P / kTile))
    unsigned long long wait_ns; // bound of every device-side wait
    int selftest;               // 1: only run a barrier whose count can never complete (timeout check)
};

// The pipelined loop over this CTA's cell tiles of one phase.  `active(m)` says whether member m
// works on this sub-step; `body(tg, view)` computes one tile.  Stage bookkeeping (`use`, `nxt`) is
// uniform across the CTA and carries over from phase to phase.
struct Pipe {
    double *dbuf[kStages];
    int *ibuf[kStages];
    unsigned long long *bar;    // [kStages]
    unsigned use[kStages];
    int nxt;
};

// Bounded wait for stage `st`'s bytes, by every thread; false (uniformly) when the bound ran out.
__device__ __forceinline__ bool stage_wait(Pipe &pp, int st, unsigned long long wait_ns) {
    const unsigned long long t0 = globaltimer_ns();
    int ok = 1;
    while (!mbar_try_wait(&pp.bar[st], pp.use[st] & 1u)) {
        if (globaltimer_ns() - t0 > wait_ns) { ok = 0; break; }
    }
    return __syncthreads_and(ok) != 0;
}

template <class Active, class Body>
__device__ __forceinline__ bool run_cell_phase(Pipe &pp, const PhaseArrays &pa, int t0, int t1, int tpm, int N,
                                               LoopCtl *loop, unsigned long long wait_ns, Active active, Body body) {
    auto next_active = [&](int t) {
        while (t < t1 && !active(t / tpm)) t++;
        return t;
    };
    int t = next_active(t0);
    if (t >= t1) return true;
    int cur = pp.nxt;
    if (threadIdx.x == 0) issue_tile(pa, tile_geom(t, tpm, N), N, pp.dbuf[cur], pp.ibuf[cur], &pp.bar[cur]);
    pp.nxt ^= 1;
    while (t < t1) {
        const int tn = next_active(t + 1);
        const int other = pp.nxt;
        if (tn < t1) {
            if (threadIdx.x == 0) {
                fence_proxy_async();
                issue_tile(pa, tile_geom(tn, tpm, N), N, pp.dbuf[other], pp.ibuf[other], &pp.bar[other]);
            }
            pp.nxt ^= 1;
        }
        // wait for the current tile's bytes (bounded: a copy that never lands sets the error word;
        // the other stage's copy, if one was issued, is then waited for with the same bound)
        if (!stage_wait(pp, cur, wait_ns)) {
            if (threadIdx.x == 0) atomicExch(&loop->bar_err, 2);
            if (tn < t1) stage_wait(pp, other, wait_ns);
            return false;
        }
        pp.use[cur]++;
        const TileGeom tg = tile_geom(t, tpm, N);
        body(tg, tile_view(tg, N, pp.dbuf[cur], pp.ibuf[cur]));
        __syncthreads();
        t = tn;
        cur = other;
    }
    return true;
}

__device__ __forceinline__ void budget_reduce(const Net &n, const State &s, int m, int k) {
    // k_budget's tree (kBudgetThreads == kTile threads): the same sums as the phase-kernel path
    if (s.ctl[m].nt < 1) return;
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
        if (k == 0 && n.ldiag_out) s.o_nadd[m] = s.o_nadd[m] + s.ctl[m].dt_def;
    }
    __syncthreads();
}

// k_ntdt's per-member NT/DT and loop bound, run by one CTA of the persistent grid
__device__ __forceinline__ void ntdt_block(const Net &n, const State &s) {
    __shared__ int smax[32];
    __shared__ long long ssum[32], snear[32];
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
                c.err = kErrNtCap;
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
    for (int o = 16; o > 0; o >>= 1) {
        ntmax = max(ntmax, __shfl_down_sync(0xffffffffu, ntmax, o));
        ntsum += __shfl_down_sync(0xffffffffu, ntsum, o);
        near += __shfl_down_sync(0xffffffffu, near, o);
    }
    if ((threadIdx.x & 31) == 0) {
        smax[threadIdx.x >> 5] = ntmax;
        ssum[threadIdx.x >> 5] = ntsum;
        snear[threadIdx.x >> 5] = near;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int v = 1;
        long long tot = 0, nr = 0;
        for (int w = 0; w < (int)((blockDim.x + 31) >> 5); w++) {
            v = max(v, smax[w]);
            tot += ssum[w];
            nr += snear[w];
        }
        v = min(v, kNtCap);
        s.loop->ntmax = v;
        s.loop->near_int += nr;
        s.loop->member_substeps += tot;
        s.loop->loop_iters += v;
        s.loop->outer_steps += 1;
    }
}

__global__ void __launch_bounds__(kTile, 2) k_persist(Net n, State s, PersistArgs pa) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ int sflag;
    const unsigned G = gridDim.x, b = blockIdx.x;
    GridBar gb{&s.loop->bar, &s.loop->bar_err, G, 0u, pa.wait_ns, &sflag};
    if (pa.selftest) {
        // barrier timeout check: the count target includes one arrival that never comes
        gb.nblocks = G + 1;
        gb.sync();
        return;
    }
    const int N = n.N, M = n.M, tpm = pa.tpm, ppm = pa.ppm;
    const int T = M * tpm, PT = M * ppm;
    const int t0 = (int)(((long long)T * b) / G), t1 = (int)(((long long)T * (b + 1)) / G);
    const int p0 = (int)(((long long)PT * b) / G), p1 = (int)(((long long)PT * (b + 1)) / G);
    const bool split = s.loop->split != 0;

    Pipe pp;
    for (int k = 0; k < kStages; k++) {
        pp.dbuf[k] = reinterpret_cast<double *>(smem + k * kStageBytes);
        pp.ibuf[k] = reinterpret_cast<int *>(smem + k * kStageBytes + (size_t)kMaxD * kDSlot * 8);
        pp.use[k] = 0;
    }
    pp.bar = reinterpret_cast<unsigned long long *>(smem + kStages * kStageBytes);
    pp.nxt = 0;
    if (threadIdx.x == 0) {
        for (int k = 0; k < kStages; k++) mbar_init(&pp.bar[k], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    // ---- stage scheme at the top of the step + CALC_ADPSTP minimum (k_stage)
    for (int t = t0; t < t1; t++) {
        const TileGeom tg = tile_geom(t, tpm, N);
        const int i = tg.i0 + threadIdx.x;
        double key = 1.0e308;
        if (i < tg.i1) {
            const size_t gi = (size_t)tg.m * N + i;
            const OwnG w{n, s};
            const StageOut o = n.llevee ? stage_levee(n, w, i, s.rivsto[gi], s.fldsto[gi], s.levsto[gi])
                                        : stage_def(n, w, i, s.rivsto[gi], s.fldsto[gi]);
            store_stage(n, s, gi, i, o);
            if (n.ladpstp && __ldg(&n.i2mask[i]) == 0) key = cfl_key(n.pcadp, (i < n.R) ? __ldg(&n.nxtdst[i]) : n.pdstmth, n.pgrv, o.rivdph);
        }
        if (n.ladpstp) {
            for (int o = 16; o > 0; o >>= 1) key = dmin(key, __shfl_down_sync(0xffffffffu, key, o));
            __shared__ double wmin[32];
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
            if (lane == 0) wmin[warp] = key;
            __syncthreads();
            if (warp == 0) {
                double x = lane < (kTile / 32) ? wmin[lane] : 1.0e308;
                for (int o = 16; o > 0; o >>= 1) x = dmin(x, __shfl_down_sync(0xffffffffu, x, o));
                if (lane == 0 && x < 1.0e308)
                    atomicMin(&s.ctl[tg.m].dtmin_bits, (unsigned long long)__double_as_longlong(x));
            }
            __syncthreads();
        }
    }
    if (!gb.sync()) return;
    if (b == 0) ntdt_block(n, s);
    if (!gb.sync()) return;
    const int ntmax = s.loop->ntmax;

    // ---- arrays each phase streams
    PhaseArrays fa{}, ra{}, sa{};
    fa.nst = A_NSTATE; fa.nsx = A_ND - A_NSTATE; fa.niv = A_NI; fa.iv_extra = 0;
    fa.st[A_RIVDPH] = s.rivdph; fa.st[A_RIVDPH_PRE] = s.rivdph_pre; fa.st[A_RIVOUT_PRE] = s.rivout_pre;
    fa.st[A_FLDSTO] = s.fldsto; fa.st[A_FLDDPH] = s.flddph; fa.st[A_FLDSTO_PRE] = s.fldsto_pre;
    fa.st[A_FLDOUT_PRE] = s.fldout_pre; fa.st[A_STORGE] = s.storge; fa.st[A_A_RIVVEL] = n.ldiag ? s.a_rivvel : nullptr;
    fa.sx[A_RIVELV - A_NSTATE] = n.rivelv; fa.sx[A_RIVHGT - A_NSTATE] = n.rivhgt; fa.sx[A_RIVWTH - A_NSTATE] = n.rivwth;
    fa.sx[A_RIVMAN - A_NSTATE] = n.rivman; fa.sx[A_INV_NXTDST - A_NSTATE] = n.inv_nxtdst;
    fa.sx[A_INV_RIVLEN - A_NSTATE] = n.inv_rivlen; fa.sx[A_ELEVTN - A_NSTATE] = n.elevtn;
    fa.sx[A_INV_RIVWTH - A_NSTATE] = n.inv_rivwth;
    fa.iv[AI_NEXT] = n.next; fa.iv[AI_I1DAM] = n.ldamout ? n.i1dam : nullptr;
    ra.nst = B_NSTATE; ra.nsx = 0; ra.niv = B_NI; ra.iv_extra = 1;
    ra.st[B_RIVOUT_RAW] = s.rivout_raw; ra.st[B_FLDOUT_RAW] = s.fldout_raw; ra.st[B_RIVSTO] = s.rivsto;
    ra.st[B_FLDSTO] = s.fldsto;
    ra.iv[BI_UP] = n.up_ptr;
    sa.nst = C_NSTATE; sa.nsx = C_ND - C_NSTATE; sa.niv = C_NI; sa.iv_extra = 1;
    sa.st[C_RATE] = s.rate; sa.st[C_RIVOUT_RAW] = s.rivout_raw; sa.st[C_FLDOUT_RAW] = s.fldout_raw;
    sa.st[C_RUNOFF] = s.runoff; sa.st[C_RIVSTO] = s.rivsto; sa.st[C_FLDSTO] = s.fldsto; sa.st[C_RIVDPH] = s.rivdph;
    sa.st[C_FLDFRC] = s.fldfrc; sa.st[C_LEVSTO] = n.llevee ? s.levsto : nullptr;
    sa.st[C_A_RIVOUT] = n.ldiag ? s.a_rivout : nullptr; sa.st[C_A_FLDOUT] = n.ldiag ? s.a_fldout : nullptr;
    sa.st[C_A_OUTFLW] = n.ldiag ? s.a_outflw : nullptr; sa.st[C_A_PTHOUT] = n.ldiag ? s.a_pthout : nullptr;
    sa.st[C_M_OUTFLW] = n.ldiag ? s.m_outflw : nullptr; sa.st[C_M_RIVDPH] = n.ldiag ? s.m_rivdph : nullptr;
    sa.st[C_M_STORGE] = n.ldiag ? s.m_storge : nullptr;
    sa.sx[C_RIVSTOMAX - C_NSTATE] = n.rivstomax; sa.sx[C_RIVLEN - C_NSTATE] = n.rivlen;
    sa.sx[C_RIVWTH - C_NSTATE] = n.rivwth; sa.sx[C_GRAREA - C_NSTATE] = n.grarea;
    sa.iv[CI_NEXT] = n.next; sa.iv[CI_UP] = n.up_ptr;

    for (int k = 0; k < ntmax; k++) {
        auto active = [&](int m) { return k < s.ctl[m].nt; };
        // ---- phase A: outflow + dam + bifurcation flux
        if (!run_cell_phase(pp, fa, t0, t1, tpm, N, s.loop, pa.wait_ns, active, [&](const TileGeom &tg, const TileView &v) {
                const int i = tg.i0 + threadIdx.x;
                if (i < tg.i1) {
                    const MemberCtl &c = s.ctl[tg.m];
                    cell_outflow(n, s, OwnTA{v, n}, tg.m, i, c.dt, c, k, split && k == 0);
                }
            }))
            return;
        for (int t = p0; t < p1; t++) {
            const int m = t / ppm, p = (t - m * ppm) * kTile + threadIdx.x;
            if (k < s.ctl[m].nt && p < n.P) path_outflow(n, s, m, p, s.ctl[m].dt);
        }
        if (!gb.sync()) return;
        // ---- phase B: storage-out gather and rate
        if (!run_cell_phase(pp, ra, t0, t1, tpm, N, s.loop, pa.wait_ns, active, [&](const TileGeom &tg, const TileView &v) {
                const int i = tg.i0 + threadIdx.x;
                if (i < tg.i1) cell_rate(n, s, OwnTB{v}, tg.m, i, s.ctl[tg.m].dt);
            }))
            return;
        if (!gb.sync()) return;
        // ---- phase C: rescale, inflow, STONXT, stage scheme, diagnostics
        if (!run_cell_phase(pp, sa, t0, t1, tpm, N, s.loop, pa.wait_ns, active, [&](const TileGeom &tg, const TileView &v) {
                const MemberCtl &c = s.ctl[tg.m];
                const double DT = c.dt;
                const bool first = (k == 0), last = (k == c.nt - 1);
                const double nadd = last ? nadd_before(k, DT) : 0.0;
                const int i = tg.i0 + threadIdx.x;
                // the last sub-step's budget terms stay in registers (128 per thread at this occupancy)
                double bl[kBudgets];
#pragma unroll
                for (int q = 0; q < kBudgets; q++) bl[q] = 0.0;
                auto bput = [&](int q, double val) { if (last) bl[q] = val; };
                if (i < tg.i1) cell_store(n, s, OwnTC{v}, tg.m, i, DT, first, last, nadd, c, bput);
                if (last) warp_budget_partials(s, tg.m, i >> 5, budget_warps(N), bl);
            }))
            return;
        for (int t = p0; t < p1; t++) {
            const int m = t / ppm, p = (t - m * ppm) * kTile + threadIdx.x;
            const MemberCtl &c = s.ctl[m];
            if (k < c.nt && p < n.P) {
                const double DT = c.dt;
                const bool last = (k == c.nt - 1);
                path_rescale(n, s, m, p, DT, k == 0, last, last ? nadd_before(k, DT) : 0.0, c.dt_def);
            }
        }
        if (!gb.sync()) return;
    }
    // ---- budgets of every member's last sub-step (k_budget)
    for (int r = b; r < M * kBudgets; r += G) budget_reduce(n, s, r / kBudgets, r % kBudgets);
    if (b == 0 && threadIdx.x == 0) s.loop->split = 0;
}

}  // namespace cmf
