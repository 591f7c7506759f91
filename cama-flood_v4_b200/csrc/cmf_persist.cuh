// cmf_persist.cuh -- one persistent, cooperative launch per outer step (CMF_PHYSICS_ADVANCE,
// src/cmf_ctrl_physics_mod.F90:21-153) on sm_100a.
//
// The grid is exactly the set of CTAs that are resident at once (cudaLaunchCooperativeKernel); the
// grid-wide dependencies of the step are software grid barriers:
//   stage + CFL minimum | NT/DT (CTA 0) | NT x { flux | rate | store } | budgets
// Work is cut into tiles of kTile cells of one member (and kTile bifurcation paths); CTA b takes
// tiles b, b + G, b + 2G, ... of every phase, so the costly tiles (flooded cells near the mouths,
// levees, dams) spread over all CTAs.  The per-cell arithmetic is the phase kernels' own code
// (cmf_kernels.cuh, global-memory accessor), so the results are identical bit for bit.
//
// Barriers spin on a counter in global memory with a bound: a CTA that waits longer than the bound
// sets LoopCtl.bar_err and every CTA leaves the kernel at its next barrier, so a wait that cannot end
// returns an error status to the host instead of holding the GPU.
#pragma once
#include "cmf_kernels.cuh"

namespace cmf {

constexpr int kTile = 256;                      // cells (or paths) per tile == threads per CTA
constexpr int kPersistMinBlocks = 3;            // 80 registers: fewer spills beat a fourth CTA per SM
constexpr unsigned long long kWaitNsDefault = 1000000000ull;   // bound of every device-side wait: 1 s
// dynamic shared memory: the last sub-step's budget terms of the tile, kBudgets per thread
constexpr size_t kPersistSmem = (size_t)kBudgets * kTile * sizeof(double);

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

struct TileGeom {
    int m, i0, i1;              // member, cells [i0, i1)
};
__device__ __forceinline__ TileGeom tile_geom(int t, int tpm, int N) {
    TileGeom g;
    g.m = t / tpm;
    g.i0 = (t - g.m * tpm) * kTile;
    g.i1 = min(g.i0 + kTile, N);
    return g;
}

struct PersistArgs {
    int tpm;                    // cell tiles per member (ceil(N / kTile))
    int ppm;                    // path tiles per member (ceil(P / kTile))
    unsigned long long wait_ns; // bound of every device-side wait
    int selftest;               // 1: only run a barrier whose count can never complete (timeout check)
};

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

__global__ void __launch_bounds__(kTile, kPersistMinBlocks) k_persist(Net n, State s, PersistArgs pa) {
    extern __shared__ __align__(16) unsigned char smem[];
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
    const bool split = s.loop->split != 0;
    double *sbud = reinterpret_cast<double *>(smem);

    // ---- stage scheme at the top of the step + CALC_ADPSTP minimum (k_stage)
    for (int t = b; t < T; t += G) {
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

    for (int k = 0; k < ntmax; k++) {
        // ---- phase A: outflow + dam + bifurcation flux (cell tiles, then path tiles)
        for (int t = b; t < T + PT; t += G) {
            if (t < T) {
                const TileGeom tg = tile_geom(t, tpm, N);
                const MemberCtl &c = s.ctl[tg.m];
                const int i = tg.i0 + threadIdx.x;
                if (k < c.nt && i < tg.i1) cell_outflow(n, s, OwnG{n, s}, tg.m, i, c.dt, c, k, split && k == 0);
            } else {
                const int q = t - T, m = q / ppm, p = (q - m * ppm) * kTile + threadIdx.x;
                if (k < s.ctl[m].nt && p < n.P) path_outflow(n, s, m, p, s.ctl[m].dt);
            }
        }
        if (!gb.sync()) return;
        // ---- phase B: storage-out gather and rate
        for (int t = b; t < T; t += G) {
            const TileGeom tg = tile_geom(t, tpm, N);
            const int i = tg.i0 + threadIdx.x;
            if (k < s.ctl[tg.m].nt && i < tg.i1) cell_rate(n, s, OwnG{n, s}, tg.m, i, s.ctl[tg.m].dt);
        }
        if (!gb.sync()) return;
        // ---- phase C: rescale, inflow, STONXT, stage scheme, diagnostics; path rescale
        for (int t = b; t < T + PT; t += G) {
            if (t < T) {
                const TileGeom tg = tile_geom(t, tpm, N);
                const MemberCtl &c = s.ctl[tg.m];
                if (k >= c.nt) continue;   // uniform over the CTA
                const double DT = c.dt;
                const bool first = (k == 0), last = (k == c.nt - 1);
                const double nadd = last ? nadd_before(k, DT) : 0.0;
                const int i = tg.i0 + threadIdx.x;
                // the last sub-step's budget terms go to shared memory, as in k_store
                double *bt = sbud + threadIdx.x;
                auto bput = [&](int q, double v) { if (last) bt[q * kTile] = v; };
                if (last && i >= tg.i1)
#pragma unroll
                    for (int q = 0; q < kBudgets; q++) bt[q * kTile] = 0.0;
                if (i < tg.i1) cell_store(n, s, OwnG{n, s}, tg.m, i, DT, first, last, nadd, c, bput);
                if (last) {
                    double bl[kBudgets];
#pragma unroll
                    for (int q = 0; q < kBudgets; q++) bl[q] = bt[q * kTile];
                    warp_budget_partials(s, tg.m, i >> 5, budget_warps(N), bl);
                }
            } else {
                const int q = t - T, m = q / ppm, p = (q - m * ppm) * kTile + threadIdx.x;
                const MemberCtl &c = s.ctl[m];
                if (k < c.nt && p < n.P) {
                    const double DT = c.dt;
                    const bool last = (k == c.nt - 1);
                    path_rescale(n, s, m, p, DT, k == 0, last, last ? nadd_before(k, DT) : 0.0, c.dt_def);
                }
            }
        }
        if (!gb.sync()) return;
    }
    // ---- budgets of every member's last sub-step (k_budget)
    for (int r = b; r < M * kBudgets; r += G) budget_reduce(n, s, r / kBudgets, r % kBudgets);
    if (b == 0 && threadIdx.x == 0) s.loop->split = 0;
}

}  // namespace cmf
