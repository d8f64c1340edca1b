// Persistent panel kernel of the stage-1 bidiagonalization.
//
// One cooperative launch (one CTA per SM at most) runs all NB column steps of
// a panel [p0, p1).  Each step is
//   row pass     (row-parallel)    finish X for the previous row reflector,
//                                  update column i, accumulate A^T x
//   barrier A    every CTA sums the row-pass partial records itself and forms
//                the column reflector (same inputs, same order: identical in
//                every CTA)
//   column pass  (column-parallel) Y(:, i), row i, row-reflector partials
//   barrier B    every CTA sums those records and forms the row reflector
// The barriers count arrivals on one monotonic counter (barrier k of a launch
// completes at cnt_base + (k+1)*G), so a barrier costs an arrival, a poll and
// the one round trip that fetches the partial records.  The exact values a
// reflector needs besides the sums (its pivot, the panel entries of row i,
// the panel entries at column i+1) are written by their owner into small
// broadcast slots.  Waits are bounded: a CTA that waits ~2 s of SM clock
// records PACO_ERR_TIMEOUT, raises the abort flag and returns; the others
// follow at their next barrier.
//
// Rows are owned cyclically (row r belongs to CTA (r - p0) % G).  When a
// CTA's rows [p0, N) fit in shared memory they are staged once per panel and
// stay resident for its NB steps, so the trailing matrix is read from HBM once
// per panel instead of once per step; otherwise they are re-staged with TMA
// bulk copies at every step (double-buffered).  Data other CTAs wrote earlier
// in the same launch is read with ld.global.cg (L2), never from L1.
#include <cstring>

#include "bidiag.cuh"
#include "tma.cuh"

using namespace bd;

namespace {

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned long long gtimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void red_release_add(unsigned *p, unsigned v)
{
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Arrive at a grid barrier and wait (bounded) until `target` arrivals.  The
// arrival is a release (it publishes every write the CTA made before the
// __syncthreads) and the poll an acquire, so no further fences are needed.
__device__ bool pk_barrier(PkCtl *c, unsigned target, DevStatus *st, int where, int *s_ok,
                           long long max_cycles = 4000000000LL)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        red_release_add(&c->cnt, 1u);
        int ok = 1;
        long long t0 = clock64();
        while (ld_acquire(&c->cnt) < target) {
            if (ld_acquire(&c->abort)) { ok = 0; break; }
            if (clock64() - t0 > max_cycles) {
                atomicAdd(&st->wait_timeouts, 1);
                dev_fail(st, PACO_ERR_TIMEOUT, where);
                atomicExch(&c->abort, 1u);
                ok = 0;
                break;
            }
        }
        *s_ok = ok;
    }
    __syncthreads();
    return *s_ok != 0;
}

// Sums the per-CTA partial records rec[t * PCAP + cta] (cta < G <= 160) into
// out[t] for t < nval <= 80.  Every warp issues all of its loads before the
// first add, so the reduction costs one L2 round trip; the sum order is fixed
// (bitwise reproducible).  Threads t < nbc also store bc_val into bc_dst[t]
// before the closing barrier (a value they loaded before the call).  Called
// by every thread of the CTA.
__device__ __forceinline__ void reduce_records_fast(const float *rec, int G, int nval, float *out, float *bc_dst,
                                                    float bc_val, int nbc)
{
    constexpr int NW = RP_THREADS / 32, VPW = 5, LPV = 5;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float x[VPW][LPV];
#pragma unroll
    for (int v = 0; v < VPW; v++) {
        const int t = warp + NW * v;
#pragma unroll
        for (int k = 0; k < LPV; k++) {
            const int c = lane + 32 * k;
            x[v][k] = (t < nval && c < G) ? __ldcg(&rec[(long)t * PCAP + c]) : 0.f;
        }
    }
#pragma unroll
    for (int v = 0; v < VPW; v++) {
        const int t = warp + NW * v;
        float sum = 0.f;
#pragma unroll
        for (int k = 0; k < LPV; k++) sum += x[v][k];
        sum = warp_sum(sum);
        if (lane == 0 && t < nval) out[t] = sum;
    }
    if ((int)threadIdx.x < nbc) bc_dst[threadIdx.x] = bc_val;
    __syncthreads();
}

}  // namespace

// Rows a row-pass batch takes (one warp per row): resident rows go 16 at a
// time, streamed rows at most RMAX per TMA stage.
constexpr int PK_RMAX = RP_THREADS / 32;
// Owned rows whose X entries a CTA keeps in shared memory (else: global).
constexpr int PK_XOWN = 64;

// RB: rows per row-pass batch the unrolled loops cover (R <= RB).
template <int CPT, int RB>
__global__ void __launch_bounds__(RP_THREADS, 1)
    bd_panel_pk(const __grid_constant__ PkMulti pm, int p0, int p1, int resident, int R)
{
    // rows of a batch kept in registers between the two uses (<= 64 floats)
    constexpr bool REG = RB * CPT <= 16 && RB <= 16;
    // CTAs [j*G, (j+1)*G) run the panel of matrix j with their own barrier
    const int mi = blockIdx.x / pm.G;
    const BdArgs &a = pm.a[mi];
    PkCtl *const ctl = pm.ctl[mi];
    const unsigned cnt_base = pm.cnt_base[mi];
    extern __shared__ __align__(128) float tiles[];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ float red[RP_THREADS / 32][PK_RMAX];
    __shared__ float xs[PK_RMAX];
    __shared__ float s_t3[NB + 1], s_t4[NB], s_ycol[NB], s_wcol[NB]; // row reflector of step i-1
    __shared__ float s_t1[NB], s_t2[NB], s_ai[NB], s_xi[NB];         // column reflector of step i
    __shared__ float s_part[PK_RMAX][PR];
    __shared__ float s_red[PR], s_bc[PR];
    // column pass: three [warp][lane] tiles; row pass (REG): the batch rows'
    // panel columns s_pan[parity][row][lane] and dot partials
    // red2[parity][warp][row] (the two passes never overlap)
    __shared__ float cpool[3][RP_THREADS / 32][32];
    __shared__ float xs2[2][16];  // the batch rows' updated column entries, by batch parity
    float(*cy)[32] = cpool[0];
    float(*cA)[32] = cpool[1];
    float(*cB)[32] = cpool[2];
    __shared__ float s_cpart[PR];
    __shared__ int s_ok;


    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int M = a.M, N = a.N, G = pm.G, b = blockIdx.x - mi * pm.G;
    const long ldw = a.ldw;
    const int L = (int)(ldw - p0);
    DevStatus *st = a.st;
    // rows owned by this CTA: p0 + b + k*G, k < nown
    const int nown = (M - p0 - b + G - 1) / G > 0 ? (M - p0 - b + G - 1) / G : 0;
    auto own_row = [&](int k) { return p0 + b + k * G; };
    unsigned nbar = 0;
    // X entries of this CTA's rows (it computes them itself) after the row
    // tiles, when at most PK_XOWN rows are owned
    const int own_max = (M - p0 + G - 1) / G;
    float *xsm = (own_max <= PK_XOWN) ? tiles + (resident ? (long)own_max * L : 2L * R * L) : nullptr;

    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_init_fence();
    }
    __syncthreads();
    uint32_t phase0 = 0, phase1 = 0;
    bool failed = false;
    // 1/v0 of the previous column reflector: scales that column's entries in
    // the next row pass (every thread holds the same value)
    float cinv_prev = 1.f;
    // streamed rows: batches of the coming row pass already on their way
    // (issued at the end of the previous row pass, so their latency hides
    // behind the barriers and the column pass)
    int pf_n = 0;
    auto first_active = [&](int step) {
        int k = 0;
        while (k < nown && own_row(k) < step) k++;
        return k;
    };
    auto issue_rows = [&](int kf, int bb, int stage) {
        int k0 = kf + bb * R, nr = min(R, nown - k0);
        mbar_expect_tx(&bars[stage], (uint32_t)nr * L * 4u);
        for (int rr = 0; rr < nr; rr++)
            tma_load_1d(tiles + ((long)stage * R + rr) * L, a.W + (long)own_row(k0 + rr) * ldw + p0, (uint32_t)L * 4u,
                        &bars[stage]);
    };

    if (resident && nown > 0) {
        if (tid == 0) {
            mbar_expect_tx(&bars[0], (uint32_t)nown * L * 4u);
            for (int k = 0; k < nown; k++)
                tma_load_1d(tiles + (long)k * L, a.W + (long)own_row(k) * ldw + p0, (uint32_t)L * 4u, &bars[0]);
        }
        bool ok = mbar_wait_bounded(&bars[0], 0, st, 90);
        phase0 = 1;
        if (__syncthreads_or(!ok)) failed = true;
    }

    // the panel's steps, then (when a trailing matrix follows) the X-only pass
    const int last_step = (p1 < N) ? p1 : p1 - 1;
    const bool tracing = a.trace && a.trace_p0 == p0 && tid == 0 && (b == 0 || b == G - 1);
    auto stamp = [&](int i, int ph) {
        if (tracing) a.trace[(((i - p0) * 16 + ph) * 2) + (b == 0 ? 0 : 1)] = gtimer();
    };
    // slots 7-8 of a step: nanoseconds its row pass waited for streamed
    // rows, and its number of row batches
    unsigned long long waited = 0;
    for (int i = p0; i <= last_step && !failed; i++) {
        stamp(i, 0);
        const bool xonly = (i == p1);
        const bool doX = (i > p0);
        const bool doCol = !xonly;
        const int ii = i - p0, iip = ii - 1;

        // ------------- finish the row reflector of step i-1 (every CTA)
        float4 u4[CPT], acc4[CPT];
        float r_taup = 0.f;  // the row reflector of step i-1 (the same in every thread)
        if (doX) {
            // all loads of this phase in flight together
            const int nbc = 2 + 2 * iip;
            const float bcv = (tid < nbc) ? __ldcg(&a.bcB[tid]) : 0.f;
            float4 rb[CPT];
#pragma unroll
            for (int k = 0; k < CPT; k++) {
                int c = p0 + 4 * (tid + k * RP_THREADS);
                rb[k] = (c < ldw) ? __ldcg(reinterpret_cast<const float4 *>(a.rowbuf + c))
                                  : make_float4(0.f, 0.f, 0.f, 0.f);
            }
            reduce_records_fast(a.cpart, G, nbc, s_red, s_bc, bcv, nbc);
            // every thread forms the same reflector from the same sums
            float beta, v0;
            make_reflector(s_bc[0], s_red[0], N - (i - 1) - 1, &beta, &r_taup, &v0);
            const float inv = 1.f / v0;
            if (b == 0 && tid == 0) { a.e[i - 1] = beta; a.taup[i - 1] = r_taup; a.inv_v0r[i - 1] = inv; }
            // t3 = Y^T u (ii values), t4 = U u (iip values); next column's panel entries
            if (tid <= iip) {
                s_t3[tid] = s_bc[1 + tid] + s_red[1 + tid] * inv;
                s_ycol[tid] = s_bc[1 + tid];                              // Y[i, q], q < ii
            }
            if (tid < iip) {
                s_t4[tid] = s_bc[2 + iip + tid] + s_red[2 + iip + tid] * inv;
                s_wcol[tid] = s_bc[2 + iip + tid];                        // U[q, i], q < iip
            }
            if (tid == iip) s_wcol[tid] = 1.f;                            // implicit 1 of row i-1
#pragma unroll
            for (int k = 0; k < CPT; k++) {
                int c = p0 + 4 * (tid + k * RP_THREADS);
                float r[4] = {rb[k].x, rb[k].y, rb[k].z, rb[k].w};
                float uv[4];
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    int j = c + e;
                    uv[e] = (j == i) ? 1.f : ((j > i && j < N) ? r[e] * inv : 0.f);
                }
                u4[k] = make_float4(uv[0], uv[1], uv[2], uv[3]);
            }
            // the scaled row reflector goes into row i-1 of W (later column passes
            // and the panel's trailing update read it)
            // (from the row values this thread already holds: no second read)
            if (b == 0) {
#pragma unroll
                for (int k = 0; k < CPT; k++) {
                    const int c = p0 + 4 * (tid + k * RP_THREADS);
                    const float r[4] = {rb[k].x, rb[k].y, rb[k].z, rb[k].w};
#pragma unroll
                    for (int e = 0; e < 4; e++)
                        if (c + e > i && c + e < N) a.W[(long)(i - 1) * ldw + c + e] = r[e] * inv;
                }
                if (xonly && tid == 0) a.W[(long)(i - 1) * ldw + i] = 1.f;
            }
        } else {
#pragma unroll
            for (int k = 0; k < CPT; k++) u4[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int k = 0; k < CPT; k++) acc4[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int t = tid; t < PK_RMAX * PR; t += RP_THREADS) (&s_part[0][0])[t] = 0.f;
        const float taup_prev = doX ? r_taup : 0.f;
        const float invc = (ii >= 1) ? cinv_prev : 1.f;

        // ------------------------------------------------------ row pass
        const int kfirst = first_active(i);
        const int nact = nown - kfirst;
        const int nbatch = (nact + R - 1) / R;
        __syncthreads();
        stamp(i, 1);
        if (!resident && tid == 0 && pf_n < min(2, nbatch)) {
            proxy_async_fence();
            asm volatile("fence.proxy.async.global;" ::: "memory");
            for (int bb = pf_n; bb < min(2, nbatch); bb++) issue_rows(kfirst, bb, bb);
        }
        pf_n = 0;
        float w_ss = 0.f, w_g1 = 0.f, w_g2 = 0.f;
        if constexpr (REG) {
            // Rows held in registers between the dot products and the A^T x
            // share (one read of the stage), two CTA barriers per batch, and
            // the stage refilled right after the first: the rows' panel
            // columns go to shared memory first for the per-row scalars,
            // which warp rr forms for row rr.
            for (int bb = 0; bb < nbatch; bb++) {
                const int k0 = kfirst + bb * R, nr = min(R, nown - k0);
                const int par = bb & 1, stage = bb & 1;
                float *span = &cpool[par][0][0];  // [RB][32]
                float *red2 = &cpool[2][0][0] + par * (RP_THREADS / 32) * 16;  // [warp][16]
                const float *T;
                if (resident) {
                    T = tiles + (long)k0 * L;
                } else {
                    const unsigned long long tw = tracing ? gtimer() : 0ull;
                    if (!mbar_wait_bounded(&bars[stage], stage ? phase1 : phase0, st, 200 + i)) failed = true;
                    if (tracing) waited += gtimer() - tw;
                    if (stage) phase1 ^= 1; else phase0 ^= 1;
                    T = tiles + (long)stage * R * L;
                }
                float4 v[RB][CPT];
#pragma unroll
                for (int rr = 0; rr < RB; rr++) {
                    float pd = 0.f;
#pragma unroll
                    for (int k = 0; k < CPT; k++) {
                        const int c4 = tid + k * RP_THREADS;
                        v[rr][k] = (rr < nr && 4 * c4 < L) ? *reinterpret_cast<const float4 *>(T + (long)rr * L + 4 * c4)
                                                           : make_float4(0.f, 0.f, 0.f, 0.f);
                        pd += v[rr][k].x * u4[k].x + v[rr][k].y * u4[k].y + v[rr][k].z * u4[k].z + v[rr][k].w * u4[k].w;
                    }
                    if (doX && rr < nr) {
                        pd = warp_sum(pd);
                        if (lane == 0) red2[warp * 16 + rr] = pd;
                    }
                }
                if (warp < nr) span[warp * 32 + lane] = T[(long)warp * L + lane];
                __syncthreads();
                if (!resident && tid == 0 && bb + 2 < nbatch) {
                    proxy_async_fence();
                    issue_rows(kfirst, bb + 2, stage);
                }
                if (warp < nr) {
                    const int rr = warp, r = own_row(k0 + rr);
                    const float pan = span[rr * 32 + lane];
                    float aq = (lane < ii) ? pan : 0.f;
                    if (lane == ii - 1) {
                        aq *= invc;
                        a.W[(long)r * ldw + (i - 1)] = aq;
                        if (resident) tiles[(long)(k0 + rr) * L + lane] = aq;
                    }
                    const float xq = (doX && lane < iip)
                                         ? (xsm ? xsm[(k0 + rr) * NB + lane] : a.X[(long)r * NB + lane])
                                         : 0.f;
                    float Xn = 0.f;
                    if (doX) {
                        float dot = 0.f;
#pragma unroll
                        for (int w2 = 0; w2 < RP_THREADS / 32; w2++) dot += red2[w2 * 16 + rr];
                        const float sx = ((lane <= iip) ? aq * s_t3[lane] : 0.f) + ((lane < iip) ? xq * s_t4[lane] : 0.f);
                        Xn = taup_prev * (dot - warp_sum(sx));
                        if (lane == 0) {
                            a.X[(long)r * NB + iip] = Xn;
                            if (xsm) xsm[(k0 + rr) * NB + iip] = Xn;
                        }
                    }
                    if (doCol) {
                        const float xrq = (lane < ii - 1) ? xq : ((lane == ii - 1) ? Xn : 0.f);
                        const float sc = (lane < ii) ? (aq * s_ycol[lane] + xrq * s_wcol[lane]) : 0.f;
                        const float xr = __shfl_sync(0xffffffffu, pan, ii & 31) - warp_sum(sc);
                        if (lane == 0) {
                            a.W[(long)r * ldw + i] = xr;
                            if (resident) tiles[(long)(k0 + rr) * L + ii] = xr;
                            xs2[par][rr] = xr;
                        }
                        if (r == i) {
                            // pivot and row-i panel entries for every CTA's column reflector
                            if (lane == 0) a.bcA[0] = xr;
                            if (lane < ii) {
                                a.bcA[1 + lane] = aq;
                                a.bcA[1 + ii + lane] = xrq;
                            }
                        } else if (r > i) {
                            if (lane == 0) w_ss += xr * xr;
                            if (lane < ii) { w_g1 += aq * xr; w_g2 += xrq * xr; }
                        }
                    }
                }
                __syncthreads();
                if (doCol) {
#pragma unroll
                    for (int rr = 0; rr < RB; rr++) {
                        if (rr < nr && own_row(k0 + rr) > i) {
                            const float xr = xs2[par][rr];
#pragma unroll
                            for (int k = 0; k < CPT; k++) {
                                acc4[k].x += v[rr][k].x * xr; acc4[k].y += v[rr][k].y * xr;
                                acc4[k].z += v[rr][k].z * xr; acc4[k].w += v[rr][k].w * xr;
                            }
                        }
                    }
                }
            }
        } else
        for (int bb = 0; bb < nbatch; bb++) {
            const int k0 = kfirst + bb * R, nr = min(R, nown - k0);
            const float *T;
            const int stage = bb & 1;
            // X entries of the staged rows, loaded before the dot products so
            // their latency overlaps them
            const float xq_pre = (warp < nr && doX && lane < iip)
                                     ? (xsm ? xsm[(k0 + warp) * NB + lane] : a.X[(long)own_row(k0 + warp) * NB + lane])
                                     : 0.f;
            if (resident) {
                T = tiles + (long)k0 * L;
            } else {
                const unsigned long long tw = tracing ? gtimer() : 0ull;
                bool ok = mbar_wait_bounded(&bars[stage], stage ? phase1 : phase0, st, 200 + i);
                if (tracing) waited += gtimer() - tw;
                if (stage) phase1 ^= 1; else phase0 ^= 1;
                if (__syncthreads_or(!ok)) { failed = true; break; }
                T = tiles + (long)stage * R * L;
            }
            if (doX) {
                float pd[RB];
#pragma unroll
                for (int rr = 0; rr < RB; rr++) pd[rr] = 0.f;
#pragma unroll
                for (int rr = 0; rr < RB; rr++) {
                    if (rr < nr) {
#pragma unroll
                        for (int k = 0; k < CPT; k++) {
                            int c4 = tid + k * RP_THREADS;
                            if (4 * c4 < L) {
                                float4 v = *reinterpret_cast<const float4 *>(T + (long)rr * L + 4 * c4);
                                pd[rr] += v.x * u4[k].x + v.y * u4[k].y + v.z * u4[k].z + v.w * u4[k].w;
                            }
                        }
                    }
                }
#pragma unroll
                for (int rr = 0; rr < RB; rr++) {
                    if (rr < nr) {
                        float v = warp_sum(pd[rr]);
                        if (lane == 0) red[warp][rr] = v;
                    }
                }
                __syncthreads();
            }
            if (warp < nr) {
                const int rr = warp, r = own_row(k0 + rr);
                float *trow = (float *)T + (long)rr * L;
                float aq = (lane < ii) ? trow[lane] : 0.f;
                if (lane == ii - 1) {
                    aq *= invc;
                    a.W[(long)r * ldw + (i - 1)] = aq;
                    if (resident) trow[lane] = aq;
                }
                const float xq = xq_pre;
                float Xn = 0.f;
                if (doX) {
                    float dot = 0.f;
#pragma unroll
                    for (int w2 = 0; w2 < RP_THREADS / 32; w2++) dot += red[w2][rr];
                    float sx = ((lane <= iip) ? aq * s_t3[lane] : 0.f) + ((lane < iip) ? xq * s_t4[lane] : 0.f);
                    Xn = taup_prev * (dot - warp_sum(sx));
                    if (lane == 0) {
                        a.X[(long)r * NB + iip] = Xn;
                        if (xsm) xsm[(k0 + rr) * NB + iip] = Xn;
                    }
                }
                if (doCol) {
                    float xrq = (lane < ii - 1) ? xq : ((lane == ii - 1) ? Xn : 0.f);
                    float sc = (lane < ii) ? (aq * s_ycol[lane] + xrq * s_wcol[lane]) : 0.f;
                    float xr = trow[ii] - warp_sum(sc);
                    __syncwarp();
                    if (lane == 0) {
                        a.W[(long)r * ldw + i] = xr;
                        if (resident) trow[ii] = xr;
                        xs[rr] = xr;
                    }
                    if (r == i) {
                        // pivot and row-i panel entries for every CTA's column reflector
                        if (lane == 0) a.bcA[0] = xr;
                        if (lane < ii) {
                            a.bcA[1 + lane] = aq;
                            a.bcA[1 + ii + lane] = xrq;
                        }
                    } else if (r > i) {
                        if (lane == 0) w_ss += xr * xr;
                        if (lane < ii) { w_g1 += aq * xr; w_g2 += xrq * xr; }
                    }
                }
            }
            __syncthreads();
            if (doCol) {
#pragma unroll
                for (int rr = 0; rr < RB; rr++) {
                    if (rr < nr && own_row(k0 + rr) > i) {
                        float xr = xs[rr];
#pragma unroll
                        for (int k = 0; k < CPT; k++) {
                            int c4 = tid + k * RP_THREADS;
                            if (4 * c4 < L) {
                                float4 v = *reinterpret_cast<const float4 *>(T + (long)rr * L + 4 * c4);
                                acc4[k].x += v.x * xr; acc4[k].y += v.y * xr;
                                acc4[k].z += v.z * xr; acc4[k].w += v.w * xr;
                            }
                        }
                    }
                }
            }
            __syncthreads();
            if (!resident && tid == 0 && bb + 2 < nbatch) {
                proxy_async_fence();
                issue_rows(kfirst, bb + 2, stage);
            }
        }
        if (__syncthreads_or(failed)) { failed = true; break; }
        if (tracing) {
            unsigned long long *tr = a.trace + (long)(i - p0) * 32 + (b == 0 ? 0 : 1);
            tr[7 * 2] = waited;
            tr[8 * 2] = (unsigned long long)nbatch;
            waited = 0;
        }
        if (!resident && i < last_step) {
            // the first two batches of the next step's row pass: its rows (>= i+1)
            // changed only in this row pass, by this CTA
            const int kf1 = first_active(i + 1);
            const int nb1 = (nown - kf1 + R - 1) / R;
            pf_n = min(2, nb1);
            if (tid == 0 && pf_n > 0) {
                asm volatile("fence.proxy.async.global;" ::: "memory");
                for (int bb = 0; bb < pf_n; bb++) issue_rows(kf1, bb, bb);
            }
        }
        stamp(i, 2);
        if (xonly) break; // the X-only pass ends the panel

        // row-pass partials: A^T x (all tile columns), |x|^2, V^T x, X^T x
#pragma unroll
        for (int k = 0; k < CPT; k++) {
            int c4 = tid + k * RP_THREADS;
            if (4 * c4 < L) *reinterpret_cast<float4 *>(a.ypart + (long)b * ldw + p0 + 4 * c4) = acc4[k];
        }
        if (warp < PK_RMAX) {
            if (lane == 0) s_part[warp][0] = w_ss;
            if (lane < ii) {
                s_part[warp][1 + lane] = w_g1;
                s_part[warp][1 + ii + lane] = w_g2;
            }
        }
        __syncthreads();
        for (int t = tid; t < PR; t += RP_THREADS) {
            float v = 0.f;
            for (int w = 0; w < PK_RMAX; w++) v += s_part[w][t];
            a.tpart[(long)t * PCAP + b] = v;
        }
        // operands of this CTA's first column-pass chunk do not depend on the
        // barrier: load them now so their latency hides behind it
        const int nchunk = (i < N - 1) ? (N - i - 1 + 31) / 32 : 0;
        float pY[2] = {0.f, 0.f}, pW[2] = {0.f, 0.f}, pwij = 0.f;
        if (b < nchunk) {
            const int j = i + 1 + b * 32 + lane;
            if (j < N) {
                pwij = __ldcg(&a.W[(long)i * ldw + j]);
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    int q = 2 * warp + e;
                    if (q < ii) {
                        pY[e] = __ldcg(&a.Yt[(long)q * ldw + j]);
                        pW[e] = __ldcg(&a.W[(long)(p0 + q) * ldw + j]);
                    }
                }
            }
        }
        stamp(i, 3);
        if (!pk_barrier(ctl, cnt_base + (++nbar) * G, st, 300 + i, &s_ok)) { failed = true; break; }

        // the partial A^T x records of this CTA's first column chunk travel
        // with the records of the column reflector: one L2 round trip
        constexpr int YV = RB_CAP / (RP_THREADS / 32);
        float yv0[YV];
        {
            const int j = i + 1 + b * 32 + lane;
            const bool v = (b < nchunk) && j < N;
#pragma unroll
            for (int k = 0; k < YV; k++) {
                const int q = warp + (RP_THREADS / 32) * k;
                yv0[k] = (v && q < G) ? __ldcg(&a.ypart[(long)q * ldw + j]) : 0.f;
            }
        }

        // ------------- column reflector of step i (every CTA, every thread)
        float c_tau, c_inv;
        {
            const int nbc = 1 + 2 * ii;
            const float bcv = (tid < nbc) ? __ldcg(&a.bcA[tid]) : 0.f;
            reduce_records_fast(a.tpart, G, 1 + 2 * ii, s_red, s_bc, bcv, nbc);
            float beta, v0;
            make_reflector(s_bc[0], s_red[0], M - i, &beta, &c_tau, &v0);
            c_inv = 1.f / v0;
            cinv_prev = c_inv;  // scales column i's entries in the next step
            if (b == 0 && tid == 0) { a.d[i] = beta; a.tauq[i] = c_tau; a.inv_v0c[i] = c_inv; }
            if (tid < ii) {
                const float inv = c_inv;
                s_ai[tid] = s_bc[1 + tid];                                  // V[i, q] (row i panel entries)
                s_xi[tid] = s_bc[1 + ii + tid];                             // X[i, q]
                s_t1[tid] = s_bc[1 + tid] + s_red[1 + tid] * inv;           // V^T v
                s_t2[tid] = s_bc[1 + ii + tid] + s_red[1 + ii + tid] * inv; // X^T v
            } else if (tid < NB) {
                // the column pass multiplies every panel slot: the unused ones
                // must hold zeros, not what an earlier kernel left in shared memory
                s_ai[tid] = 0.f;
                s_xi[tid] = 0.f;
                s_t1[tid] = 0.f;
                s_t2[tid] = 0.f;
            }
            for (int t = tid; t < PR; t += RP_THREADS) s_cpart[t] = 0.f;
            __syncthreads();
        }
        stamp(i, 4);
        if (i >= N - 1) break; // no row reflector after the last column

        // --------------------------------------------------- column pass
        const float tq = c_tau, invc_i = c_inv;
        for (int ch = b; ch < nchunk; ch += G) {
            const int j = i + 1 + ch * 32 + lane;
            const bool valid = j < N;
            const bool first = (ch == b);
            float yv[YV];
#pragma unroll
            for (int k = 0; k < YV; k++) {
                int q = warp + (RP_THREADS / 32) * k;
                yv[k] = first ? yv0[k] : ((valid && q < G) ? __ldcg(&a.ypart[(long)q * ldw + j]) : 0.f);
            }
            float ys = 0.f;
#pragma unroll
            for (int k = 0; k < YV; k++) ys += yv[k];
            cy[warp][lane] = ys;
            // warp w owns panel indices q in [2w, 2w+2)
            float Yq[2], Wq[2], pa = 0.f, pb = 0.f;
#pragma unroll
            for (int e = 0; e < 2; e++) {
                int q = 2 * warp + e;
                bool use = valid && q < ii;
                Yq[e] = first ? pY[e] : (use ? __ldcg(&a.Yt[(long)q * ldw + j]) : 0.f);
                Wq[e] = first ? pW[e] : (use ? __ldcg(&a.W[(long)(p0 + q) * ldw + j]) : 0.f);
                pa += Yq[e] * s_t1[q] + Wq[e] * s_t2[q];
                pb += Yq[e] * s_ai[q] + Wq[e] * s_xi[q];
            }
            cA[warp][lane] = pa;
            cB[warp][lane] = pb;
            __syncthreads();
            float y = 0.f, sa = 0.f, sb = 0.f;
#pragma unroll
            for (int w = 0; w < RP_THREADS / 32; w++) { y += cy[w][lane]; sa += cA[w][lane]; sb += cB[w][lane]; }
            float Ynew = 0.f, aj = 0.f;
            if (valid) {
                float wij = first ? pwij : __ldcg(&a.W[(long)i * ldw + j]);
                Ynew = tq * (wij + y * invc_i - sa);
                aj = wij - Ynew - sb;
                if (warp == 0) {
                    a.Yt[(long)ii * ldw + j] = Ynew;
                    a.rowbuf[j] = aj;
                }
            }
            if (j == i + 1) {
                // pivot and column-(i+1) panel entries for every CTA's row reflector
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    int q = 2 * warp + e;
                    if (q < ii) {
                        a.bcB[1 + q] = Yq[e];
                        a.bcB[2 + ii + q] = Wq[e];
                    }
                }
                if (warp == 0) {
                    a.bcB[0] = aj;
                    a.bcB[1 + ii] = Ynew;
                }
            }
            float m = (valid && j >= i + 2) ? aj : 0.f;
#pragma unroll
            for (int e = 0; e < 2; e++) {
                int q = 2 * warp + e;
                if (q < ii) {
                    float g3 = warp_sum(Yq[e] * m), g4 = warp_sum(Wq[e] * m);
                    if (lane == 0) { s_cpart[1 + q] += g3; s_cpart[2 + ii + q] += g4; }
                }
            }
            if (warp == 0) {
                float ss = warp_sum(m * m), g3 = warp_sum(Ynew * m);
                if (lane == 0) { s_cpart[0] += ss; s_cpart[1 + ii] += g3; }
            }
            __syncthreads();
        }
        stamp(i, 5);
        for (int t = tid; t < PR; t += RP_THREADS) a.cpart[(long)t * PCAP + b] = s_cpart[t];
        if (!pk_barrier(ctl, cnt_base + (++nbar) * G, st, 400 + i, &s_ok)) { failed = true; break; }
        stamp(i, 6);
    }
    // a step that ended early leaves prefetched rows in flight: they land
    // before the CTA exits
    if (!resident && tid == 0)
        for (int bb = 0; bb < pf_n; bb++)
            mbar_wait_bounded(&bars[bb], bb ? phase1 : phase0, st, 91, 1000000000LL);
}

// Grid barriers one launch for panel [p0, p1) passes (host and kernel agree):
// barrier A at every step, barrier B at every step but a last column.
static unsigned pk_barriers(int N, int p0, int p1)
{
    const int nbp = p1 - p0;
    return (unsigned)(2 * nbp - (p1 == N ? 1 : 0));
}

// Host side: launches the persistent kernel for panel [p0, p1) of k matrices
// of one shape cooperatively, G CTAs per matrix.  cnt[j] is matrix j's
// arrival counter value before the launch; it is advanced by the arrivals
// this launch makes.  Returns false when a cooperative launch of k * G CTAs
// is not possible.
bool bd_panel_pk_launch_multi(int k, const BdArgs *a, PkCtl *const *ctl, int p0, int p1, int G, unsigned *cnt,
                              cudaStream_t s)
{
    if (k < 1 || k > PK_KMAX) return false;
    const int L = (int)(a[0].ldw - p0);
    const int own = (a[0].M - p0 + G - 1) / G;
    const long budget = 200 * 1024;
    int resident = ((long)own * L * 4 <= budget) ? 1 : 0;
    int R = std::max(1, std::min(RMAX, (int)(budget / (2L * L * 4))));
    size_t smem = resident ? (size_t)own * L * 4 : (size_t)2 * R * L * 4;
    const int chunks = ceil_div(L, 4 * RP_THREADS);
    // resident rows go 16 per batch (8 with two float4 chunks a thread, so a
    // batch stays in registers)
    if (resident) R = (chunks == 2) ? RMAX : PK_RMAX;
    if (own <= PK_XOWN) smem += (size_t)own * NB * 4;  // X entries of the owned rows
    void *fn;
    if (resident) fn = chunks <= 1 ? (void *)bd_panel_pk<1, PK_RMAX> : chunks == 2 ? (void *)bd_panel_pk<2, RMAX>
                                                                                 : (void *)bd_panel_pk<4, PK_RMAX>;
    else fn = chunks <= 1 ? (void *)bd_panel_pk<1, RMAX> : chunks == 2 ? (void *)bd_panel_pk<2, RMAX>
                                                                       : (void *)bd_panel_pk<4, RMAX>;
    PkMulti pm;
    memset(&pm, 0, sizeof(pm));
    pm.G = G;
    for (int j = 0; j < k; j++) {
        pm.a[j] = a[j];
        pm.ctl[j] = ctl[j];
        pm.cnt_base[j] = cnt[j];
    }
    void *args[] = {&pm, &p0, &p1, &resident, &R};
    paco_count_launch();
    if (cudaLaunchCooperativeKernel(fn, dim3(k * G), dim3(RP_THREADS), args, smem, s) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    for (int j = 0; j < k; j++) cnt[j] += pk_barriers(a[j].N, p0, p1) * (unsigned)G;
    return true;
}

bool bd_panel_pk_launch(const BdArgs &a, PkCtl *ctl, int p0, int p1, int G, unsigned *cnt, cudaStream_t s)
{
    return bd_panel_pk_launch_multi(1, &a, &ctl, p0, p1, G, cnt, s);
}

// Test hook: every CTA of a cooperative grid arrives at a grid barrier whose
// target (one arrival more than the grid has) is never reached; the waits
// give up after max_cycles, record PACO_ERR_TIMEOUT and raise the abort flag.
__global__ void pk_dbg_barrier_timeout(PkCtl *ctl, DevStatus *st, long long max_cycles)
{
    __shared__ int s_ok;
    pk_barrier(ctl, gridDim.x + 1, st, 999, &s_ok, max_cycles);
}

bool bd_pk_debug_timeout(PkCtl *ctl, DevStatus *st, int G, long long max_cycles, cudaStream_t s)
{
    if (cudaMemsetAsync(ctl, 0, sizeof(PkCtl), s) != cudaSuccess) return false;
    void *args[] = {&ctl, &st, &max_cycles};
    paco_count_launch();
    return cudaLaunchCooperativeKernel((void *)pk_dbg_barrier_timeout, dim3(G), dim3(64), args, 0, s) == cudaSuccess;
}

void bd_pk_init_attrs()
{
    static bool done[PACO_MAX_DEVICES] = {};
    const int dev = paco_device();
    if (done[dev]) return;
    int maxs = 200 * 1024 + PK_XOWN * NB * 4 + 1024;
    cudaFuncSetAttribute(bd_panel_pk<1, PK_RMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs);
    cudaFuncSetAttribute(bd_panel_pk<4, PK_RMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs);
    cudaFuncSetAttribute(bd_panel_pk<1, RMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs);
    cudaFuncSetAttribute(bd_panel_pk<2, RMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs);
    cudaFuncSetAttribute(bd_panel_pk<4, RMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs);
    done[dev] = true;
}
