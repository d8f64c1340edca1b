// Device bodies of the bidiagonal divide and conquer (BDC) phases.  Each body
// does the work of one "virtual block" of its phase, so the same code runs as
// one kernel per phase over a whole tree level (bdc.cu, single large matrix)
// and as loops inside one CTA that owns a whole small matrix (batched.cu).
// Bodies that synchronize (prepare, finalize, rank) need all 256 threads of
// the CTA; the others are per thread or per warp.
//
// Reference: svd.cpp (DEAVEN-MITCH/paco-svd), a LAPACK sbdsdc/slasd1-4 style
// solver: 3-column leaves (svd.cpp:1596-1864, partition svd_tiling.cpp:83-130),
// bottom-up pairwise merges with the odd tail carried (svd.cpp:168-189), each
// merge = scale (:225-323), deflation (:325-975), secular roots (:977-1336),
// Loewner z and vectors (:1337-1496), back-transform matmul (:1498-1521),
// idxq sort (:1523-1590); then a descending sort (:1866-1909).
#pragma once

#include <math_constants.h>

#include <cfloat>

#include "bdc.cuh"
#include "gemm.cuh"

#define BDC_SEC_MAXIT 100
// Iteration limit the secular solver applies (BDC_SEC_MAXIT unless a test
// lowers it to force the non-convergence report).  Each translation unit
// that includes this header has its own copy; bdc_set_sec_maxit (bdc.cu) and
// bt_set_sec_maxit (batched.cu) set theirs.
static __device__ int g_sec_maxit = BDC_SEC_MAXIT;
#define BDC_MAX_LEVELS 32
#define GATHER_ROWS 16

static __device__ __forceinline__ double sgn1(double x) { return x < 0 ? -1.0 : 1.0; }

struct LevelArgs {
    int N, off;
    const float *d_e; // e (superdiagonal)
    float *d;
    float *QT, *ST, *WT, *GT;  // ld N
    int *idxq;
    float *f, *l, *dsig, *zhat;
    int *srow;
    float *diff; // N x N, ld N
    BdcWs w;
};

// --------------------------------------------------------------- schedule

// Builds leaves and merges of every level from N (the canonical partition)
// and checks that the caller's tiling blob describes the same partition; a
// null blob means "use the canonical partition".  Level l holds merges
// [lv_off[l], lv_off[l] + lv_nm[l]) when lv_off is given.  One thread.
static __device__ int bdc_schedule_dev(int N, const uint8_t *tiling, const BdcWs &w, int *lv_off, int *lv_nm)
{
    int nleaf = leaf_partition(N, w.leaf_s, w.leaf_e);
    bool ok = true;
    if (tiling) {
        const TilingHeader *h = (const TilingHeader *)tiling;
        ok = h->magic == PACO_TILING_MAGIC && (int)h->N == N && (int)h->nleaf == nleaf && h->offset == 32;
        if (ok) {
            const uint32_t *lv = (const uint32_t *)(tiling + 32);
            for (int t = 0; t < nleaf && ok; t++)
                ok = (int)lv[2 * t] == w.leaf_s[t] && (int)lv[2 * t + 1] == w.leaf_e[t];
        }
    }
    if (!ok) dev_fail(w.st, PACO_ERR_BAD_TILING, N);
    // merge levels: stack entries [s, e); pairs of adjacent entries merge
    int *ss = w.perm, *ee = (int *)w.sig; // scratch (N >= nleaf)
    for (int t = 0; t < nleaf; t++) { ss[t] = w.leaf_s[t]; ee[t] = w.leaf_e[t]; }
    int cnt = nleaf, out = 0, nlev = 0;
    while (cnt > 1) {
        if (lv_off && nlev < BDC_MAX_LEVELS) { lv_off[nlev] = out; lv_nm[nlev] = 0; }
        int wpos = 0, r = 0;
        while (r < cnt - 1) {
            w.mg_s[out] = ss[r]; w.mg_m[out] = ss[r + 1]; w.mg_e[out] = ee[r + 1]; out++;
            if (lv_off && nlev < BDC_MAX_LEVELS) lv_nm[nlev]++;
            ss[wpos] = ss[r]; ee[wpos] = ee[r + 1]; wpos++;
            r += 2;
        }
        if (r == cnt - 1) { ss[wpos] = ss[r]; ee[wpos] = ee[r]; wpos++; }
        cnt = wpos;
        nlev++;
    }
    return nlev;
}

// ------------------------------------------------------------------ leaves

// SVD of the upper-triangular 2x2 [[f,g],[0,h]]: rows of u/v are the vectors,
// B v_i = s_i u_i, s1 >= s2 >= 0, det[u1 u2] = sign(f h).
static __device__ void dev_svd2x2(double f, double g, double h, double *s, double *u, double *v)
{
    if (g == 0.0) {
        if (fabs(f) >= fabs(h)) {
            s[0] = fabs(f); s[1] = fabs(h);
            v[0] = 1; v[1] = 0; u[0] = sgn1(f); u[1] = 0;
            v[2] = 0; v[3] = 1; u[2] = 0; u[3] = sgn1(h);
        } else {
            s[0] = fabs(h); s[1] = fabs(f);
            v[0] = 0; v[1] = 1; u[0] = 0; u[1] = sgn1(h);
            v[2] = 1; v[3] = 0; u[2] = sgn1(f); u[3] = 0;
        }
        return;
    }
    double fa = fabs(f), ha = fabs(h);
    double s1 = 0.5 * (hypot(fa + ha, g) + hypot(fa - ha, g));
    double s2 = fa * ha / s1;
    double s1q = s1 * s1;
    double ax = f * g, ay = s1q - f * f, bx = s1q - g * g - h * h, by = f * g;
    double vx, vy;
    if (ax * ax + ay * ay >= bx * bx + by * by) { vx = ax; vy = ay; } else { vx = bx; vy = by; }
    double nv = hypot(vx, vy);
    vx /= nv; vy /= nv;
    double ux = f * vx + g * vy, uy = h * vy, nu = hypot(ux, uy);
    ux /= nu; uy /= nu;
    double sd = (f * h >= 0) ? 1.0 : -1.0;
    s[0] = s1; s[1] = s2;
    v[0] = vx; v[1] = vy; v[2] = -vy; v[3] = vx;
    u[0] = ux; u[1] = uy; u[2] = -sd * uy; u[3] = sd * ux;
}

// leaf t (compute_base_case_svd, svd.cpp:1596-1625)
static __device__ void bdc_leaf_dev(int t, int N, const BdcWs &w, float *d, const float *e, float *QT, float *WT,
                                    int *idxq, float *fv, float *lv)
{
    const int s = w.leaf_s[t], end = w.leaf_e[t];
    const int cols = end - s, rows = (end == N) ? cols : cols - 1;
    auto Q = [&](int r, int c) -> float & { return QT[(long)(s + r) * N + s + c]; };
    auto Wm = [&](int r, int c) -> float & { return WT[(long)(s + r) * N + s + c]; };
    double sv[2], u[4], v[4];
    if (rows == 1 && cols == 1) {
        double a = d[s];
        idxq[s] = 0;
        Q(0, 0) = (float)sgn1(a);
        Wm(0, 0) = 1.f;
        d[s] = (float)fabs(a);
    } else if (rows == 1 && cols == 2) {
        double a = d[s], b = e[s], sq = hypot(a, b);
        idxq[s] = 0;
        d[s] = (float)sq;
        if (sq != 0) {
            Wm(0, 0) = (float)(a / sq); Wm(0, 1) = (float)(b / sq);
            Wm(1, 0) = (float)(b / sq); Wm(1, 1) = (float)(-a / sq);
        }
    } else if (rows == 2 && cols == 2) {
        dev_svd2x2(d[s], e[s], d[s + 1], sv, u, v);
        idxq[s] = 1; idxq[s + 1] = 0;
        d[s] = (float)sv[0]; d[s + 1] = (float)sv[1];
        for (int i = 0; i < 2; i++)
            for (int j = 0; j < 2; j++) { Q(i, j) = (float)u[2 * i + j]; Wm(i, j) = (float)v[2 * i + j]; }
    } else {
        // [[a, b, 0], [0, c, f]]: rotate columns (1,2) then (0,2) to [[r2, c1 b, 0], [0, r1, 0]]
        double a = d[s], b = e[s], c = d[s + 1], f = e[s + 1];
        double r1 = hypot(c, f), c1 = 1, s1 = 0;
        if (r1 != 0) { c1 = c / r1; s1 = f / r1; }
        double r2 = hypot(a, s1 * b), c2 = 1, s2 = 0;
        if (r2 != 0) { c2 = a / r2; s2 = -s1 * b / r2; }
        dev_svd2x2(r2, c1 * b, r1, sv, u, v);
        double G[3][3] = {{c2, 0, -s2}, {-s1 * s2, c1, -s1 * c2}, {c1 * s2, s1, c1 * c2}};
        idxq[s] = 1; idxq[s + 1] = 0;
        d[s] = (float)sv[0]; d[s + 1] = (float)sv[1];
        for (int i = 0; i < 2; i++) {
            Q(i, 0) = (float)u[2 * i]; Q(i, 1) = (float)u[2 * i + 1];
            for (int r = 0; r < 3; r++) Wm(i, r) = (float)(G[r][0] * v[2 * i] + G[r][1] * v[2 * i + 1]);
        }
        for (int r = 0; r < 3; r++) Wm(2, r) = (float)G[r][2];
    }
    for (int j = 0; j < cols; j++) {
        fv[s + j] = Wm(j, 0);
        lv[s + j] = Wm(j, cols - 1);
    }
}

// ------------------------------------------------------------- merge bodies

// number of elements of the ascending run a[0..n) that are < v (strict) or <= v
static __device__ __forceinline__ int count_below(const float *a, int n, float v, bool inclusive)
{
    int lo = 0, hi = n;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        bool below = inclusive ? (a[mid] <= v) : (a[mid] < v);
        if (below) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// Scale, z, merge of the two sorted runs and the FP64 deflation scan of merge
// mg.  256 threads; `sm` holds 20 * (n - 1) bytes.
static __device__ void bdc_prepare_dev(const LevelArgs &A, int mg, unsigned char *sm)
{
    __shared__ float s_red[8];
    __shared__ int s_knd;
    const int s = A.w.mg_s[A.off + mg], m = A.w.mg_m[A.off + mg], e_end = A.w.mg_e[A.off + mg];
    const int N = A.N;
    const int nl = m - s, nr = e_end - m, sq = (e_end == N);
    const int Lr = nl - 1, Rr = nr - 1 + sq, n = Lr + Rr + 1, nc = n + 1 - sq, dn = n - 1;
    const int tid = threadIdx.x;
    double *sz = (double *)sm;                  // dn
    float *sd = (float *)(sz + dn);             // dn
    int *srowp = (int *)(sd + dn);              // dn
    float *runs = (float *)(srowp + dn);        // dn, later reused as idxp
    int *idxp = (int *)runs;

    const float alpha = A.d[m - 1], beta = A.d_e[m - 1];
    // orgnrm = max(|alpha|, |beta|, |d_i|)  (MergeSubMatrix, svd.cpp:250-263)
    float mx = fmaxf(fabsf(alpha), fabsf(beta));
    for (int t = tid; t < n; t += 256)
        if (t != Lr) mx = fmaxf(mx, fabsf(A.d[s + t]));
    mx = warp_max(mx);
    if ((tid & 31) == 0) s_red[tid >> 5] = mx;
    for (int a = tid; a < Lr; a += 256) runs[a] = A.d[s + A.idxq[s + a]];
    for (int b = tid; b < Rr; b += 256) runs[Lr + b] = A.d[m + A.idxq[m + b]];
    __syncthreads();
    float orgnrm = s_red[0];
    for (int q = 1; q < 8; q++) orgnrm = fmaxf(orgnrm, s_red[q]);
    if (orgnrm == 0.f) orgnrm = 1.f;
    const double as = (double)alpha / orgnrm, bs = (double)beta / orgnrm;

    // every slot gets a valid default first, so that even non-finite data
    // (which breaks the ordering) leaves only in-range row indices
    for (int p = tid; p < dn; p += 256) { sd[p] = 0.f; sz[p] = 0.0; srowp[p] = 0; }
    __syncthreads();
    // sorted merge of the two ascending runs (ties: left run first)
    for (int a = tid; a < Lr; a += 256) {
        float v = runs[a];
        int p = min(dn - 1, a + count_below(runs + Lr, Rr, v, false));
        int li = min(max(A.idxq[s + a], 0), Lr - 1);
        sd[p] = v / orgnrm;
        sz[p] = as * (double)A.l[s + li];
        srowp[p] = li;
    }
    for (int b = tid; b < Rr; b += 256) {
        float v = runs[Lr + b];
        int p = min(dn - 1, b + count_below(runs, Lr, v, true));
        int ri = min(max(A.idxq[m + b], 0), Rr - 1);
        sd[p] = v / orgnrm;
        sz[p] = bs * (double)A.f[m + ri];
        srowp[p] = nl + ri;
    }
    __syncthreads();
    const double tol = 8.0 * (double)FLT_EPSILON *
                       fmax(fmax(fabs(as), fabs(bs)), dn > 0 ? fabs((double)sd[dn - 1]) : 0.0);

    // deflation scan (Deflation, svd.cpp:636-739), serial in FP64
    if (tid == 0) {
        int k = 0, kd = 0, jprev = -1, nrot = 0;
        for (int p = 0; p < dn; p++) {
            if (fabs(sz[p]) <= tol) { idxp[dn - 1 - kd++] = p; continue; }
            if (jprev < 0) { jprev = p; continue; }
            if (fabs((double)sd[p] - (double)sd[jprev]) <= tol) {
                double sn = sz[jprev], cs = sz[p], t = hypot(cs, sn);
                cs /= t; sn = -sn / t;
                sz[p] = t; sz[jprev] = 0.0;
                RotEntry re;
                re.ra = srowp[jprev]; re.rb = srowp[p]; re.c = (float)cs; re.s = (float)sn;
                A.w.rot[s + nrot++] = re;
                idxp[dn - 1 - kd++] = jprev;
                jprev = p;
            } else {
                idxp[k++] = jprev;
                jprev = p;
            }
        }
        if (jprev >= 0) idxp[k++] = jprev;
        for (int x = k, y = dn - 1; x < y; x++, y--) { int t = idxp[x]; idxp[x] = idxp[y]; idxp[y] = t; }
        // the deflated run is sorted up to inversions within tol (a small-z
        // entry can sit between a rotated pair); a stable insertion sort makes
        // it ascending so that the idxq merge of the finalize step is exact
        for (int x = k + 1; x < dn; x++) {
            int key = idxp[x];
            float kv = sd[key];
            int y = x - 1;
            while (y >= k && sd[idxp[y]] > kv) { idxp[y + 1] = idxp[y]; y--; }
            idxp[y + 1] = key;
        }
        s_knd = k;
        MergeMeta mm;
        mm.n = n; mm.nc = nc; mm.nl = nl; mm.Lr = Lr; mm.nrot = nrot; mm.sq = sq; mm.pad = 0;
        mm.orgnrm = orgnrm; mm.tol = (float)tol;
        // z0 and the extra-column rotation of a non-square block (svd.cpp:781-812)
        double z0 = as * (double)A.l[s + Lr], zz0, cns = 1.0, sns = 0.0;
        if (nc > n) {
            double zn = bs * (double)A.f[m + Rr];
            zz0 = hypot(z0, zn);
            if (zz0 <= tol) { cns = 1.0; sns = 0.0; zz0 = tol; }
            else { cns = z0 / zz0; sns = zn / zz0; }
        } else {
            zz0 = (fabs(z0) <= tol) ? tol : z0;
        }
        mm.k = k + 1;
        mm.cns = (float)cns; mm.sns = (float)sns;
        A.w.meta[s] = mm;
        A.w.zsec[s] = zz0;
        A.dsig[s] = 0.f;
        A.srow[s] = -1;
    }
    __syncthreads();
    const int knd = s_knd;
    for (int t = 1 + tid; t < n; t += 256) {
        int p = idxp[t - 1];
        A.dsig[s + t] = sd[p];
        A.srow[s + t] = srowp[p];
        if (t <= knd) A.w.zsec[s + t] = sz[p];
    }
    __syncthreads();
    // keep the smallest pole away from 0 (svd.cpp:803-809); only a pole of the
    // secular equation is moved, a deflated value keeps its place in the order
    if (tid == 0 && n > 1 && knd >= 1) {
        float h = (float)(tol / 2);
        if (fabsf(A.dsig[s + 1]) <= h) A.dsig[s + 1] = h;
    }
    __syncthreads();
    for (int t = knd + 1 + tid; t < n; t += 256) A.d[s + t] = A.dsig[s + t];
    __syncthreads();
}

// Givens rotations of the deflation of merge mg, in order, on column c
static __device__ void bdc_rotate_dev(const LevelArgs &A, int mg, int c)
{
    const int s = A.w.mg_s[A.off + mg];
    const MergeMeta mm = A.w.meta[s];
    if (c >= mm.nc || mm.nrot == 0) return;
    const int N = A.N;
    for (int t = 0; t < mm.nrot; t++) {
        RotEntry r = A.w.rot[s + t];
        if (c < mm.n) {
            float *x = A.QT + (long)(s + r.ra) * N + s + c, *y = A.QT + (long)(s + r.rb) * N + s + c;
            float a = *x, b = *y;
            *x = r.c * a + r.s * b;
            *y = -r.s * a + r.c * b;
        }
        float *x = A.WT + (long)(s + r.ra) * N + s + c, *y = A.WT + (long)(s + r.rb) * N + s + c;
        float a = *x, b = *y;
        *x = r.c * a + r.s * b;
        *y = -r.s * a + r.c * b;
    }
}

// st/gt rows [t0, t1) of merge mg in deflation order, column c (svd.cpp:787-801, 868-945)
static __device__ void bdc_gather_dev(const LevelArgs &A, int mg, int c, int t0, int t1)
{
    const int s = A.w.mg_s[A.off + mg];
    const MergeMeta mm = A.w.meta[s];
    if (c >= mm.nc) return;
    const int N = A.N;
    const long cs = s + c;
    t1 = min(t1, mm.nc);
    for (int t = t0; t < t1; t++) {
        const long rowt = (long)(s + t) * N;
        if (t == 0) {
            if (c < mm.n) A.ST[rowt + cs] = (c == mm.Lr) ? 1.f : 0.f;
            float wl = A.WT[(long)(s + mm.Lr) * N + cs];
            float g;
            if (mm.nc > mm.n) g = (c < mm.nl) ? mm.cns * wl : mm.sns * A.WT[(long)(s + mm.nc - 1) * N + cs];
            else g = wl;
            A.GT[rowt + cs] = g;
        } else if (t < mm.n) {
            long src = (long)(s + A.srow[s + t]) * N + cs;
            if (c < mm.n) A.ST[rowt + cs] = A.QT[src];
            A.GT[rowt + cs] = A.WT[src];
        } else { // t == nc - 1 of a non-square block: the new null vector
            float wl = A.WT[(long)(s + mm.Lr) * N + cs];
            float wr = A.WT[(long)(s + mm.nc - 1) * N + cs];
            A.GT[rowt + cs] = (c < mm.nl) ? -mm.sns * wl : mm.cns * wr;
        }
    }
}

// deflated rows [max(k, t0), t1) and the new null vector back into qt/wt, column c
static __device__ void bdc_copyback_dev(const LevelArgs &A, int mg, int c, int t0, int t1)
{
    const int s = A.w.mg_s[A.off + mg];
    const MergeMeta mm = A.w.meta[s];
    if (c >= mm.nc) return;
    const int N = A.N;
    const long cs = s + c;
    t0 = max(mm.k, t0);
    t1 = min(mm.nc, t1);
    for (int t = t0; t < t1; t++) {
        const long rowt = (long)(s + t) * N;
        if (t < mm.n && c < mm.n) A.QT[rowt + cs] = A.ST[rowt + cs];
        A.WT[rowt + cs] = A.GT[rowt + cs];
    }
}

// merge of a level containing column g (merge starts of a level ascend); -1 if none
static __device__ __forceinline__ int bdc_merge_of(const LevelArgs &A, int nm, int g)
{
    int lo = 0, hi = nm - 1, mg = -1;
    while (lo <= hi) {
        int mid = (lo + hi) >> 1;
        if (A.w.mg_s[A.off + mid] <= g) { mg = mid; lo = mid + 1; } else hi = mid - 1;
    }
    return mg;
}

// Sum over a group of G lanes (G = 32: the warp, G = 1: one thread).
template <int G, typename T>
static __device__ __forceinline__ T gsum(T v)
{
    if (G == 32) return warp_sum(v);
    return v;
}

// FP64 root i of 1 + sum_j z_j^2 / ((d_j - s)(d_j + s)) = 0 for the column gw
// of the level, one group of G lanes (a warp, or one thread for small merges);
// only merges with klo < k <= khi are handled.  sigma = o + tau with o the nearer pole, so
// d_j - sigma = (d_j - o) - tau keeps its relative accuracy (d_j, o are FP32
// values: d_j - o is exact).
template <int G>
static __device__ void bdc_secular_dev(const LevelArgs &A, int nm, int gw, int lane, int klo, int khi)
{
    const int N = A.N;
    if (gw >= N) return;
    const int mg = bdc_merge_of(A, nm, gw);
    if (mg < 0) return;
    const int s = A.w.mg_s[A.off + mg];
    const MergeMeta mm = A.w.meta[s];
    const int i = gw - s, k = mm.k;
    if (i >= k || i >= mm.n || k <= klo || k > khi) return;
    const float *ds = A.dsig + s;
    const double *z = A.w.zsec + s;
    float *drow = A.diff + (long)(s + i) * N + s;
    if (k == 1) {
        if (lane == 0) A.d[s] = (float)fabs(z[0]);
        return;
    }
    double o, tlo, thi;
    if (i < k - 1) {
        double dlo = ds[i], dhi = ds[i + 1], h = dhi - dlo, mid = dlo + 0.5 * h;
        double fm = 0.0;
        for (int j = lane; j < k; j += G) {
            double dj = ds[j];
            fm += z[j] * z[j] / ((dj - mid) * (dj + mid));
        }
        fm = 1.0 + gsum<G>(fm);
        if (fm > 0) { o = dlo; tlo = 0.0; thi = 0.5 * h; }
        else { o = dhi; tlo = -0.5 * h; thi = 0.0; }
    } else {
        double zn2 = 0.0;
        for (int j = lane; j < k; j += G) zn2 += z[j] * z[j];
        zn2 = gsum<G>(zn2);
        o = ds[k - 1];
        tlo = 0.0;
        thi = zn2 / (sqrt(o * o + zn2) + o);
    }
    double tau = 0.5 * (tlo + thi), fprev = 1e300;
    const double di = ds[i], dn = (i + 1 < k) ? (double)ds[i + 1] : 0.0;
    bool conv = false;
    const int maxit = g_sec_maxit;
    for (int it = 0; it < maxit; it++) {
        double p1 = 0, p2 = 0, q1 = 0, q2 = 0;
        for (int j = lane; j < k; j += G) {
            double dj = ds[j];
            double D = ((dj - o) - tau) * (dj + o + tau);
            double r = 1.0 / D;
            double t = z[j] * z[j] * r;
            if (j <= i) { p1 += t; q1 += t * r; } else { p2 += t; q2 += t * r; }
        }
        p1 = gsum<G>(p1); p2 = gsum<G>(p2); q1 = gsum<G>(q1); q2 = gsum<G>(q2);
        const double Di = ((di - o) - tau) * (di + o + tau);
        const double Dn = ((dn - o) - tau) * (dn + o + tau);
        const double fv = 1.0 + p1 + p2;
        const double tolf = 8.0 * k * DBL_EPSILON * (1.0 + fabs(p1) + fabs(p2));
        if (fabs(fv) <= tolf) { conv = true; break; }
        if (fv > 0) thi = tau; else tlo = tau;
        if (thi - tlo <= 2.0 * DBL_EPSILON * fmax(fabs(tlo), fabs(thi))) { conv = true; break; }
        double eta = CUDART_NAN;
        if (i < k - 1) {
            double c1 = q1 * Di * Di, c1h = p1 - q1 * Di;
            double c2 = q2 * Dn * Dn, c2h = p2 - q2 * Dn;
            double c3 = 1.0 + c1h + c2h;
            double qa = c3, qb = -(c3 * (Di + Dn) + c1 + c2), qc = Di * Dn * fv;
            if (qa == 0.0) {
                if (qb != 0.0) eta = -qc / qb;
            } else {
                double disc = fmax(qb * qb - 4.0 * qa * qc, 0.0);
                double q = -0.5 * (qb + copysign(sqrt(disc), qb));
                double r1 = q / qa, r2 = (q != 0.0) ? qc / q : CUDART_NAN;
                if (r1 > Di && r1 < Dn) eta = r1;
                else if (r2 > Di && r2 < Dn) eta = r2;
            }
        } else {
            double c1 = q1 * Di * Di, c1h = p1 - q1 * Di;
            if (1.0 + c1h > 0.0) eta = Di + c1 / (1.0 + c1h);
        }
        double tn = CUDART_NAN;
        if (isfinite(eta)) {
            double sg = o + tau, s2 = sg * sg + eta;
            if (s2 > 0.0) tn = tau + eta / (sg + sqrt(s2));
        }
        if (!(tn > tlo && tn < thi) || (it > 2 && fabs(fv) > 0.5 * fprev)) tn = 0.5 * (tlo + thi);
        fprev = fabs(fv);
        tau = tn;
    }
    if (!conv && lane == 0) atomicAdd(&A.w.st->secular_nonconv, 1);
    for (int j = lane; j < k; j += G) {
        double dj = ds[j];
        drow[j] = (float)(((dj - o) - tau) * (dj + o + tau));
    }
    if (lane == 0) A.d[s + i] = (float)(o + tau);
}

// Loewner (Gu-Eisenstat) z of the pole at column g, one group of G lanes:
// each lane multiplies the FP64 ratios of its share of j, then a butterfly
// product combines the lanes (the same product in every lane, so the result
// is reproducible) (svd.cpp:1422-1438); only merges with klo < k <= khi.
template <int G>
static __device__ void bdc_lowner_dev(const LevelArgs &A, int nm, int g, int lane, int klo, int khi)
{
    const int N = A.N;
    if (g >= N) return;
    const int mg = bdc_merge_of(A, nm, g);
    if (mg < 0) return;
    const int s = A.w.mg_s[A.off + mg];
    const MergeMeta mm = A.w.meta[s];
    const int i = g - s, k = mm.k;
    if (i >= k || k < 2 || k <= klo || k > khi) return;
    const float *ds = A.dsig + s;
    const float *D = A.diff + (long)s * N + s; // D[j*N + i] = d_i^2 - sigma_j^2
    const double dii = ds[i];
    double p = 1.0;
    for (int j = lane; j < k - 1; j += G) {
        double dj = (j < i) ? (double)ds[j] : (double)ds[j + 1];
        p *= (double)D[(long)j * N + i] / ((dii - dj) * (dii + dj));
    }
    if (G == 32) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) p *= __shfl_xor_sync(0xffffffffu, p, o);
    }
    p *= (double)D[(long)(k - 1) * N + i];
    if (lane == 0) A.zhat[s + i] = (float)copysign(sqrt(fabs(p)), A.w.zsec[s + i]);
}

// normalized singular vectors of the secular problem for column gw, one group
// of G lanes (svd.cpp:1440-1496); only merges with klo < k <= khi.
template <int G>
static __device__ void bdc_vectors_dev(const LevelArgs &A, int nm, int gw, int lane, int klo, int khi)
{
    const int N = A.N;
    if (gw >= N) return;
    const int mg = bdc_merge_of(A, nm, gw);
    if (mg < 0) return;
    const int s = A.w.mg_s[A.off + mg];
    const MergeMeta mm = A.w.meta[s];
    const int i = gw - s, k = mm.k;
    if (i >= k || i >= mm.n || k <= klo || k > khi) return;
    float *us = A.w.Us + (long)(s + i) * N + s, *vs = A.w.Vs + (long)(s + i) * N + s;
    if (k == 1) {
        if (lane == 0) { us[0] = (float)sgn1(A.w.zsec[s]); vs[0] = 1.f; }
        return;
    }
    const float *ds = A.dsig + s, *zh = A.zhat + s;
    const float *Drow = A.diff + (long)(s + i) * N + s;
    double nv = 0.0, nu = 0.0;
    for (int j = lane; j < k; j += G) {
        double v = (double)zh[j] / (double)Drow[j];
        double u = (j == 0) ? -1.0 : (double)ds[j] * v;
        nv += v * v; nu += u * u;
    }
    nv = 1.0 / sqrt(gsum<G>(nv));
    nu = 1.0 / sqrt(gsum<G>(nu));
    for (int j = lane; j < k; j += G) {
        double v = (double)zh[j] / (double)Drow[j];
        double u = (j == 0) ? -1.0 : (double)ds[j] * v;
        vs[j] = (float)(v * nv);
        us[j] = (float)(u * nu);
    }
}

// Tile (tm, tn) of qt[s:s+k, s:s+n] = Us st[s:s+k, s:s+n] (which = 0) or
// wt[s:s+k, s:s+nc] = Vs gt[s:s+k, s:s+nc] (which = 1).  256 threads.
static __device__ void bdc_btgemm_dev(const LevelArgs &A, int mg, int which, int tm, int tn)
{
    const int s = A.w.mg_s[A.off + mg];
    const MergeMeta mm = A.w.meta[s];
    const int N = A.N;
    const int k = mm.k, ncols = which ? mm.nc : mm.n;
    if (tm * 128 >= k || tn * 128 >= ncols) return;
    const long off = (long)s * N + s;
    const float *Asrc = which ? A.w.Vs : A.w.Us;
    const float *Bsrc = which ? A.GT : A.ST;
    float *C = which ? A.WT : A.QT;
    gemm_tile(k, ncols, 0, k, 1.f, gop(Asrc + off, N, 1), gop(Bsrc + off, N, 1), 0.f, C + off, N, tm * 128,
              tn * 128);
}

// f/l of the merged block, its idxq, and the unscaling of d.  256 threads.
static __device__ void bdc_finalize_dev(const LevelArgs &A, int mg)
{
    const int s = A.w.mg_s[A.off + mg];
    const MergeMeta mm = A.w.meta[s];
    const int N = A.N, n = mm.n, nc = mm.nc, k = mm.k;
    const int tid = threadIdx.x;
    for (int t = tid; t < nc; t += 256) {
        if (t < n || t == nc - 1) {
            A.f[s + t] = A.WT[(long)(s + t) * N + s];
            A.l[s + t] = A.WT[(long)(s + t) * N + s + nc - 1];
        }
    }
    // idxq: stable merge of d[0:k) (roots) and d[k:n) (deflated), both ascending
    const float *dd = A.d + s;
    for (int t = tid; t < n; t += 256) A.idxq[s + t] = t;
    __syncthreads();
    for (int a = tid; a < k; a += 256) A.idxq[s + min(n - 1, a + count_below(dd + k, n - k, dd[a], false))] = a;
    for (int b = tid; b < n - k; b += 256) A.idxq[s + min(n - 1, b + count_below(dd, k, dd[k + b], true))] = k + b;
    __syncthreads();
    for (int t = tid; t < n; t += 256) A.d[s + t] = dd[t] * mm.orgnrm;
    __syncthreads();
}

// Descending rank of d[i] for i = base + threadIdx.x (ties: lower index
// first); perm[rank] = i, sig[rank] = d[i].  All threads of the CTA call it
// with the same base.
static __device__ void bdc_rank_desc_dev(int N, const float *d, int *perm, float *sig, int base)
{
    __shared__ float tile[1024];
    const int i = base + threadIdx.x;
    // NaN is ordered below -inf, which keeps the ranks a permutation
    auto key = [](float x) { return isnan(x) ? -CUDART_INF_F : x; };
    const float v = (i < N) ? key(d[i]) : 0.f;
    int rank = 0;
    for (int j0 = 0; j0 < N; j0 += 1024) {
        __syncthreads();
        for (int t = threadIdx.x; t < 1024; t += blockDim.x) tile[t] = (j0 + t < N) ? key(d[j0 + t]) : 0.f;
        __syncthreads();
        if (i < N) {
            int jn = min(1024, N - j0);
            for (int t = 0; t < jn; t++) {
                float x = tile[t];
                rank += (x > v) || (x == v && j0 + t < i);
            }
        }
    }
    __syncthreads();
    if (i < N) { perm[rank] = i; sig[rank] = d[i]; }
}
