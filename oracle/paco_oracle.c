/*
 * paco_oracle.c -- TEST INFRASTRUCTURE ONLY (the parity checker; see the
 * header).  A plain-C, FP64 restatement of the reference's two device kernels.
 * It follows the reference's data layout (qt/wt rows, f/l, idxq, idxp) and its
 * step order, with the deviations listed below, each of which fixes a defect
 * of the reference that would make its output wrong:
 *
 *  (D1) Leaves (svd.cpp:1596-1864): the closed forms there divide by zero when
 *       an off-diagonal is exactly 0 and, for the 2x2 cases, pick the sign of
 *       the right vector independently of the left one (wrong when a11 < 0).
 *       Here every leaf is reduced to a 2x2 upper-triangular block by Givens
 *       rotations and solved with sign-consistent formulas; the leaf partition
 *       and the qt/wt/d/idxq/f/l contract are unchanged.
 *  (D2) k == 2 merges (svd.cpp:1379-1411) use the general secular path for the
 *       same sign reason.
 *  (D3) When every z is deflated, svd.cpp:654-660 jumps past the reversal of
 *       idxp (svd.cpp:733-739), leaving the deflated values descending; the
 *       reversal is applied in all cases so the merged d stays sorted.
 *  (D4) orgnrm == 0 (svd.cpp:262, a TODO there) skips the scaling.
 *  (D5) Secular roots are found in FP64 with a bracketed rational iteration
 *       (the reference's FP32 solver, svd.cpp:977-1336, keeps no bracket).
 *  (D6) N <= 2 uses a single leaf [0,N) (svd_tiling.cpp:104-128 writes
 *       svdStack[-1] for N <= 2; svd.cpp:140-159 special-cases these N).
 *  (D7) The final descending order is a full stable sort of d: the merge of
 *       idxq runs (svd.cpp:1523-1590) assumes both runs sorted, which the
 *       tol/2 substitution of svd.cpp:805-809 can break for tiny values.
 *  (D8) The deflated values are kept ascending (stable sort of their idxp
 *       run, whose order a small-z entry between a rotated pair disturbs by
 *       less than tol), and the tol/2 substitution moves a secular pole only.
 */
#include "paco_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define SEC_MAXIT 100

static double sgn1(double x) { return x < 0 ? -1.0 : 1.0; }

/* ------------------------------------------------------------------ tiling */

int oracle_leaf_partition(int N, int *starts, int *ends)
{
    /* svd_tiling.cpp:83-130: N/3+1 entries; leaves are (c-1) x c blocks except
     * the last, which is square.  remainder 0: ... 2x3, 1x2, 1x1;
     * remainder 1: ... 2x3, 1x1; remainder 2: ... 2x3, 2x2. */
    if (N <= 0) return 0;
    if (N <= 2) { starts[0] = 0; ends[0] = N; return 1; }
    int total = N / 3 + 1, rem = N % 3;
    for (int i = 0; i < total - 2; i++) { starts[i] = 3 * i; ends[i] = 3 * i + 3; }
    int i = total - 2;
    starts[i] = 3 * i;
    ends[i] = 3 * i + (rem == 0 ? 2 : 3);
    i = total - 1;
    if (rem == 0) { starts[i] = 3 * i - 1; ends[i] = 3 * i; }
    else if (rem == 1) { starts[i] = 3 * i; ends[i] = 3 * i + 1; }
    else { starts[i] = 3 * i; ends[i] = 3 * i + 2; }
    return total;
}

/* ----------------------------------------------------------------- stage 1 */

/* Reflector of upper_bidiagonalization.cpp:182-218: sigma = sum x[1:]^2,
 * mu = +sqrt(x0^2+sigma); v0 = x0-mu (x0<=0) or -sigma/(x0+mu) (Parlett);
 * tau = 2 v0^2/(sigma+v0^2); x[1:] <- x[1:]/v0, x0 <- mu.  sigma==0 or a
 * length-1 vector gives tau=0 and keeps x untouched. */
static void house(double *x, int len, long stride, double *beta, double *tau)
{
    double x0 = x[0];
    if (len <= 1) { *tau = 0; *beta = x0; return; }
    double sigma = 0;
    for (int r = 1; r < len; r++) sigma += x[r * stride] * x[r * stride];
    if (sigma == 0) { *tau = 0; *beta = x0; return; }
    double mu = sqrt(x0 * x0 + sigma);
    double v0 = (x0 <= 0) ? x0 - mu : -sigma / (x0 + mu);
    *tau = 2 * v0 * v0 / (sigma + v0 * v0);
    double inv = 1.0 / v0;
    for (int r = 1; r < len; r++) x[r * stride] *= inv;
    x[0] = mu;
    *beta = mu;
}

int oracle_bidiag(int M, int N, double *A, double *U, double *Vt,
                  double *d, double *e, double *tauq, double *taup)
{
    if (M < N || N <= 0) return 1;
    for (int i = 0; i < N; i++) {
        /* column reflector (upper_bidiagonalization.cpp:123-150) */
        double *col = A + (long)i * N + i;
        house(col, M - i, N, &d[i], &tauq[i]);
        if (tauq[i] != 0) {
            /* ApplyColumnTransformV2 (:426-474): every trailing column */
            for (int j = i + 1; j < N; j++) {
                double s = A[(long)i * N + j];
                for (int r = i + 1; r < M; r++) s += A[(long)r * N + j] * A[(long)r * N + i];
                s *= tauq[i];
                A[(long)i * N + j] -= s;
                for (int r = i + 1; r < M; r++) A[(long)r * N + j] -= s * A[(long)r * N + i];
            }
        }
        if (i < N - 1) {
            /* row reflector (:151-180) */
            double *row = A + (long)i * N + i + 1;
            house(row, N - i - 1, 1, &e[i], &taup[i]);
            if (taup[i] != 0) {
                /* ApplyRowTransformV2 (:475-528): every trailing row */
                for (int j = i + 1; j < M; j++) {
                    double *aj = A + (long)j * N;
                    double s = aj[i + 1];
                    for (int c = i + 2; c < N; c++) s += aj[c] * row[c - i - 1];
                    s *= taup[i];
                    aj[i + 1] -= s;
                    for (int c = i + 2; c < N; c++) aj[c] -= s * row[c - i - 1];
                }
            }
        }
    }
    /* GetUVt (:774-893): backward accumulation from the identity */
    memset(U, 0, sizeof(double) * (size_t)M * M);
    for (int r = 0; r < M; r++) U[(long)r * M + r] = 1;
    for (int i = N - 1; i >= 0; i--) {
        if (tauq[i] == 0) continue;
        for (int j = i; j < M; j++) {
            double s = U[(long)i * M + j];
            for (int r = i + 1; r < M; r++) s += U[(long)r * M + j] * A[(long)r * N + i];
            s *= tauq[i];
            U[(long)i * M + j] -= s;
            for (int r = i + 1; r < M; r++) U[(long)r * M + j] -= s * A[(long)r * N + i];
        }
    }
    memset(Vt, 0, sizeof(double) * (size_t)N * N);
    for (int r = 0; r < N; r++) Vt[(long)r * N + r] = 1;
    for (int i = N - 2; i >= 0; i--) {
        if (taup[i] == 0) continue;
        const double *u = A + (long)i * N + i + 1; /* u[0] is implicitly 1 */
        for (int j = i; j < N; j++) {
            double *vj = Vt + (long)j * N + i + 1;
            double s = vj[0];
            for (int c = 1; c < N - i - 1; c++) s += vj[c] * u[c];
            s *= taup[i];
            vj[0] -= s;
            for (int c = 1; c < N - i - 1; c++) vj[c] -= s * u[c];
        }
    }
    return 0;
}

/* ----------------------------------------------------------------- leaves */

/* SVD of the upper-triangular 2x2 [[f,g],[0,h]]: B v_i = s_i u_i, s1 >= s2 >= 0,
 * V = [v1 v2] a rotation, u2 chosen so that det[u1 u2] = sign(f h). */
static void svd2x2(double f, double g, double h, double *s, double *u, double *v)
{
    /* u, v: row-major 2x2 with row i = vector i */
    if (g == 0) {
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
    double s1sq = s1 * s1;
    double ax = f * g, ay = s1sq - f * f;
    double bx = s1sq - g * g - h * h, by = f * g;
    double vx, vy;
    if (ax * ax + ay * ay >= bx * bx + by * by) { vx = ax; vy = ay; } else { vx = bx; vy = by; }
    double nv = hypot(vx, vy);
    vx /= nv; vy /= nv;
    double ux = (f * vx + g * vy), uy = h * vy;
    double nu = hypot(ux, uy);
    ux /= nu; uy /= nu;
    double sd = (f * h >= 0) ? 1.0 : -1.0;
    s[0] = s1; s[1] = s2;
    v[0] = vx; v[1] = vy; v[2] = -vy; v[3] = vx;
    u[0] = ux; u[1] = uy; u[2] = -sd * uy; u[3] = sd * ux;
}

typedef struct {
    int M, N;
    double *d, *e, *f, *l, *qt, *wt, *st, *gt;
    int *idxq;
    int merges, deflated, maxit, nonconv;
} bdc_ctx;

#define QT(c, r, col) (c)->qt[(long)(r) * (c)->N + (col)]
#define WT(c, r, col) (c)->wt[(long)(r) * (c)->N + (col)]
#define ST(c, r, col) (c)->st[(long)(r) * (c)->N + (col)]
#define GT(c, r, col) (c)->gt[(long)(r) * (c)->N + (col)]

static void leaf_svd(bdc_ctx *c, int s, int e_end)
{
    /* compute_base_case_svd (svd.cpp:1596-1625) with the solves of (D1) */
    const int N = c->N;
    int cols = e_end - s, rows = (e_end == N) ? cols : cols - 1;
    double *d = c->d + s;
    double ev = (s == N - 1) ? 0.0 : c->e[s];
    double sv[2], u[4], v[4];
    if (rows == 1 && cols == 1) {
        c->idxq[s] = 0;
        QT(c, s, s) = sgn1(d[0]);
        WT(c, s, s) = 1;
        d[0] = fabs(d[0]);
    } else if (rows == 1 && cols == 2) {
        double a = d[0], b = ev, sq = hypot(a, b);
        c->idxq[s] = 0;
        d[0] = sq;
        if (sq != 0) {
            WT(c, s, s) = a / sq; WT(c, s, s + 1) = b / sq;
            WT(c, s + 1, s) = b / sq; WT(c, s + 1, s + 1) = -a / sq;
        }
    } else if (rows == 2 && cols == 2) {
        svd2x2(d[0], ev, d[1], sv, u, v);
        c->idxq[s] = 1; c->idxq[s + 1] = 0;
        d[0] = sv[0]; d[1] = sv[1];
        for (int i = 0; i < 2; i++)
            for (int j = 0; j < 2; j++) { QT(c, s + i, s + j) = u[2 * i + j]; WT(c, s + i, s + j) = v[2 * i + j]; }
    } else { /* rows == 2, cols == 3: [[a,b,0],[0,cc,ee]] */
        double a = d[0], b = ev, cc = d[1], ee = c->e[s + 1];
        double r1 = hypot(cc, ee), c1 = 1, s1 = 0;
        if (r1 != 0) { c1 = cc / r1; s1 = ee / r1; }
        double r2 = hypot(a, s1 * b), c2 = 1, s2 = 0;
        if (r2 != 0) { c2 = a / r2; s2 = -s1 * b / r2; }
        svd2x2(r2, c1 * b, r1, sv, u, v);
        /* G = G1*G2 (columns (1,2) then (0,2)) */
        double G[3][3] = {{c2, 0, -s2}, {-s1 * s2, c1, -s1 * c2}, {c1 * s2, s1, c1 * c2}};
        c->idxq[s] = 1; c->idxq[s + 1] = 0;
        d[0] = sv[0]; d[1] = sv[1];
        for (int i = 0; i < 2; i++) {
            QT(c, s + i, s) = u[2 * i]; QT(c, s + i, s + 1) = u[2 * i + 1];
            for (int r = 0; r < 3; r++) WT(c, s + i, s + r) = G[r][0] * v[2 * i] + G[r][1] * v[2 * i + 1];
        }
        for (int r = 0; r < 3; r++) WT(c, s + 2, s + r) = G[r][2];
    }
    for (int j = 0; j < cols; j++) {
        c->f[s + j] = WT(c, s + j, s);
        c->l[s + j] = WT(c, s + j, s + cols - 1);
    }
}

/* ------------------------------------------------------------- secular root */

int oracle_secular_root(int k, const double *ds, const double *z, int i,
                        double *sigma, double *diff)
{
    if (k == 1) {
        *sigma = fabs(z[0]);
        diff[0] = (ds[0] - *sigma) * (ds[0] + *sigma);
        return 0;
    }
    double o, tlo, thi;
    if (i < k - 1) {
        double lo = ds[i], hi = ds[i + 1], h = hi - lo, mid = lo + 0.5 * h;
        double fm = 1;
        for (int j = 0; j < k; j++) fm += z[j] * z[j] / ((ds[j] - mid) * (ds[j] + mid));
        /* svd.cpp:1075-1089: origin by the sign of f at the midpoint */
        if (fm > 0) { o = lo; tlo = 0; thi = 0.5 * h; }
        else { o = hi; tlo = -0.5 * h; thi = 0; }
    } else {
        double zn2 = 0;
        for (int j = 0; j < k; j++) zn2 += z[j] * z[j];
        o = ds[k - 1];
        tlo = 0;
        thi = zn2 / (sqrt(o * o + zn2) + o);
    }
    double tau = 0.5 * (tlo + thi), fprev = INFINITY;
    int it, conv = 0;
    for (it = 0; it < SEC_MAXIT; it++) {
        double psi1 = 0, psi2 = 0, dp1 = 0, dp2 = 0, Di = 0, Dn = 0;
        for (int j = 0; j < k; j++) {
            double D = ((ds[j] - o) - tau) * (ds[j] + o + tau);
            double t = z[j] * z[j] / D;
            if (j <= i) { psi1 += t; dp1 += t / D; } else { psi2 += t; dp2 += t / D; }
            if (j == i) Di = D;
            if (j == i + 1) Dn = D;
        }
        double fv = 1 + psi1 + psi2;
        double tolf = 8.0 * k * DBL_EPSILON * (1 + fabs(psi1) + fabs(psi2));
        if (fabs(fv) <= tolf) { conv = 1; break; }
        if (fv > 0) thi = tau; else tlo = tau;
        if (thi - tlo <= 2 * DBL_EPSILON * fmax(fabs(tlo), fabs(thi))) { conv = 1; break; }
        double eta = NAN;
        if (i < k - 1) {
            double c1 = dp1 * Di * Di, c1h = psi1 - dp1 * Di;
            double c2 = dp2 * Dn * Dn, c2h = psi2 - dp2 * Dn;
            double c3 = 1 + c1h + c2h;
            double qa = c3, qb = -(c3 * (Di + Dn) + c1 + c2), qc = Di * Dn * fv;
            if (qa == 0) {
                if (qb != 0) eta = -qc / qb;
            } else {
                double disc = qb * qb - 4 * qa * qc;
                if (disc < 0) disc = 0;
                double q = -0.5 * (qb + copysign(sqrt(disc), qb));
                double r1 = q / qa, r2 = (q != 0) ? qc / q : NAN;
                if (r1 > Di && r1 < Dn) eta = r1;
                else if (r2 > Di && r2 < Dn) eta = r2;
            }
        } else {
            double c1 = dp1 * Di * Di, c1h = psi1 - dp1 * Di;
            if (1 + c1h > 0) eta = Di + c1 / (1 + c1h);
        }
        double tn = NAN;
        if (isfinite(eta)) {
            double sg = o + tau, s2 = sg * sg + eta;
            if (s2 > 0) tn = tau + eta / (sg + sqrt(s2));
        }
        /* bracket safeguard: bisect when the model leaves the bracket or
         * |f| failed to halve */
        if (!(tn > tlo && tn < thi) || (it > 2 && fabs(fv) > 0.5 * fprev)) tn = 0.5 * (tlo + thi);
        fprev = fabs(fv);
        tau = tn;
    }
    *sigma = o + tau;
    for (int j = 0; j < k; j++) diff[j] = ((ds[j] - o) - tau) * (ds[j] + o + tau);
    return conv ? it : -1;
}

/* ------------------------------------------------------------------ merges */

static void rotate_rows(double *x, double *y, int len, double cs, double sn)
{
    for (int t = 0; t < len; t++) {
        double a = x[t], b = y[t];
        x[t] = cs * a + sn * b;
        y[t] = -sn * a + cs * b;
    }
}

/* stable merge of two ascending runs a[0..na), b[0..nb): out[p] = index of the
 * p-th smallest in the concatenation (ties: left run first) */
static void merge_runs(const double *a, int na, const double *b, int nb, int *out)
{
    int p = 0, x = 0, y = 0;
    while (x < na && y < nb) out[p++] = (b[y] < a[x]) ? na + y++ : x++;
    while (x < na) out[p++] = x++;
    while (y < nb) out[p++] = na + y++;
}

static void merge_blocks(bdc_ctx *c, int s, int m, int e_end)
{
    const int N = c->N;
    const int nl = m - s, nr = e_end - m, sq = (e_end == N);
    const int Lr = nl - 1, Rr = nr - 1 + sq, n = Lr + Rr + 1, nc = n + 1 - sq;
    double *d = c->d + s, *f = c->f + s, *l = c->l + s;
    int *idxq = c->idxq + s;
    double *z = calloc(n + 2, sizeof(double)), *zs = calloc(n + 2, sizeof(double));
    double *runv = calloc(n + 1, sizeof(double)), *dsig = calloc(n + 1, sizeof(double));
    double *diff = calloc((size_t)n * n, sizeof(double)), *Us = calloc((size_t)n * n, sizeof(double));
    double *Vs = calloc((size_t)n * n, sizeof(double)), *tmp = calloc((size_t)n * (n + 1), sizeof(double));
    int *perm = calloc(n + 1, sizeof(int)), *orig = calloc(n + 1, sizeof(int));
    int *idxp = calloc(n + 1, sizeof(int)), *srow = calloc(n + 1, sizeof(int));

    /* MergeSubMatrix scaling (svd.cpp:240-284) */
    double alpha = d[Lr], beta = c->e[m - 1];
    d[Lr] = 0;
    double orgnrm = fmax(fabs(alpha), fabs(beta));
    for (int i = 0; i < n; i++) orgnrm = fmax(orgnrm, fabs(d[i]));
    if (orgnrm == 0) orgnrm = 1; /* (D4) */
    alpha /= orgnrm; beta /= orgnrm;
    for (int i = 0; i < n; i++) d[i] /= orgnrm;

    /* Deflation: z, shifted d, shifted idxq (svd.cpp:339-429) */
    z[0] = alpha * l[Lr];
    for (int j = 0; j < Lr; j++) z[1 + j] = alpha * l[j];
    for (int j = 0; j < nr; j++) z[nl + j] = beta * f[nl + j];
    for (int j = Lr - 1; j >= 0; j--) { d[j + 1] = d[j]; idxq[j + 1] = idxq[j] + 1; }
    d[0] = 0;
    for (int j = 0; j < Rr; j++) idxq[nl + j] += nl;

    /* sorted merge of the two ascending runs (svd.cpp:447-593) */
    const int dn = n - 1;
    for (int j = 0; j < dn; j++) runv[j] = d[idxq[1 + j]];
    merge_runs(runv, Lr, runv + Lr, Rr, perm);
    for (int p = 0; p < dn; p++) {
        orig[1 + p] = idxq[1 + perm[p]];
        zs[1 + p] = z[orig[1 + p]];
        dsig[1 + p] = runv[perm[p]];
    }
    for (int p = 1; p <= dn; p++) { d[p] = dsig[p]; z[p] = zs[p]; }

    /* deflation scan (svd.cpp:636-739) */
    double tol = 8.0 * FLT_EPSILON * fmax(fmax(fabs(alpha), fabs(beta)), fabs(d[dn]));
    int k = 0, k2 = n, jprev = -1;
#define ROWOF(pos) ((pos) < nl ? (pos) - 1 : (pos))
    for (int j = 1; j < n; j++) {
        if (fabs(z[j]) <= tol) { idxp[--k2] = j; continue; }
        if (jprev < 0) { jprev = j; continue; }
        if (fabs(d[j] - d[jprev]) <= tol) {
            double sn = z[jprev], cs = z[j], t = hypot(cs, sn);
            cs /= t; sn = -sn / t;
            z[j] = t; z[jprev] = 0;
            int rp = ROWOF(orig[jprev]), rj = ROWOF(orig[j]);
            rotate_rows(&QT(c, s + rp, s), &QT(c, s + rj, s), n, cs, sn);
            rotate_rows(&WT(c, s + rp, s), &WT(c, s + rj, s), nc, cs, sn);
            idxp[--k2] = jprev;
            jprev = j;
        } else {
            idxp[++k] = jprev;
            jprev = j;
        }
    }
    if (jprev >= 0) idxp[++k] = jprev;
    for (int a = k + 1, b = n - 1; a < b; a++, b--) { int t = idxp[a]; idxp[a] = idxp[b]; idxp[b] = t; } /* (D3) */
    /* (D8) stable insertion sort of the deflated run by value: a small-z entry
     * between a rotated pair leaves inversions within tol */
    for (int a = k + 2; a < n; a++) {
        int key = idxp[a], b = a - 1;
        while (b >= k + 1 && d[idxp[b]] > d[key]) { idxp[b + 1] = idxp[b]; b--; }
        idxp[b + 1] = key;
    }
    c->deflated += (n - 1) - k;

    /* dsigma, st/gt gathers (svd.cpp:741-801) */
    for (int j = 1; j < n; j++) { dsig[j] = d[idxp[j]]; srow[j] = ROWOF(orig[idxp[j]]); }
    dsig[0] = 0;
    if (k >= 1 && fabs(dsig[1]) <= tol / 2) dsig[1] = tol / 2; /* (D8) poles only */
    double cns = 1, sns = 0;
    if (nc > n) {
        double z0 = z[0];
        z[0] = hypot(z0, z[n]);
        if (z[0] <= tol) { cns = 1; sns = 0; z[0] = tol; }
        else { cns = z0 / z[0]; sns = z[n] / z[0]; }
    } else if (fabs(z[0]) <= tol) {
        z[0] = tol;
    }
    k++;
    zs[0] = z[0];
    for (int j = 1; j < k; j++) zs[j] = z[idxp[j]];
    for (int j = 1; j < n; j++) {
        memcpy(&ST(c, s + j, s), &QT(c, s + srow[j], s), sizeof(double) * n);
        memcpy(&GT(c, s + j, s), &WT(c, s + srow[j], s), sizeof(double) * nc);
    }
    for (int t = 0; t < n; t++) ST(c, s, s + t) = (t == Lr) ? 1.0 : 0.0;
    if (nc > n) {
        for (int t = 0; t < nc; t++) {
            double wl = WT(c, s + Lr, s + t), wr = WT(c, s + nc - 1, s + t);
            GT(c, s, s + t) = (t < nl) ? cns * wl : sns * wr;
            GT(c, s + nc - 1, s + t) = (t < nl) ? -sns * wl : cns * wr;
        }
        memcpy(&WT(c, s + nc - 1, s), &GT(c, s + nc - 1, s), sizeof(double) * nc);
        f[nc - 1] = GT(c, s + nc - 1, s);
        l[nc - 1] = GT(c, s + nc - 1, s + nc - 1);
    } else {
        memcpy(&GT(c, s, s), &WT(c, s + Lr, s), sizeof(double) * nc);
    }
    for (int j = k; j < n; j++) {
        d[j] = dsig[j];
        memcpy(&QT(c, s + j, s), &ST(c, s + j, s), sizeof(double) * n);
        memcpy(&WT(c, s + j, s), &GT(c, s + j, s), sizeof(double) * nc);
        f[j] = GT(c, s + j, s);
        l[j] = GT(c, s + j, s + nc - 1);
    }

    /* MergeSubMatrix_step2 (svd.cpp:1337-1594) */
    if (k == 1) {
        d[0] = fabs(z[0]);
        memcpy(&WT(c, s, s), &GT(c, s, s), sizeof(double) * nc);
        f[0] = GT(c, s, s); l[0] = GT(c, s, s + nc - 1);
        double sg = (z[0] < 0) ? -1.0 : 1.0;
        for (int t = 0; t < n; t++) QT(c, s, s + t) = sg * ST(c, s, s + t);
    } else {
        for (int i = 0; i < k; i++) {
            double sig;
            int it = oracle_secular_root(k, dsig, zs, i, &sig, diff + (long)i * k);
            if (it < 0) c->nonconv++; else if (it > c->maxit) c->maxit = it;
            d[i] = sig;
        }
        /* Loewner z (svd.cpp:1422-1438), in FP64 */
        double *zh = tmp;
        for (int i = 0; i < k; i++) {
            double p = diff[(long)(k - 1) * k + i];
            for (int j = 0; j < i; j++) p *= diff[(long)j * k + i] / ((dsig[i] - dsig[j]) * (dsig[i] + dsig[j]));
            for (int j = i; j < k - 1; j++) p *= diff[(long)j * k + i] / ((dsig[i] - dsig[j + 1]) * (dsig[i] + dsig[j + 1]));
            zh[i] = copysign(sqrt(fabs(p)), zs[i]);
        }
        /* singular vectors of the secular problem (svd.cpp:1440-1496) */
        for (int i = 0; i < k; i++) {
            double nv = 0, nu = 0;
            for (int j = 0; j < k; j++) {
                double v = zh[j] / diff[(long)i * k + j];
                double u = (j == 0) ? -1.0 : dsig[j] * v;
                Vs[(long)i * k + j] = v; Us[(long)i * k + j] = u;
                nv += v * v; nu += u * u;
            }
            nv = 1.0 / sqrt(nv); nu = 1.0 / sqrt(nu);
            for (int j = 0; j < k; j++) { Vs[(long)i * k + j] *= nv; Us[(long)i * k + j] *= nu; }
        }
        /* back-transform (svd.cpp:1498-1521): qt[0:k] = Us*st[0:k], wt[0:k] = Vs*gt[0:k] */
        for (int i = 0; i < k; i++)
            for (int t = 0; t < n; t++) {
                double acc = 0;
                for (int j = 0; j < k; j++) acc += Us[(long)i * k + j] * ST(c, s + j, s + t);
                tmp[(long)i * (n + 1) + t] = acc;
            }
        for (int i = 0; i < k; i++) memcpy(&QT(c, s + i, s), tmp + (long)i * (n + 1), sizeof(double) * n);
        for (int i = 0; i < k; i++)
            for (int t = 0; t < nc; t++) {
                double acc = 0;
                for (int j = 0; j < k; j++) acc += Vs[(long)i * k + j] * GT(c, s + j, s + t);
                tmp[(long)i * (n + 1) + t] = acc;
            }
        for (int i = 0; i < k; i++) {
            memcpy(&WT(c, s + i, s), tmp + (long)i * (n + 1), sizeof(double) * nc);
            f[i] = WT(c, s + i, s);
            l[i] = WT(c, s + i, s + nc - 1);
        }
    }
    /* FormIdxq (svd.cpp:1523-1590) */
    merge_runs(d, k, d + k, n - k, idxq);
    for (int i = 0; i < n; i++) d[i] *= orgnrm;
    c->merges++;
#undef ROWOF
    free(z); free(zs); free(runv); free(dsig); free(diff); free(Us); free(Vs); free(tmp);
    free(perm); free(orig); free(idxp); free(srow);
}

int oracle_bdc(int M, int N, double *d, double *e, double *U, double *Vt, int *stats)
{
    if (M < N || N <= 0) return 1;
    bdc_ctx c;
    memset(&c, 0, sizeof(c));
    c.M = M; c.N = N; c.d = d; c.e = e;
    size_t nn = (size_t)N * N;
    c.qt = calloc(nn, sizeof(double)); c.wt = calloc(nn, sizeof(double));
    c.st = calloc(nn, sizeof(double)); c.gt = calloc(nn, sizeof(double));
    c.f = calloc(N, sizeof(double)); c.l = calloc(N, sizeof(double));
    c.idxq = calloc(N, sizeof(int));
    for (int i = 0; i < N; i++) { c.qt[(long)i * N + i] = 1; c.wt[(long)i * N + i] = 1; }

    int *ls = malloc(sizeof(int) * (N / 3 + 2)), *le = malloc(sizeof(int) * (N / 3 + 2));
    int nleaf = oracle_leaf_partition(N, ls, le);
    for (int i = 0; i < nleaf; i++) leaf_svd(&c, ls[i], le[i]);
    /* merge tree (svd.cpp:168-189): adjacent pairs, odd tail carried */
    while (nleaf > 1) {
        int w = 0, r = 0;
        while (r < nleaf - 1) {
            merge_blocks(&c, ls[r], ls[r + 1], le[r + 1]);
            ls[w] = ls[r]; le[w] = le[r + 1]; w++; r += 2;
        }
        if (r == nleaf - 1) { ls[w] = ls[r]; le[w] = le[r]; w++; }
        nleaf = w;
    }
    /* rearrange_qwtAccordingToIdxq (svd.cpp:1866-1909): descending order,
     * as a full stable sort (D7): rank(i) = #{d_j > d_i} + #{j < i: d_j == d_i} */
    double *dd = malloc(sizeof(double) * N);
    int *perm = malloc(sizeof(int) * N);
    for (int i = 0; i < N; i++) {
        int rank = 0;
        for (int j = 0; j < N; j++) rank += (d[j] > d[i]) || (d[j] == d[i] && j < i);
        perm[rank] = i;
    }
    for (int r = 0; r < N; r++) dd[r] = d[perm[r]];
    memcpy(d, dd, sizeof(double) * N);
    for (int r = 0; r < N; r++) {
        memcpy(c.st + (long)r * N, c.qt + (long)perm[r] * N, sizeof(double) * N);
        memcpy(c.gt + (long)r * N, c.wt + (long)perm[r] * N, sizeof(double) * N);
    }
    free(perm);
    /* updateUVt (svd.cpp:1911-1981): U[:, :N] <- U[:, :N] * Q^T ... with Q rows = st */
    double *row = malloc(sizeof(double) * N);
    for (int mrow = 0; mrow < M; mrow++) {
        for (int j = 0; j < N; j++) {
            double acc = 0;
            for (int t = 0; t < N; t++) acc += U[(long)mrow * M + t] * c.st[(long)j * N + t];
            row[j] = acc;
        }
        memcpy(U + (long)mrow * M, row, sizeof(double) * N);
    }
    double *vt2 = malloc(sizeof(double) * nn);
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) {
            double acc = 0;
            for (int t = 0; t < N; t++) acc += c.gt[(long)i * N + t] * Vt[(long)t * N + j];
            vt2[(long)i * N + j] = acc;
        }
    memcpy(Vt, vt2, sizeof(double) * nn);
    if (stats) { stats[0] = c.merges; stats[1] = c.deflated; stats[2] = c.maxit; stats[3] = c.nonconv; }
    free(vt2); free(row); free(dd); free(ls); free(le);
    free(c.qt); free(c.wt); free(c.st); free(c.gt); free(c.f); free(c.l); free(c.idxq);
    return 0;
}

int oracle_svd(int M, int N, const float *A, double *sigma, double *U, double *Vt)
{
    if (M < N || N <= 0) return 1;
    double *a = malloc(sizeof(double) * (size_t)M * N);
    double *e = calloc(N, sizeof(double)), *tq = malloc(sizeof(double) * N), *tp = calloc(N, sizeof(double));
    for (size_t t = 0; t < (size_t)M * N; t++) a[t] = A[t];
    int rc = oracle_bidiag(M, N, a, U, Vt, sigma, e, tq, tp);
    if (!rc) rc = oracle_bdc(M, N, sigma, e, U, Vt, NULL);
    free(a); free(e); free(tq); free(tp);
    return rc;
}
