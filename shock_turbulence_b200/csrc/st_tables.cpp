// st_tables.cpp - constant LU factors and segmented-solve tables.
//
// The reference stores the left-hand sides as 135 full (lot,n) arrays
// (src/header:64-150, src/LES_header:1-63) and re-factorises them on every
// call (src/tridiagonal.f90:39, src/pentadiagonal.f90:42).  Every line of a
// direction has the same left-hand side (the Setup loops assign one value for
// all lines, src/derivCDopt6_sym_tri.f:41-63), so one factorisation per
// (direction, scheme, boundary kind) computed with the reference's own
// operation order gives the same pivots and multipliers.
//
// The segmented solve splits each line into P contiguous segments of S rows.
// Each segment runs the Thomas recurrences with a zero carry; the true carry
// into segment s is a linear combination of the end values of the segments
// before it (forward) or after it (backward), with the constant weights
// wf/wb (mf/mb for 2-vector carries), and it is added back through the
// per-row carry responses (g, h).  In exact arithmetic this is the Thomas
// algorithm.
#include <cfloat>
#include <cmath>
#include <algorithm>
#include <cstring>
#include "st_internal.h"

namespace st {

static const double kTiny = (double)FLT_MIN;   // tiny(1.0), src/tridiagonal.f90:275

int choose_seg(int n) {
    static const int sup[] = {2, 3, 4, 6, 8, 12, 16};
    for (int S : sup)
        if (n % S == 0 && n / S <= kMaxSeg) return S;
    return 0;
}

void fill_consts(Consts &k) {
    // FDL3DI sixth-order compact tridiagonal set, src/header:191-204
    k.a1 = 14.0 / 18.0; k.b1 = 1.0 / 36.0;
    k.a2 = 12.0 / 11.0; k.b2 = 3.0 / 44.0; k.c2 = 2.0 * (k.a2 + k.b2);
    k.closure1 = 5.0 / 9.0; k.closure2 = 1.0 / 18.0;              // src/header:173-175
    // Cook-Cabot eighth-order filter, src/LES_header:107-113
    k.fa0 = 9.9965e-01; k.fa1 = 0.66652; k.fa2 = 0.16674; k.fa3 = 4.0e-05; k.fa4 = -5.0e-06;
    const double ab = 0.45, af = 6.6624e-01, bf = 1.6688e-01;   // src/LES_header:118-146
    k.bc1[0] = 0.0;
    k.bc1[1] = 15.0 / 16.0; k.bc1[2] = 1.0 / 4.0; k.bc1[3] = -3.0 / 8.0;
    k.bc1[4] = 1.0 / 4.0; k.bc1[5] = -1.0 / 16.0;
    k.bc2[0] = (1.0 / 2.0 + ab);
    k.bc2[1] = (1.0 / 16.0 + (7.0 / 8.0) * ab);
    k.bc2[2] = (3.0 / 4.0 + (1.0 / 2.0) * ab);
    k.bc2[3] = (3.0 / 8.0 + (1.0 / 4.0) * ab);
    k.bc2[4] = (-1.0 / 4.0 + (1.0 / 2.0) * ab);
    k.bc2[5] = (1.0 / 16.0 - (1.0 / 8.0) * ab);
    k.bc3[0] = (5.0 / 8.0 + (3.0 / 4.0) * ab);
    k.bc3[1] = (1.0 / 2.0 + ab) / 2.0;
    k.bc3[2] = (-1.0 / 8.0 + ab / 4.0) / 2.0;
    k.bc4[0] = (11.0 / 16.0 + (5.0 / 8.0) * af - (5.0 / 8.0) * bf);
    k.bc4[1] = (15.0 / 32.0 + (17.0 / 16.0) * af + (15.0 / 16.0) * bf) / 2.0;
    k.bc4[2] = (-3.0 / 16.0 + (3.0 / 8.0) * af + (13.0 / 8.0) * bf) / 2.0;
    k.bc4[3] = (1.0 / 32.0 - af / 16.0 + bf / 16.0) / 2.0;
    // Gaussian filter: implicit REAL parameters, src/LES_header:153-157
    k.ga[0] = (double)(float)(3565.0 / 10368.0);
    k.ga[1] = (double)(float)(3091.0 / 12960.0);
    k.ga[2] = (double)(float)(1997.0 / 25920.0);
    k.ga[3] = (double)(float)(149.0 / 12960.0);
    k.ga[4] = (double)(float)(107.0 / 103680.0);
}

// ---- left-hand sides ------------------------------------------------------
// Setup_Derivatives_Sym/_Asym (src/derivCDopt6_sym_tri.f:41-372,
// src/derivCDopt6_asym_tri.f:41-374), one-rank case.
static void deriv_lhs(int n, int order, int asym, std::vector<double> &a, std::vector<double> &b,
                      std::vector<double> &c) {
    const double al1 = 1.0 / 3.0, al2 = 2.0 / 11.0;
    double al = order == 1 ? al1 : al2;
    a.assign(n, al); b.assign(n, 1.0); c.assign(n, al);
    if (order == 1) {
        a[0] = 0.0; b[0] = 1.0; c[0] = asym ? 2.0 * al1 : 0.0;
        a[n - 1] = 2.0; b[n - 1] = 1.0; c[n - 1] = 0.0;
        a[1] = al1; b[1] = 1.0; c[1] = al1;
        a[n - 2] = 1.0 / 2.0; b[n - 2] = 1.0; c[n - 2] = 1.0 / 6.0;
    } else {
        a[0] = 0.0; b[0] = 1.0; c[0] = asym ? 0.0 : 2.0 * al2;
        a[n - 1] = 1.1e1; b[n - 1] = 1.0; c[n - 1] = 0.0;
        a[1] = al2; b[1] = 1.0; c[1] = al2;
        a[n - 2] = -7.0 / 2.0e1; b[n - 2] = 1.0; c[n - 2] = 1.0e-1;
    }
}

// Init_Filters_sym/_asym (src/filters_sym.f:44-382, src/filters_asym.f:44-384)
static void filter_lhs(int n, int asym, std::vector<double> M[5]) {
    const double af = 6.6624e-01, bf = 1.6688e-01, ab = 0.45;
    M[0].assign(n, bf); M[1].assign(n, af); M[2].assign(n, 1.0); M[3].assign(n, af); M[4].assign(n, bf);
    auto row = [&](int r, double A, double B, double C, double D, double E) {
        M[0][r] = A; M[1][r] = B; M[2][r] = C; M[3][r] = D; M[4][r] = E;
    };
    if (asym) row(0, 0, 0, 1, 0, 0); else row(0, 0, 0, 1, 2.0 * af, 2.0 * bf);
    row(n - 1, 0, 0, 1, 0, 0);
    if (asym) row(1, 0, af, 1.0 - bf, af, bf); else row(1, 0, af, 1.0 + bf, af, bf);
    row(n - 2, 0, ab, 1, ab, 0);
    row(2, bf, af, 1, af, bf);
    row(n - 3, 0, ab, 1, ab, 0);
    row(3, bf, af, 1, af, bf);
    row(n - 4, bf, af, 1, af, bf);
}

// Periodic family: the cyclic systems of src/derivCDopt6_periodic.f (first and
// second derivative, solved with pentadiagonal(...,nper=1), i.e.
// pentadiagonal_periodic_serial, src/pentadiagonal.f90:381-504) and of
// src/filters_periodic.f:9-75 have constant rows (beta, alpha, 1, alpha, beta)
// that wrap around the line.  They are solved as the banded (non-wrapping)
// part, which the segmented solve handles like any other left-hand side, plus
// a rank-k correction for the corner entries (Sherman-Morrison-Woodbury):
//   A_cyc = A_band + U M V^T,  U = [e_j], V^T x = (x_j) for the k corner rows
//   j = {0, n-1} (k = 2) or {0, 1, n-2, n-1} (k = 4),
//   x = y - K (V^T y),  y = A_band^{-1} r,  K = Z (I + M V^T Z)^{-1} M,
//   Z = A_band^{-1} U.
// K is computed here in long double; the device adds -K (V^T y) after the
// banded solve.  Both systems are symmetric positive definite Toeplitz
// matrices (the filter's smallest eigenvalue is about 1.3e-3), so the banded
// elimination needs no pivoting.
static void band_rows(int n, double bt, double al, std::vector<double> M[5]) {
    M[0].assign(n, bt); M[1].assign(n, al); M[2].assign(n, 1.0); M[3].assign(n, al); M[4].assign(n, bt);
    M[0][0] = 0.0; M[0][1 % n] = 0.0; M[1][0] = 0.0;
    M[3][n - 1] = 0.0; M[4][n - 1] = 0.0; M[4][n - 2] = 0.0;
}

static std::vector<double> cyclic_correction(int n, double bt, double al, int k) {
    typedef long double R;
    const int w = 2;
    // banded LU (no pivoting) of the non-wrapping part, rows stored [i][j-i+w]
    std::vector<R> B((size_t)n * (2 * w + 1), 0.0L);
    auto at = [&](int i, int j) -> R & { return B[(size_t)i * (2 * w + 1) + (j - i + w)]; };
    const R co[5] = {bt, al, 1.0L, al, bt};
    for (int i = 0; i < n; i++)
        for (int j = i - w; j <= i + w; j++)
            if (j >= 0 && j < n) at(i, j) = co[j - i + w];
    for (int j = 0; j < n; j++)
        for (int i = j + 1; i <= j + w && i < n; i++) {
            R l = at(i, j) / at(j, j);
            at(i, j) = l;
            for (int q = j + 1; q <= j + w && q < n; q++) at(i, q) -= l * at(j, q);
        }
    auto solve = [&](std::vector<R> &x) {
        for (int i = 0; i < n; i++)
            for (int j = std::max(0, i - w); j < i; j++) x[i] -= at(i, j) * x[j];
        for (int i = n - 1; i >= 0; i--) {
            for (int j = i + 1; j <= i + w && j < n; j++) x[i] -= at(i, j) * x[j];
            x[i] /= at(i, i);
        }
    };
    int idx[4];
    R Mm[4][4] = {{0}};
    if (k == 2) {
        idx[0] = 0; idx[1] = n - 1;
        Mm[0][1] = al; Mm[1][0] = al;                    // row 0: al*x_{n-1}; row n-1: al*x_0
    } else {
        idx[0] = 0; idx[1] = 1; idx[2] = n - 2; idx[3] = n - 1;
        Mm[0][2] = bt; Mm[0][3] = al;                    // row 0:   bt*x_{n-2} + al*x_{n-1}
        Mm[1][3] = bt;                                   // row 1:   bt*x_{n-1}
        Mm[2][0] = bt;                                   // row n-2: bt*x_0
        Mm[3][0] = al; Mm[3][1] = bt;                    // row n-1: al*x_0 + bt*x_1
    }
    std::vector<std::vector<R>> Z(k, std::vector<R>(n, 0.0L));
    for (int q = 0; q < k; q++) { Z[q][idx[q]] = 1.0L; solve(Z[q]); }
    // S = I + M V^T Z  (k x k), then its inverse by Gauss-Jordan with pivoting
    R S[4][8] = {{0}};
    for (int a = 0; a < k; a++)
        for (int b = 0; b < k; b++) {
            R v = a == b ? 1.0L : 0.0L;
            for (int q = 0; q < k; q++) v += Mm[a][q] * Z[b][idx[q]];
            S[a][b] = v;
            S[a][k + b] = a == b ? 1.0L : 0.0L;
        }
    for (int col = 0; col < k; col++) {
        int piv = col;
        for (int r = col + 1; r < k; r++) if (fabsl(S[r][col]) > fabsl(S[piv][col])) piv = r;
        for (int q = 0; q < 2 * k; q++) std::swap(S[col][q], S[piv][q]);
        R d = S[col][col];
        for (int q = 0; q < 2 * k; q++) S[col][q] /= d;
        for (int r = 0; r < k; r++)
            if (r != col) {
                R f = S[r][col];
                for (int q = 0; q < 2 * k; q++) S[r][q] -= f * S[col][q];
            }
    }
    // K = Z Sinv M ;  stored negated, row-major [n][k]
    R SM[4][4];
    for (int a = 0; a < k; a++)
        for (int b = 0; b < k; b++) {
            R v = 0.0L;
            for (int q = 0; q < k; q++) v += S[a][k + q] * Mm[q][b];
            SM[a][b] = v;
        }
    std::vector<double> K((size_t)n * k);
    for (int i = 0; i < n; i++)
        for (int b = 0; b < k; b++) {
            R v = 0.0L;
            for (int a = 0; a < k; a++) v += Z[a][i] * SM[a][b];
            K[(size_t)i * k + b] = (double)(-v);
        }
    return K;
}

// ---- tables ---------------------------------------------------------------
struct TriHost {
    std::vector<double> l, g, up, id, h, wf, wb, sf, sb;
    int kf = 0, kb = 0;
    int slo = 0, shi = 0;
};
struct PenHost {
    std::vector<double> p1, p2, g1, g2, q1, q2, id, h1, h2, sf, sb;
    int slo = 0, shi = 0;
};

// The contiguous range [slo, shi) of segments around the middle one in which
// every listed coefficient array holds, on every row, exactly (bitwise) its
// value at the middle row; empty when the middle segment itself varies (the
// antisymmetric filter's factorisation ends in a cycle, not a fixed point).
static void flat_segments(const std::vector<const std::vector<double> *> &arrs, int n, int S, int *slo,
                          int *shi) {
    const int P = n / S, mid = n / 2;
    auto flat = [&](int s) {
        for (const auto *v : arrs)
            for (int i = s * S; i < s * S + S; i++)
                if ((*v)[i] != (*v)[mid]) return false;
        return true;
    };
    int sm = mid / S;
    *slo = *shi = 0;
    if (!flat(sm)) return;
    int lo = sm, hi = sm + 1;
    while (lo > 0 && flat(lo - 1)) lo--;
    while (hi < P && flat(hi)) hi++;
    *slo = lo; *shi = hi;
}

// Carry weights decay geometrically with the distance between segments.
// Contributions with weight below 1e-20 cannot change an FP64 result of the
// size of the solution, so the device loops stop at the farthest segment
// whose weight (max norm of the 2x2 block for pentadiagonal carries) is at
// least that large.
static int carry_span(const std::vector<double> &w, int P, int blk, bool fwd, double floor = 1e-20) {
    int span = 0;
    for (int s = 0; s < P; s++)
        for (int sp = 0; sp < P; sp++) {
            int dist = fwd ? s - sp : sp - s;
            if (dist <= 0) continue;
            double m = 0.0;
            for (int q = 0; q < blk; q++) m = std::fmax(m, std::fabs(w[((size_t)sp * P + s) * blk + q]));
            if (m >= floor && dist > span) span = dist;
        }
    return span;
}

static TriHost tri_tables(const std::vector<double> &a, const std::vector<double> &b,
                          const std::vector<double> &c, int n, int S) {
    TriHost t;
    std::vector<double> bp(n);
    t.l.assign(n, 0.0);
    bp[0] = b[0];
    for (int i = 1; i < n; i++) {
        t.l[i] = a[i] / (bp[i - 1] + kTiny);
        bp[i] = b[i] - c[i - 1] * t.l[i];
    }
    t.up = c;
    t.id.resize(n);
    for (int i = 0; i < n - 1; i++) t.id[i] = 1.0 / (bp[i] + kTiny);
    t.id[n - 1] = 1.0 / bp[n - 1];
    const int P = n / S;
    t.g.assign(n, 0.0); t.h.assign(n, 0.0);
    std::vector<double> B(P), G(P);
    for (int s = 0; s < P; s++) {
        int a0 = s * S;
        double pr = 1.0;
        for (int q = 0; q < S; q++) { pr *= -t.l[a0 + q]; t.g[a0 + q] = pr; }
        B[s] = t.g[a0 + S - 1];
        pr = 1.0;
        for (int q = S - 1; q >= 0; q--) { pr *= -(t.up[a0 + q] * t.id[a0 + q]); t.h[a0 + q] = pr; }
        G[s] = t.h[a0];
    }
    // carry weights: C_s = sum_{s'<s} (prod_{u=s'+1}^{s-1} B_u) A_{s'}
    t.wf.assign((size_t)P * P, 0.0); t.wb.assign((size_t)P * P, 0.0);
    for (int s = 0; s < P; s++) {
        double w = 1.0;
        for (int sp = s - 1; sp >= 0; sp--) { t.wf[(size_t)sp * P + s] = w; w *= B[sp]; }
        w = 1.0;
        for (int sp = s + 1; sp < P; sp++) { t.wb[(size_t)sp * P + s] = w; w *= G[sp]; }
    }
    t.kf = carry_span(t.wf, P, 1, true);
    t.kb = carry_span(t.wb, P, 1, false);
    flat_segments({&t.l, &t.up, &t.id}, n, S, &t.slo, &t.shi);
    // scan factors: products of 2^k consecutive B ending at s and G starting
    // at s; entries whose span leaves [0, P) stay 0 (never read)
    t.sf.assign((size_t)kScanSteps * kMaxSeg, 0.0);
    t.sb.assign((size_t)kScanSteps * kMaxSeg, 0.0);
    for (int s = 0; s < P; s++) { t.sf[s] = B[s]; t.sb[s] = G[s]; }
    for (int k = 1, d = 1; k < kScanSteps; k++, d <<= 1)
        for (int s = 0; s < P; s++) {
            if (s - d >= 0) t.sf[k * kMaxSeg + s] = t.sf[(k - 1) * kMaxSeg + s] * t.sf[(k - 1) * kMaxSeg + s - d];
            if (s + d < P) t.sb[k * kMaxSeg + s] = t.sb[(k - 1) * kMaxSeg + s] * t.sb[(k - 1) * kMaxSeg + s + d];
        }
    return t;
}

static void mat2mul(const double *A, const double *B, double *C) {  // C = A*B (row-major 2x2)
    double r[4] = {A[0] * B[0] + A[1] * B[2], A[0] * B[1] + A[1] * B[3],
                   A[2] * B[0] + A[3] * B[2], A[2] * B[1] + A[3] * B[3]};
    std::memcpy(C, r, sizeof(r));
}

static PenHost pen_tables(std::vector<double> M[5], int n, int S) {
    PenHost t;
    std::vector<double> A = M[0], B = M[1], C = M[2], D = M[3], E = M[4];
    std::vector<double> k1(n, 0.0), k2(n, 0.0);
    for (int i = 0; i <= n - 3; i++) {
        k1[i] = B[i + 1] / (C[i] + kTiny);
        C[i + 1] = C[i + 1] - D[i] * k1[i];
        D[i + 1] = D[i + 1] - E[i] * k1[i];
        k2[i] = A[i + 2] / (C[i] + kTiny);
        B[i + 2] = B[i + 2] - D[i] * k2[i];
        C[i + 2] = C[i + 2] - E[i] * k2[i];
    }
    double k3 = B[n - 1] / (C[n - 2] + kTiny);
    C[n - 1] = C[n - 1] - D[n - 2] * k3;
    t.p1.assign(n, 0.0); t.p2.assign(n, 0.0);
    t.p1[1] = k1[0];
    for (int i = 2; i <= n - 2; i++) { t.p1[i] = k1[i - 1]; t.p2[i] = k2[i - 2]; }
    t.p1[n - 1] = k3; t.p2[n - 1] = k2[n - 3];
    t.q1.assign(n, 0.0); t.q2.assign(n, 0.0); t.id.resize(n);
    for (int i = 0; i <= n - 2; i++) t.q1[i] = D[i];
    for (int i = 0; i <= n - 3; i++) t.q2[i] = E[i];
    for (int i = 0; i < n; i++) t.id[i] = 1.0 / (C[i] + kTiny);
    const int P = n / S;
    t.g1.assign(n, 0.0); t.g2.assign(n, 0.0); t.h1.assign(n, 0.0); t.h2.assign(n, 0.0);
    std::vector<double> Mseg(P * 4), Nseg(P * 4);
    for (int s = 0; s < P; s++) {
        int a0 = s * S;
        for (int which = 0; which < 2; which++) {
            // forward homogeneous response to (r'_{a-1}, r'_{a-2}) = e_which
            double hm1 = which == 0 ? 1.0 : 0.0, hm2 = which == 0 ? 0.0 : 1.0;
            for (int q = 0; q < S; q++) {
                int i = a0 + q;
                double v = (0.0 - t.p2[i] * hm2) - t.p1[i] * hm1;
                (which == 0 ? t.g1 : t.g2)[i] = v;
                hm2 = hm1; hm1 = v;
            }
            // backward homogeneous response to (x_{b+1}, x_{b+2}) = e_which
            double kp1 = which == 0 ? 1.0 : 0.0, kp2 = which == 0 ? 0.0 : 1.0;
            for (int q = S - 1; q >= 0; q--) {
                int i = a0 + q;
                double v = ((0.0 - t.q1[i] * kp1) - t.q2[i] * kp2) * t.id[i];
                (which == 0 ? t.h1 : t.h2)[i] = v;
                kp2 = kp1; kp1 = v;
            }
        }
        double *m = &Mseg[s * 4], *nn = &Nseg[s * 4];
        int e = a0 + S - 1;
        if (S >= 2) {
            m[0] = t.g1[e]; m[1] = t.g2[e]; m[2] = t.g1[e - 1]; m[3] = t.g2[e - 1];
            nn[0] = t.h1[a0]; nn[1] = t.h2[a0]; nn[2] = t.h1[a0 + 1]; nn[3] = t.h2[a0 + 1];
        } else {
            m[0] = t.g1[e]; m[1] = t.g2[e]; m[2] = 1.0; m[3] = 0.0;
            nn[0] = t.h1[a0]; nn[1] = t.h2[a0]; nn[2] = 1.0; nn[3] = 0.0;
        }
    }
    flat_segments({&t.p1, &t.p2, &t.q1, &t.q2, &t.id}, n, S, &t.slo, &t.shi);
    // scan factors: T_0(s) = M_s, T_{k+1}(s) = T_k(s) T_k(s-2^k);
    // U_0(s) = N_s, U_{k+1}(s) = U_k(s) U_k(s+2^k); entries whose span leaves
    // [0, P) stay 0 (never read)
    t.sf.assign((size_t)kScanSteps * kMaxSeg * 4, 0.0);
    t.sb.assign((size_t)kScanSteps * kMaxSeg * 4, 0.0);
    for (int s = 0; s < P; s++) {
        std::memcpy(&t.sf[(size_t)s * 4], &Mseg[s * 4], 32);
        std::memcpy(&t.sb[(size_t)s * 4], &Nseg[s * 4], 32);
    }
    for (int k = 1, d = 1; k < kScanSteps; k++, d <<= 1)
        for (int s = 0; s < P; s++) {
            if (s - d >= 0)
                mat2mul(&t.sf[((size_t)(k - 1) * kMaxSeg + s) * 4], &t.sf[((size_t)(k - 1) * kMaxSeg + s - d) * 4],
                        &t.sf[((size_t)k * kMaxSeg + s) * 4]);
            if (s + d < P)
                mat2mul(&t.sb[((size_t)(k - 1) * kMaxSeg + s) * 4], &t.sb[((size_t)(k - 1) * kMaxSeg + s + d) * 4],
                        &t.sb[((size_t)k * kMaxSeg + s) * 4]);
        }
    return t;
}

static const double *upload(st_ctx *c, const std::vector<double> &v, int *err) {
    void *p = nullptr;
    if (cudaMalloc(&p, v.size() * sizeof(double)) != cudaSuccess) { *err = 1; return nullptr; }
    c->table_allocs.push_back(p);
    c->table_bytes += v.size() * sizeof(double);
    if (cudaMemcpy(p, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
        *err = 1;
    return (const double *)p;
}
static const float *upload_f(st_ctx *c, const std::vector<double> &v, int *err) {
    std::vector<float> f(v.begin(), v.end());
    void *p = nullptr;
    if (cudaMalloc(&p, f.size() * sizeof(float)) != cudaSuccess) { *err = 1; return nullptr; }
    c->table_allocs.push_back(p);
    c->table_bytes += f.size() * sizeof(float);
    if (cudaMemcpy(p, f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) *err = 1;
    return (const float *)p;
}

// The FP32 mode's tridiagonal factors: the double tables rounded to float.
// Carry weights below 1e-12 cannot change a float result of the size of the
// solution (float epsilon 6e-8 times the few segment end values they scale).
static void upload_tri(st_ctx *c, st::TriTab &t, st::TriTabT<float> &tf, const TriHost &h,
                       const std::vector<double> *K, int P, int *err) {
    t.l = upload(c, h.l, err); t.g = upload(c, h.g, err); t.up = upload(c, h.up, err);
    t.id = upload(c, h.id, err); t.h = upload(c, h.h, err);
    t.wf = upload(c, h.wf, err); t.wb = upload(c, h.wb, err);
    t.sf = upload(c, h.sf, err); t.sb = upload(c, h.sb, err);
    t.kf = h.kf; t.kb = h.kb;
    t.cyc = K ? upload(c, *K, err) : nullptr;
    const int mid = (int)h.l.size() / 2;
    t.slo = h.slo; t.shi = h.shi;
    t.cl = h.l[mid]; t.cup = h.up[mid]; t.cid = h.id[mid];
    tf = st::TriTabT<float>{};
    tf.slo = h.slo; tf.shi = h.shi;
    tf.cl = (float)t.cl; tf.cup = (float)t.cup; tf.cid = (float)t.cid;
    if (c->p.precision != ST_PRECISION_FP32) return;
    tf.l = upload_f(c, h.l, err); tf.g = upload_f(c, h.g, err); tf.up = upload_f(c, h.up, err);
    tf.id = upload_f(c, h.id, err); tf.h = upload_f(c, h.h, err);
    tf.wf = upload_f(c, h.wf, err); tf.wb = upload_f(c, h.wb, err);
    tf.sf = upload_f(c, h.sf, err); tf.sb = upload_f(c, h.sb, err);
    tf.kf = carry_span(h.wf, P, 1, true, 1e-12);
    tf.kb = carry_span(h.wb, P, 1, false, 1e-12);
    tf.cyc = K ? upload_f(c, *K, err) : nullptr;
}

// Periodic family: every derivative and filter kind of a direction gets the
// cyclic tables (the periodic routines have no sym/asym variants).  The FDL3DI
// constants are used as the tridiagonal scheme they define (beta = 0), see
// the oracle's note on the periodic constant set.
static int build_tables_periodic(st_ctx *c) {
    int err = 0;
    const double al1 = 1.0 / 3.0, al2 = 2.0 / 11.0, af = 6.6624e-01, bf = 1.6688e-01;
    for (int d = 0; d < 3; d++) {
        int n = c->dm.n[d];
        for (int order = 1; order <= 2; order++) {
            std::vector<double> M[5];
            double al = order == 1 ? al1 : al2;
            band_rows(n, 0.0, al, M);
            TriHost h = tri_tables(M[1], M[2], M[3], n, c->seg[d]);
            std::vector<double> K = cyclic_correction(n, 0.0, al, 2);
            for (int asym = 0; asym < 2; asym++) {
                const int kind = (order - 1) * 2 + asym;
                upload_tri(c, c->tri[d][kind], c->trif[d][kind], h, &K, n / c->seg[d], &err);
            }
        }
        std::vector<double> M[5];
        band_rows(n, bf, af, M);
        PenHost h = pen_tables(M, n, c->seg[d]);
        std::vector<double> K = cyclic_correction(n, bf, af, 4);
        for (int kind = 0; kind < 2; kind++) {
            PenTab &t = c->pen[d][kind];
            t.p1 = upload(c, h.p1, &err); t.p2 = upload(c, h.p2, &err);
            t.g1 = upload(c, h.g1, &err); t.g2 = upload(c, h.g2, &err);
            t.q1 = upload(c, h.q1, &err); t.q2 = upload(c, h.q2, &err);
            t.id = upload(c, h.id, &err); t.h1 = upload(c, h.h1, &err); t.h2 = upload(c, h.h2, &err);
            t.sf = upload(c, h.sf, &err); t.sb = upload(c, h.sb, &err);
            {
                const int mid = n / 2;
                t.slo = h.slo; t.shi = h.shi;
                t.cp1 = h.p1[mid]; t.cp2 = h.p2[mid]; t.cq1 = h.q1[mid]; t.cq2 = h.q2[mid]; t.cid = h.id[mid];
            }
            t.cyc = upload(c, K, &err);
        }
    }
    if (err) return fail(c, ST_E_NOMEM, "could not allocate or upload the LU tables");
    return ST_OK;
}

int build_tables(st_ctx *c) {
    if (c->p.family == ST_FAMILY_PERIODIC) return build_tables_periodic(c);
    int err = 0;
    for (int d = 0; d < 3; d++) {
        int n = c->dm.n[d];
        for (int kind = 0; kind < 4; kind++) {
            std::vector<double> a, b, cc;
            deriv_lhs(n, kind < 2 ? 1 : 2, kind & 1, a, b, cc);
            TriHost h = tri_tables(a, b, cc, n, c->seg[d]);
            upload_tri(c, c->tri[d][kind], c->trif[d][kind], h, nullptr, n / c->seg[d], &err);
        }
        for (int kind = 0; kind < 2; kind++) {
            std::vector<double> M[5];
            filter_lhs(n, kind, M);
            PenHost h = pen_tables(M, n, c->seg[d]);
            PenTab &t = c->pen[d][kind];
            t.p1 = upload(c, h.p1, &err); t.p2 = upload(c, h.p2, &err);
            t.g1 = upload(c, h.g1, &err); t.g2 = upload(c, h.g2, &err);
            t.q1 = upload(c, h.q1, &err); t.q2 = upload(c, h.q2, &err);
            t.id = upload(c, h.id, &err); t.h1 = upload(c, h.h1, &err); t.h2 = upload(c, h.h2, &err);
            t.sf = upload(c, h.sf, &err); t.sb = upload(c, h.sb, &err);
            {
                const int mid = n / 2;
                t.slo = h.slo; t.shi = h.shi;
                t.cp1 = h.p1[mid]; t.cp2 = h.p2[mid]; t.cq1 = h.q1[mid]; t.cq2 = h.q2[mid]; t.cid = h.id[mid];
            }
            t.cyc = nullptr;
        }
    }
    if (err) return fail(c, ST_E_NOMEM, "could not allocate or upload the LU tables");
    return ST_OK;
}

void free_tables(st_ctx *c) {
    for (void *p : c->table_allocs) cudaFree(p);
    c->table_allocs.clear();
}

}  // namespace st
