// FP64 device math shared by every kernel of the search: the d0 schedule,
// the Horn-quaternion Kabsch solve, rigid transforms and TM terms.  The
// eigen-solve finds the dominant eigenvector from the characteristic
// polynomial (see qcp_rotation), which returns the reference Jacobi's
// rotation to rounding whenever the top eigenvalue is separated, and runs
// the reference's own Jacobi sequence (indialign_c/core.h:29-90) when it is
// not; covariances are formed from raw
// moments accumulated in one pass (sum p, sum q, sum p q^T, count) instead of
// the reference's centroid pass + centred pass (core.h:94-123), which is the
// same matrix up to FP64 rounding and lets a selection pass and its Kabsch
// fuse into a single sweep over the residues.
#pragma once
#include <stdint.h>

#define IA_DEV __device__ __forceinline__

namespace ia {

__constant__ static const double kD0Mults[6] = {2.0, 1.5, 1.0, 0.75, 0.5, 0.25};

// d0, d0_search and score_d8 from the normalisation length
// (indialign_c/core.h:12-25).
IA_DEV void d0_from_length(double L, double &d0, double &d0s, double &sd8) {
    double Lc = L > 1.0 ? L : 1.0;
    if (Lc <= 11.0) d0 = 0.3;
    else if (Lc <= 15.0) d0 = 0.4;
    else if (Lc <= 19.0) d0 = 0.5;
    else if (Lc <= 23.0) d0 = 0.6;
    else d0 = 0.7;
    if (Lc >= 30.0) d0 = 0.6 * sqrt(Lc - 0.5) - 2.5;
    if (d0 < 0.3) d0 = 0.3;
    double m = Lc - 15.0 > 0.0 ? Lc - 15.0 : 0.0;
    double v = 1.24 * cbrt(m) - 1.8;
    d0s = v < 4.5 ? 4.5 : (v > 8.0 ? 8.0 : v);
    sd8 = 1.5 * pow(Lc, 0.3) + 3.5;
}

// Cutoff list: d0s x {2,1.5,1,.75,.5,.25}, then d0+{1..5} unless within 0.01
// of an earlier entry (indialign_c/indialign.cpp:54-67).  Returns C <= 11.
IA_DEV int d0_candidates(double d0, double d0s, double *cand) {
    int C = 0;
    for (int c = 0; c < 6; c++) cand[C++] = d0s * kD0Mults[c];
    for (int c = 1; c <= 5; c++) {
        double v = d0 + (double)c;
        bool dup = false;
        for (int e = 0; e < C; e++) dup |= fabs(cand[e] - v) < 0.01;
        if (!dup) cand[C++] = v;
    }
    return C;
}

struct Rt {
    double R[9], t[3];
};

IA_DEV void set_identity(double *R, double *t) {
#pragma unroll
    for (int i = 0; i < 9; i++) R[i] = (i % 4 == 0) ? 1.0 : 0.0;
    t[0] = t[1] = t[2] = 0.0;
}

// aligned_d = sum_k p_k R[3k+d] + t_d (indialign_c/core.h:127-132)
IA_DEV void xform(const double *R, const double *t, double px, double py,
                  double pz, double &mx, double &my, double &mz) {
    mx = px * R[0] + py * R[3] + pz * R[6] + t[0];
    my = px * R[1] + py * R[4] + pz * R[7] + t[1];
    mz = px * R[2] + py * R[5] + pz * R[8] + t[2];
}

IA_DEV double dist2(const double *R, const double *t, double px, double py,
                    double pz, double qx, double qy, double qz) {
    double mx, my, mz;
    xform(R, t, px, py, pz, mx, my, mz);
    double dx = mx - qx, dy = my - qy, dz = mz - qz;
    return dx * dx + dy * dy + dz * dz;
}

// One Jacobi rotation of the pair (p,q), skipped when |A[p][q]| < 1e-15
// (indialign_c/core.h:39-58).  Indices are compile-time so A and V stay in
// registers.
template <int p, int q>
IA_DEV void jacobi_rot(double (&A)[4][4], double (&V)[4][4]) {
    double apq = A[p][q];
    if (fabs(apq) < 1e-15) return;
    double tau = (A[q][q] - A[p][p]) / (2.0 * apq);
    double t = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
    double c = 1.0 / sqrt(1.0 + t * t), s = t * c;
    A[p][p] -= t * apq;
    A[q][q] += t * apq;
    A[p][q] = A[q][p] = 0.0;
#pragma unroll
    for (int r = 0; r < 4; r++) {
        if (r == p || r == q) continue;
        double rp = A[r][p], rq = A[r][q];
        A[r][p] = A[p][r] = c * rp - s * rq;
        A[r][q] = A[q][r] = s * rp + c * rq;
    }
#pragma unroll
    for (int r = 0; r < 4; r++) {
        double vp = V[r][p], vq = V[r][q];
        V[r][p] = c * vp - s * vq;
        V[r][q] = s * vp + c * vq;
    }
}

// Reciprocal by Newton-Raphson (y <- y + y(1 - xy), quadratic convergence)
// from the hardware's fast double approximation (rcp.approx.f64, about 20
// correct bits): two steps take the seed error below double rounding, so the
// result is within 1 ulp of 1/x (checked on the device against 1/x by the
// test suite).  Valid for normal |x| well inside the double range.
IA_DEV double rcp_nr(double x) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    double e = fma(-x, y, 1.0);
    y = fma(y, e, y);
    e = fma(-x, y, 1.0);
    return fma(y, e, y);
}

IA_DEV void horn_matrix(const double (&H)[3][3], double (&A)[4][4]) {
    A[0][0] = H[0][0] + H[1][1] + H[2][2];
    A[0][1] = A[1][0] = H[1][2] - H[2][1];
    A[0][2] = A[2][0] = H[2][0] - H[0][2];
    A[0][3] = A[3][0] = H[0][1] - H[1][0];
    A[1][1] = H[0][0] - H[1][1] - H[2][2];
    A[1][2] = A[2][1] = H[0][1] + H[1][0];
    A[1][3] = A[3][1] = H[2][0] + H[0][2];
    A[2][2] = -H[0][0] + H[1][1] - H[2][2];
    A[2][3] = A[3][2] = H[1][2] + H[2][1];
    A[3][3] = -H[0][0] - H[1][1] + H[2][2];
}

IA_DEV void set_eye4(double (&V)[4][4]) {
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) V[i][j] = (i == j) ? 1.0 : 0.0;
}

// Dominant eigenvector (first index among equal diagonal maxima) -> unit
// quaternion -> rotation (indialign_c/core.h:76-89).
IA_DEV void quat_to_rotation(const double (&A)[4][4], const double (&V)[4][4], double *R) {
    int best = 0;
    double bv = A[0][0];
    if (A[1][1] > bv) { best = 1; bv = A[1][1]; }
    if (A[2][2] > bv) { best = 2; bv = A[2][2]; }
    if (A[3][3] > bv) { best = 3; bv = A[3][3]; }
    double q0, q1, q2, q3;
    q0 = best == 0 ? V[0][0] : best == 1 ? V[0][1] : best == 2 ? V[0][2] : V[0][3];
    q1 = best == 0 ? V[1][0] : best == 1 ? V[1][1] : best == 2 ? V[1][2] : V[1][3];
    q2 = best == 0 ? V[2][0] : best == 1 ? V[2][1] : best == 2 ? V[2][2] : V[2][3];
    q3 = best == 0 ? V[3][0] : best == 1 ? V[3][1] : best == 2 ? V[3][2] : V[3][3];
    double qn = sqrt(q0 * q0 + q1 * q1 + q2 * q2 + q3 * q3);
    if (qn < 1e-12) {
        q0 = 1; q1 = q2 = q3 = 0;
    } else {
        q0 /= qn; q1 /= qn; q2 /= qn; q3 /= qn;
    }
    R[0] = q0 * q0 + q1 * q1 - q2 * q2 - q3 * q3;
    R[1] = 2 * (q1 * q2 + q0 * q3);
    R[2] = 2 * (q1 * q3 - q0 * q2);
    R[3] = 2 * (q1 * q2 - q0 * q3);
    R[4] = q0 * q0 - q1 * q1 + q2 * q2 - q3 * q3;
    R[5] = 2 * (q2 * q3 + q0 * q1);
    R[6] = 2 * (q1 * q3 + q0 * q2);
    R[7] = 2 * (q2 * q3 - q0 * q1);
    R[8] = q0 * q0 - q1 * q1 - q2 * q2 + q3 * q3;
}

// The reference eigen-solve exactly: 8 cyclic sweeps in its pair order with
// correctly rounded divides and square roots (indialign_c/core.h:29-60).
IA_DEV void jacobi_reference(double (&A)[4][4], double (&V)[4][4]) {
    set_eye4(V);
#pragma unroll 1
    for (int sweep = 0; sweep < 8; sweep++) {
        jacobi_rot<0, 1>(A, V);
        jacobi_rot<0, 2>(A, V);
        jacobi_rot<0, 3>(A, V);
        jacobi_rot<1, 2>(A, V);
        jacobi_rot<1, 3>(A, V);
        jacobi_rot<2, 3>(A, V);
    }
}

IA_DEV double det3(double a, double b, double c, double d, double e, double f, double g, double h, double i) {
    return a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
}

// Determinant of A without row `row` and column `col`.
template <int row, int col>
IA_DEV double minor3(const double (&A)[4][4]) {
    constexpr int r0 = row == 0 ? 1 : 0, r1 = row <= 1 ? 2 : 1, r2 = row <= 2 ? 3 : 2;
    constexpr int c0 = col == 0 ? 1 : 0, c1 = col <= 1 ? 2 : 1, c2 = col <= 2 ? 3 : 2;
    return det3(A[r0][c0], A[r0][c1], A[r0][c2], A[r1][c0], A[r1][c1], A[r1][c2], A[r2][c0], A[r2][c1],
                A[r2][c2]);
}

// Column c of adj(A): adj[r][c] = (-1)^(r+c) * minor(c, r).
template <int c>
IA_DEV void adj_column(const double (&A)[4][4], double (&v)[4]) {
    v[0] = ((0 + c) & 1 ? -1.0 : 1.0) * minor3<c, 0>(A);
    v[1] = ((1 + c) & 1 ? -1.0 : 1.0) * minor3<c, 1>(A);
    v[2] = ((2 + c) & 1 ? -1.0 : 1.0) * minor3<c, 2>(A);
    v[3] = ((3 + c) & 1 ? -1.0 : 1.0) * minor3<c, 3>(A);
}

// Dominant eigenvector of Horn's key matrix F by its characteristic
// polynomial -- the QCP method (Theobald 2005, "Rapid calculation of RMSDs
// using a quaternion-based characteristic polynomial").  F is traceless, so
// P(x) = x^4 + c2 x^2 + c1 x + c0 with c2 = -tr(F^2)/2, c1 = -tr(F^3)/3,
// c0 = det F.  The largest root l1 comes from Newton's method started at
// sqrt(tr(F^2)) >= l1, where P is increasing and convex, so the iterates
// fall monotonically onto l1.  P'(l1) is the product of the gaps to the
// other eigenvalues, each at most 2 sqrt(tr(F^2)); when it cannot prove
// l1 - l2 >= 1e-4 sqrt(tr(F^2)), l2 is found the same way on P(x)/(x - l1).
// A top pair closer than that returns false: the eigenvector inside a
// (near-)degenerate pair depends on the solver, and the caller reruns the
// reference's Jacobi sequence.  Otherwise the eigenvector is the adjugate
// column of F - l1 I with the largest diagonal entry.  A CPU build of the
// oracle with this eigen-solve matched the reference build's final scores to
// 3e-16 on 560 pairs, Jacobi rerunning in ~6e-5 of the solves.
IA_DEV bool qcp_rotation(const double (&F)[4][4], double *R) {
    double p2 = 0.0, p3 = 0.0;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int k = 0; k < 4; k++) {
            double f2 = 0.0;
#pragma unroll
            for (int j = 0; j < 4; j++) f2 = fma(F[i][j], F[j][k], f2);
            p3 = fma(f2, F[k][i], p3);
            p2 = fma(F[i][k], F[i][k], p2);
        }
    const double s0 = F[0][0] * F[1][1] - F[1][0] * F[0][1], s1 = F[0][0] * F[1][2] - F[1][0] * F[0][2];
    const double s2 = F[0][0] * F[1][3] - F[1][0] * F[0][3], s3 = F[0][1] * F[1][2] - F[1][1] * F[0][2];
    const double s4 = F[0][1] * F[1][3] - F[1][1] * F[0][3], s5 = F[0][2] * F[1][3] - F[1][2] * F[0][3];
    const double k5 = F[2][2] * F[3][3] - F[3][2] * F[2][3], k4 = F[2][1] * F[3][3] - F[3][1] * F[2][3];
    const double k3 = F[2][1] * F[3][2] - F[3][1] * F[2][2], k2 = F[2][0] * F[3][3] - F[3][0] * F[2][3];
    const double k1 = F[2][0] * F[3][2] - F[3][0] * F[2][2], k0 = F[2][0] * F[3][1] - F[3][0] * F[2][1];
    const double c0 = s0 * k5 - s1 * k4 + s2 * k3 + s3 * k2 - s4 * k1 + s5 * k0;
    const double c2 = -0.5 * p2, c1 = -p3 * (1.0 / 3.0);
    if (!(p2 > 0.0)) return false;
    const double scale = sqrt(p2);
    double l1 = scale, dp = 0.0;
#pragma unroll 1
    for (int it = 0; it < 64; it++) {
        const double x2 = l1 * l1;
        const double g = fma(fma(x2 + c2, l1, c1), l1, c0);
        dp = fma(fma(4.0 * x2, 1.0, 2.0 * c2), l1, c1);
        if (!(dp > 0.0)) break;
        const double nx = l1 - g * rcp_nr(dp);
        if (!(nx < l1)) break;
        const bool done = l1 - nx <= 1e-16 * scale;
        l1 = nx;
        if (done) break;
    }
    dp = fma(fma(4.0 * l1 * l1, 1.0, 2.0 * c2), l1, c1);  // P'(l1)
    if (!(dp >= 4e-4 * p2 * scale)) {
        // second eigenvalue: largest root of x^3 + l1 x^2 + (c2 + l1^2) x + (c1 + l1 c2 + l1^3)
        const double b2 = l1, b1 = fma(l1, l1, c2), b0 = fma(l1, b1, c1);
        double x = l1;
#pragma unroll 1
        for (int it = 0; it < 128; it++) {
            const double g = fma(fma(x + b2, x, b1), x, b0);
            const double dg = fma(fma(3.0, x, 2.0 * b2), x, b1);
            if (!(dg > 0.0)) break;
            const double nx = x - g * rcp_nr(dg);
            if (!(nx < x)) break;
            const bool done = x - nx <= 1e-16 * scale;
            x = nx;
            if (done) break;
        }
        if (!(l1 - x >= 1e-4 * scale)) return false;
    }
    double A[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) A[i][j] = i == j ? F[i][j] - l1 : F[i][j];
    // adj(A) = P'(l1) q q^T: its largest diagonal entry marks the best column
    const double a0 = fabs(minor3<0, 0>(A)), a1 = fabs(minor3<1, 1>(A)), a2 = fabs(minor3<2, 2>(A)),
                 a3 = fabs(minor3<3, 3>(A));
    double v[4];
    if (a0 >= a1 && a0 >= a2 && a0 >= a3) adj_column<0>(A, v);
    else if (a1 >= a2 && a1 >= a3) adj_column<1>(A, v);
    else if (a2 >= a3) adj_column<2>(A, v);
    else adj_column<3>(A, v);
    const double n2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2] + v[3] * v[3];
    if (!(n2 > 0.0)) return false;
    const double inv = 1.0 / sqrt(n2);
    const double q0 = v[0] * inv, q1 = v[1] * inv, q2 = v[2] * inv, q3 = v[3] * inv;
    R[0] = q0 * q0 + q1 * q1 - q2 * q2 - q3 * q3;
    R[1] = 2 * (q1 * q2 + q0 * q3);
    R[2] = 2 * (q1 * q3 - q0 * q2);
    R[3] = 2 * (q1 * q2 - q0 * q3);
    R[4] = q0 * q0 - q1 * q1 + q2 * q2 - q3 * q3;
    R[5] = 2 * (q2 * q3 + q0 * q1);
    R[6] = 2 * (q1 * q3 + q0 * q2);
    R[7] = 2 * (q2 * q3 - q0 * q1);
    R[8] = q0 * q0 - q1 * q1 - q2 * q2 + q3 * q3;
    return true;
}

// Horn's 4x4 from the 3x3 covariance H -> dominant eigenvector -> rotation
// (indialign_c/core.h:64-90): the characteristic-polynomial solve above, or
// the reference's Jacobi sequence when the top eigenvalue is not separated.
IA_DEV void cov_to_rotation(const double (&H)[3][3], double *R) {
    double A[4][4], V[4][4];
    horn_matrix(H, A);
    if (qcp_rotation(A, R)) return;
    jacobi_reference(A, V);
    quat_to_rotation(A, V, R);
}

// Raw first and second moments of a selected point set.
struct Moments {
    double sp[3], sq[3], h[9], w;
    IA_DEV void clear() {
#pragma unroll
        for (int i = 0; i < 3; i++) sp[i] = sq[i] = 0.0;
#pragma unroll
        for (int i = 0; i < 9; i++) h[i] = 0.0;
        w = 0.0;
    }
    IA_DEV void add(double px, double py, double pz, double qx, double qy,
                    double qz) {
        sp[0] += px; sp[1] += py; sp[2] += pz;
        sq[0] += qx; sq[1] += qy; sq[2] += qz;
        h[0] += px * qx; h[1] += px * qy; h[2] += px * qz;
        h[3] += py * qx; h[4] += py * qy; h[5] += py * qz;
        h[6] += pz * qx; h[7] += pz * qy; h[8] += pz * qz;
        w += 1.0;
    }
    IA_DEV void add_w(double wi, double px, double py, double pz, double qx,
                      double qy, double qz) {
        double wx = wi * px, wy = wi * py, wz = wi * pz;
        sp[0] += wx; sp[1] += wy; sp[2] += wz;
        sq[0] += wi * qx; sq[1] += wi * qy; sq[2] += wi * qz;
        h[0] += wx * qx; h[1] += wx * qy; h[2] += wx * qz;
        h[3] += wy * qx; h[4] += wy * qy; h[5] += wy * qz;
        h[6] += wz * qx; h[7] += wz * qy; h[8] += wz * qz;
        w += wi;
    }
    // Butterfly sum over the lanes of `width` (power of two) so that every
    // lane of the group ends with the group total.
    IA_DEV void group_sum(int width) {
        for (int o = 1; o < width; o <<= 1) {
#pragma unroll
            for (int i = 0; i < 3; i++) {
                sp[i] += __shfl_xor_sync(0xffffffffu, sp[i], o);
                sq[i] += __shfl_xor_sync(0xffffffffu, sq[i], o);
            }
#pragma unroll
            for (int i = 0; i < 9; i++) h[i] += __shfl_xor_sync(0xffffffffu, h[i], o);
            w += __shfl_xor_sync(0xffffffffu, w, o);
        }
    }
};

// Kabsch from moments: identity when the weight is below `min_w`
// (3 points for the plain Kabsch, 1e-12 for the weighted one).
static __device__ __noinline__ void kabsch_from_moments(const Moments &m, double min_w, double *R,
                                                  double *t) {
    if (m.w < min_w) {
        set_identity(R, t);
        return;
    }
    double cP[3], cQ[3], H[3][3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        cP[d] = m.sp[d] / m.w;
        cQ[d] = m.sq[d] / m.w;
    }
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) H[r][c] = m.h[r * 3 + c] - m.sp[r] * cQ[c];
    cov_to_rotation(H, R);
#pragma unroll
    for (int d = 0; d < 3; d++)
        t[d] = cQ[d] - (cP[0] * R[d] + cP[1] * R[3 + d] + cP[2] * R[6 + d]);
}

IA_DEV double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

IA_DEV int warp_sum_int(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Compact coordinate views of one pair (pred / native restricted to their
// valid residues), as used by the chain and ranker kernels.
struct Pts {
    const double *P;  // pred compact xyz
    const double *Q;  // native compact xyz
};

// Kabsch over pairs (P[a+i], Q[b+i]), i < cnt (a window), by the warp.
IA_DEV void warp_kabsch_window(const Pts &x, int a, int b, int cnt, double *R, double *t) {
    Moments m;
    m.clear();
    for (int i = threadIdx.x & 31; i < cnt; i += 32) {
        const double *p = x.P + 3 * (a + i), *q = x.Q + 3 * (b + i);
        m.add(p[0], p[1], p[2], q[0], q[1], q[2]);
    }
    m.group_sum(32);
    kabsch_from_moments(m, 3.0, R, t);
}

}  // namespace ia
