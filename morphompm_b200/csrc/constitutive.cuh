// Constitutive models of the growth step, forward Kirchhoff stress and the
// hand-written vector-Jacobian products, on register-resident 3x3 matrices.
//
//   neo-Hookean        python/morphompm/constitutive.py:25-39
//   Hencky             python/morphompm/constitutive.py:42-75
//   Herschel-Bulkley   python/morphompm/constitutive.py:106-147
//
// Morphoelastic kinematics Fe = F Fg^{-1}.  Hencky is evaluated as an
// isotropic function of b = Fe Fe^T through a symmetric 3x3 eigensolve (FP64:
// cyclic Jacobi rotations, Rutishauser's update; FP32: closed form from the
// characteristic cubic), which is equivalent to the reference's SVD form
// tau = U diag(2 mu ln s + lam sum ln s) U^T since b = U S^2 U^T.
#pragma once

#include "mpm_common.cuh"

namespace mpm {

// ---------------------------------------------------------------------------
// symmetric 3x3 eigen-decomposition by cyclic Jacobi rotations.
// On return lam[i] are the eigenvalues and column i of V (row-major) the
// corresponding unit eigenvector.
// ---------------------------------------------------------------------------
// One rotation annihilating A[p][q].  An off-diagonal entry at or below the
// rounding level of its diagonal (|a_pq| <= eps (|a_pp| + |a_qq|) / 4) is set to
// zero without rotating; returns whether a rotation was applied.
template <typename R>
__device__ __forceinline__ bool jacobi_rotate(R A[3][3], R V[9], int p, int q) {
    R apq = A[p][q];
    if (d_abs(apq) <= R(0.25) * Num<R>::eps * (d_abs(A[p][p]) + d_abs(A[q][q]))) {
        A[p][q] = R(0);
        A[q][p] = R(0);
        return false;
    }
    R t, c, s, tau;
    if constexpr (sizeof(R) == 4) {
        // FP32: hardware reciprocal / reciprocal square root.  t need not be
        // the exact tangent (the annihilated entry is set to zero, an error at
        // rounding level); c gets one Newton step for 1/sqrt so that (c, s)
        // stays a rotation to rounding level.
        const float theta = __fdividef(A[q][q] - A[p][p], 2.0f * apq);
        const float h2 = fmaf(theta, theta, 1.0f);
        t = __fdividef(1.0f, fabsf(theta) + h2 * rsqrtf(h2));
        if (theta < 0.0f) t = -t;
        const float u = fmaf(t, t, 1.0f);
        float r = rsqrtf(u);
        r = r * fmaf(-0.5f * u * r, r, 1.5f);
        c = r;
        s = t * c;
        tau = __fdividef(s, 1.0f + c);
    } else {
        R theta = (A[q][q] - A[p][p]) / (R(2) * apq);
        t = R(1) / (d_abs(theta) + d_sqrt(theta * theta + R(1)));
        if (theta < R(0)) t = -t;
        c = R(1) / d_sqrt(t * t + R(1));
        s = t * c;
        tau = s / (R(1) + c);
    }
    A[p][p] -= t * apq;
    A[q][q] += t * apq;
    A[p][q] = R(0);
    A[q][p] = R(0);
    int r = 3 - p - q;
    R arp = A[r][p], arq = A[r][q];
    R nrp = arp - s * (arq + tau * arp);
    R nrq = arq + s * (arp - tau * arq);
    A[r][p] = nrp; A[p][r] = nrp;
    A[r][q] = nrq; A[q][r] = nrq;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        R vkp = V[3 * k + p], vkq = V[3 * k + q];
        V[3 * k + p] = vkp - s * (vkq + tau * vkp);
        V[3 * k + q] = vkq + s * (vkp - tau * vkq);
    }
    return true;
}

// Cyclic sweeps until a sweep finds every off-diagonal entry at rounding level
// (quadratic convergence: typically 3-4 sweeps in FP64, 2-3 in FP32).
template <typename R>
__device__ __forceinline__ void sym_eig3(const R S[9], R lam[3], R V[9]) {
    R A[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) A[i][j] = R(0.5) * (S[3 * i + j] + S[3 * j + i]);
#pragma unroll
    for (int i = 0; i < 9; ++i) V[i] = (i % 4 == 0) ? R(1) : R(0);
    const int max_sweeps = sizeof(R) == 8 ? 10 : 6;
    for (int sweep = 0; sweep < max_sweeps; ++sweep) {
        bool r0 = jacobi_rotate(A, V, 0, 1);
        bool r1 = jacobi_rotate(A, V, 0, 2);
        bool r2 = jacobi_rotate(A, V, 1, 2);
        if (!(r0 || r1 || r2)) break;
    }
    lam[0] = A[0][0];
    lam[1] = A[1][1];
    lam[2] = A[2][2];
}

// FP32 symmetric 3x3 eigensolve in closed form, no iteration (the trigonometric
// solution of the characteristic cubic; Smith, "Eigenvalues of a symmetric 3x3
// matrix", CACM 4(4), 1961):
//   m = tr(A)/3, p = sqrt(|A - mI|_F^2 / 6), r = det((A - mI)/p)/2,
//   phi = acos(r)/3, lambda = m + 2p cos(phi + 2k pi/3).
// The eigenvector of the eigenvalue farthest from the other two is the largest
// cross product of two rows of A - lambda I (well conditioned: its gap is at
// least half the spread).  The other two come from one Jacobi rotation of A
// restricted to the orthogonal complement of that vector, and all three
// eigenvalues are then Rayleigh quotients, accurate to FP32 rounding of |A|
// also when two of them are close (the cubic's roots are not, there).
// Columns of V are the eigenvectors, V[3k + j] = component k of vector j.
__device__ __forceinline__ void sym_eig3_closed(const float S[9], float lam[3], float V[9]) {
    const float a00 = S[0], a11 = S[4], a22 = S[8];
    const float a01 = 0.5f * (S[1] + S[3]), a02 = 0.5f * (S[2] + S[6]), a12 = 0.5f * (S[5] + S[7]);
    const float m = (a00 + a11 + a22) * (1.0f / 3.0f);
    const float b00 = a00 - m, b11 = a11 - m, b22 = a22 - m;
    const float p2 = (b00 * b00 + b11 * b11 + b22 * b22 + 2.0f * (a01 * a01 + a02 * a02 + a12 * a12)) * (1.0f / 6.0f);
    if (!(p2 > 1e-15f * m * m)) {
        // spread below FP32 resolution of the trace: the diagonal is the spectrum
        lam[0] = a00; lam[1] = a11; lam[2] = a22;
#pragma unroll
        for (int i = 0; i < 9; ++i) V[i] = (i % 4 == 0) ? 1.0f : 0.0f;
        return;
    }
    const float ip = rsqrtf(p2), p = p2 * ip;
    const float c00 = b00 * ip, c11 = b11 * ip, c22 = b22 * ip, c01 = a01 * ip, c02 = a02 * ip, c12 = a12 * ip;
    float r = 0.5f * (c00 * (c11 * c22 - c12 * c12) - c01 * (c01 * c22 - c12 * c02) + c02 * (c01 * c12 - c11 * c02));
    r = fminf(1.0f, fmaxf(-1.0f, r));
    float sp, cp;
    sincosf(acosf(r) * (1.0f / 3.0f), &sp, &cp);
    const float l0 = m + 2.0f * p * cp;                                   // largest
    const float l2 = m - p * (cp + 1.7320508075688772f * sp);             // smallest: cos(phi + 2pi/3)
    const float l1 = 3.0f * m - l0 - l2;
    const float le = (l0 - l1) >= (l1 - l2) ? l0 : l2;
    // rows of A - le I; eigenvector = largest cross product of two rows
    const float r00 = a00 - le, r11 = a11 - le, r22 = a22 - le;
    float x0 = a01 * a12 - a02 * r11, x1 = a02 * a01 - r00 * a12, x2 = r00 * r11 - a01 * a01;   // row0 x row1
    float y0 = a01 * r22 - a02 * a12, y1 = a02 * a02 - r00 * r22, y2 = r00 * a12 - a01 * a02;   // row0 x row2
    float z0 = r11 * r22 - a12 * a12, z1 = a12 * a02 - a01 * r22, z2 = a01 * a12 - r11 * a02;   // row1 x row2
    float nx = x0 * x0 + x1 * x1 + x2 * x2, ny = y0 * y0 + y1 * y1 + y2 * y2, nz = z0 * z0 + z1 * z1 + z2 * z2;
    if (ny > nx) { x0 = y0; x1 = y1; x2 = y2; nx = ny; }
    if (nz > nx) { x0 = z0; x1 = z1; x2 = z2; nx = nz; }
    float v0 = 1.0f, v1 = 0.0f, v2 = 0.0f;
    if (nx > 0.0f) {
        const float in = rsqrtf(nx);
        v0 = x0 * in; v1 = x1 * in; v2 = x2 * in;
    }
    // orthonormal complement u, w of v
    float u0, u1, u2;
    if (fabsf(v0) > fabsf(v1)) {
        const float in = rsqrtf(v0 * v0 + v2 * v2);
        u0 = -v2 * in; u1 = 0.0f; u2 = v0 * in;
    } else {
        const float in = rsqrtf(v1 * v1 + v2 * v2);
        u0 = 0.0f; u1 = v2 * in; u2 = -v1 * in;
    }
    const float w0 = v1 * u2 - v2 * u1, w1 = v2 * u0 - v0 * u2, w2 = v0 * u1 - v1 * u0;
    // A restricted to span(u, w): [[a, b], [b, c]]
    const float Au0 = a00 * u0 + a01 * u1 + a02 * u2, Au1 = a01 * u0 + a11 * u1 + a12 * u2,
                Au2 = a02 * u0 + a12 * u1 + a22 * u2;
    const float Aw0 = a00 * w0 + a01 * w1 + a02 * w2, Aw1 = a01 * w0 + a11 * w1 + a12 * w2,
                Aw2 = a02 * w0 + a12 * w1 + a22 * w2;
    const float Av0 = a00 * v0 + a01 * v1 + a02 * v2, Av1 = a01 * v0 + a11 * v1 + a12 * v2,
                Av2 = a02 * v0 + a12 * v1 + a22 * v2;
    const float ra = u0 * Au0 + u1 * Au1 + u2 * Au2;
    const float rb = u0 * Aw0 + u1 * Aw1 + u2 * Aw2;
    const float rc = w0 * Aw0 + w1 * Aw1 + w2 * Aw2;
    float t = 0.0f;
    if (rb != 0.0f) {
        const float th = (rc - ra) / (2.0f * rb);
        t = copysignf(1.0f, th) / (fabsf(th) + sqrtf(th * th + 1.0f));
    }
    const float cs = rsqrtf(t * t + 1.0f), sn = t * cs;
    lam[0] = v0 * Av0 + v1 * Av1 + v2 * Av2;
    lam[1] = ra - t * rb;
    lam[2] = rc + t * rb;
    V[0] = v0; V[3] = v1; V[6] = v2;
    V[1] = cs * u0 - sn * w0; V[4] = cs * u1 - sn * w1; V[7] = cs * u2 - sn * w2;
    V[2] = sn * u0 + cs * w0; V[5] = sn * u1 + cs * w1; V[8] = sn * u2 + cs * w2;
}

// Model parameters in the arithmetic type of the path.
template <typename R>
struct ModelParams {
    int kind;
    R mu, lam;
    R kappa, K, n, tau_y, m, eps;
    __device__ __forceinline__ void load(const MpmScene& sc) {
        kind = sc.model;
        mu = (R)sc.mu; lam = (R)sc.lam;
        kappa = (R)sc.kappa; K = (R)sc.K; n = (R)sc.n_exp;
        tau_y = (R)sc.tau_y; m = (R)sc.m_pap; eps = (R)sc.eps;
    }
};

// F_bar = Fe_bar Fg^{-T};  Fg_bar = -Fg^{-T} F^T Fe_bar Fg^{-T}   (constitutive.py:37-38, 73-74)
template <typename R>
__device__ __forceinline__ void pull_back(const R F[9], const R Fgi[9], const R Feb[9], R Fb[9], R Fgb[9]) {
    mmT(Feb, Fgi, Fb);              // Fe_bar Fg^{-T}
    R T1[9], T2[9];
    mTm(F, Fb, T1);                 // F^T (Fe_bar Fg^{-T})
    mTm(Fgi, T1, T2);               // Fg^{-T} F^T Fe_bar Fg^{-T}
#pragma unroll
    for (int i = 0; i < 9; ++i) Fgb[i] = -T2[i];
}

// ---------------------------------------------------------------------------
// neo-Hookean: tau = mu (Fe Fe^T - I) + lam ln J I
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ void nh_stress(const R F[9], const R Fg[9], R mu, R lam, R tau[9]) {
    R Fgi[9], Fe[9];
    inv3(Fg, Fgi);
    mm(F, Fgi, Fe);
    R J = det3(Fe);
    R lnJ = d_log(J);
    mmT(Fe, Fe, tau);
#pragma unroll
    for (int i = 0; i < 9; ++i) tau[i] = mu * (tau[i] - ((i % 4 == 0) ? R(1) : R(0)));
    tau[0] += lam * lnJ; tau[4] += lam * lnJ; tau[8] += lam * lnJ;
}
template <typename R>
__device__ __forceinline__ void nh_vjp(const R F[9], const R Fg[9], R mu, R lam, const R tau_bar[9],
                                       R Fb[9], R Fgb[9]) {
    R Fgi[9], Fe[9], Fei[9], tb[9];
    inv3(Fg, Fgi);
    mm(F, Fgi, Fe);
    inv3(Fe, Fei);
    sym(tau_bar, tb);
    R tr = tb[0] + tb[4] + tb[8];
    R Feb[9], T[9];
    mm(tb, Fe, T);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            Feb[3 * i + j] = R(2) * mu * T[3 * i + j] + lam * tr * Fei[3 * j + i];
    pull_back(F, Fgi, Feb, Fb, Fgb);
}

// ---------------------------------------------------------------------------
// Hencky.  The FP64 instantiation applies the reference's divided-difference
// rule exactly (|beta_i - beta_j| > 1e-9 -> (ln bi - ln bj)/(bi - bj), else
// 1/beta_i; constitutive.py:66-70).  The FP32 instantiation uses the
// cancellation-free form log1p(d)/(beta_j d), d = (beta_i - beta_j)/beta_j, and
// recomputes particles whose relative singular-value gap is below the
// threshold in FP64.
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ void hencky_eig(const R F[9], const R Fg[9], R Fgi[9], R Fe[9], R beta[3], R V[9]) {
    inv3(Fg, Fgi);
    mm(F, Fgi, Fe);
    R b[9];
    mmT(Fe, Fe, b);
    if constexpr (sizeof(R) == 4) {
        sym_eig3_closed(b, beta, V);      // FP32: closed form
    } else {
        sym_eig3(b, beta, V);             // FP64: Jacobi sweeps to full precision
    }
}

template <typename R>
__device__ __forceinline__ void hencky_tau_from_eig(const R beta[3], const R V[9], R mu, R lam, R tau[9]) {
    R lb[3] = {d_log(beta[0]), d_log(beta[1]), d_log(beta[2])};
    R S = lb[0] + lb[1] + lb[2];
    R h[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) h[i] = mu * lb[i] + R(0.5) * lam * S;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j) {
            tau[3 * i + j] = V[3 * i] * h[0] * V[3 * j] + V[3 * i + 1] * h[1] * V[3 * j + 1]
                           + V[3 * i + 2] * h[2] * V[3 * j + 2];
            tau[3 * j + i] = tau[3 * i + j];
        }
}

template <typename R>
__device__ __forceinline__ R dk_entry(R bi, R bj, R lbi, R lbj);

template <>
__device__ __forceinline__ double dk_entry<double>(double bi, double bj, double lbi, double lbj) {
    double d = bi - bj;
    return fabs(d) > 1.0e-9 ? (lbi - lbj) / d : 1.0 / bi;
}
template <>
__device__ __forceinline__ float dk_entry<float>(float bi, float bj, float, float) {
    if (bi == bj) return 1.0f / bi;
    float d = (bi - bj) / bj;
    return log1pf(d) / (bj * d);
}
// the cancellation-free form in FP64 (the FP64 recompute of an FP32 particle
// near degeneracy must not fall back to the 1e-9 switch)
__device__ __forceinline__ double dk_stable(double bi, double bj) {
    if (bi == bj) return 1.0 / bi;
    const double d = (bi - bj) / bj;
    return log1p(d) / (bj * d);
}

// STABLE: the cancellation-free divided difference also in FP64.
template <typename R, bool STABLE = false>
__device__ __forceinline__ void hencky_vjp_from_eig(const R F[9], const R Fgi[9], const R Fe[9], const R beta[3],
                                                    const R V[9], R mu, R lam, const R tau_bar[9],
                                                    R Fb[9], R Fgb[9]) {
    R tb[9];
    sym(tau_bar, tb);
    R tr = tb[0] + tb[4] + tb[8];
    R M[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) M[i] = mu * tb[i] + ((i % 4 == 0) ? R(0.5) * lam * tr : R(0));
    // M, V^T M V and V (. o L) V^T are symmetric: only the upper triangle is formed
    R T[9], UtMU[9];
    mTm(V, M, T);         // V^T M
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j) {
            UtMU[3 * i + j] = T[3 * i] * V[j] + T[3 * i + 1] * V[3 + j] + T[3 * i + 2] * V[6 + j];
            UtMU[3 * j + i] = UtMU[3 * i + j];
        }
    R lb[3];
    if constexpr (!STABLE) {
#pragma unroll
        for (int i = 0; i < 3; ++i) lb[i] = d_log(beta[i]);
    }
    auto dk = [&](int i, int j) -> R {
        if constexpr (STABLE) return dk_stable(beta[i], beta[j]);
        else return dk_entry<R>(beta[i], beta[j], lb[i], lb[j]);
    };
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        UtMU[4 * i] *= dk(i, i);
#pragma unroll
        for (int j = i + 1; j < 3; ++j) {
            const R L = dk(i, j);
            UtMU[3 * i + j] *= L;
            UtMU[3 * j + i] *= L;
        }
    }
    R Bb[9];
    mm(V, UtMU, T);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j) {
            Bb[3 * i + j] = T[3 * i] * V[3 * j] + T[3 * i + 1] * V[3 * j + 1] + T[3 * i + 2] * V[3 * j + 2];
            Bb[3 * j + i] = Bb[3 * i + j];
        }
    R Feb[9];
    mm(Bb, Fe, Feb);
#pragma unroll
    for (int i = 0; i < 9; ++i) Feb[i] *= R(2);
    pull_back(F, Fgi, Feb, Fb, Fgb);
}

// relative singular-value gap: min |s_i - s_j| / max s  with s = sqrt(beta)
template <typename R>
__device__ __forceinline__ R sv_gap(const R beta[3]) {
    R s0 = d_sqrt(beta[0] > R(0) ? beta[0] : R(0));
    R s1 = d_sqrt(beta[1] > R(0) ? beta[1] : R(0));
    R s2 = d_sqrt(beta[2] > R(0) ? beta[2] : R(0));
    R mx = s0 > s1 ? s0 : s1;
    mx = mx > s2 ? mx : s2;
    R g01 = d_abs(s0 - s1), g02 = d_abs(s0 - s2), g12 = d_abs(s1 - s2);
    R g = g01 < g02 ? g01 : g02;
    g = g < g12 ? g : g12;
    return g / mx;
}

template <typename R>
struct Hencky {
    // both return whether the FP64 path was taken
    static __device__ __forceinline__ bool stress(const R F[9], const R Fg[9], R mu, R lam, float, R tau[9]) {
        R Fgi[9], Fe[9], beta[3], V[9];
        hencky_eig(F, Fg, Fgi, Fe, beta, V);
        hencky_tau_from_eig(beta, V, mu, lam, tau);
        return false;
    }
    static __device__ __forceinline__ bool vjp(const R F[9], const R Fg[9], R mu, R lam, float, const R tb[9],
                                               R Fb[9], R Fgb[9]) {
        R Fgi[9], Fe[9], beta[3], V[9];
        hencky_eig(F, Fg, Fgi, Fe, beta, V);
        hencky_vjp_from_eig(F, Fgi, Fe, beta, V, mu, lam, tb, Fb, Fgb);
        return false;
    }
};

// FP64 recompute of an FP32 Hencky particle (stress, VJP): float in and out,
// double inside.  The stable divided difference is used here too (the
// recompute of a near-degenerate particle must not fall back to the 1e-9
// switch).
__device__ __forceinline__ void hencky_stress_fp64(const float F[9], const float Fg[9], float mu, float lam,
                                                   float tau[9]) {
    double Fd[9], Fgd[9], Fgid[9], Fed[9], bd[3], Vd[9], td[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) { Fd[i] = F[i]; Fgd[i] = Fg[i]; }
    hencky_eig(Fd, Fgd, Fgid, Fed, bd, Vd);
    hencky_tau_from_eig(bd, Vd, (double)mu, (double)lam, td);
#pragma unroll
    for (int i = 0; i < 9; ++i) tau[i] = (float)td[i];
}
__device__ __forceinline__ void hencky_vjp_fp64(const float F[9], const float Fg[9], float mu, float lam,
                                                const float tb[9], float Fb[9], float Fgb[9]) {
    double Fd[9], Fgd[9], Fgid[9], Fed[9], bd[3], Vd[9], tbd[9], Fbd[9], Fgbd[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) { Fd[i] = F[i]; Fgd[i] = Fg[i]; tbd[i] = tb[i]; }
    hencky_eig(Fd, Fgd, Fgid, Fed, bd, Vd);
    hencky_vjp_from_eig<double, true>(Fd, Fgid, Fed, bd, Vd, (double)mu, (double)lam, tbd, Fbd, Fgbd);
#pragma unroll
    for (int i = 0; i < 9; ++i) { Fb[i] = (float)Fbd[i]; Fgb[i] = (float)Fgbd[i]; }
}

template <>
struct Hencky<float> {
    static __device__ __forceinline__ bool stress(const float F[9], const float Fg[9], float mu, float lam,
                                                  float thresh, float tau[9]) {
        float Fgi[9], Fe[9], beta[3], V[9];
        hencky_eig(F, Fg, Fgi, Fe, beta, V);
        if (sv_gap(beta) >= thresh) {
            hencky_tau_from_eig(beta, V, mu, lam, tau);
            return false;
        }
        hencky_stress_fp64(F, Fg, mu, lam, tau);
        return true;
    }
    static __device__ __forceinline__ bool vjp(const float F[9], const float Fg[9], float mu, float lam,
                                               float thresh, const float tb[9], float Fb[9], float Fgb[9]) {
        float Fgi[9], Fe[9], beta[3], V[9];
        hencky_eig(F, Fg, Fgi, Fe, beta, V);
        if (sv_gap(beta) >= thresh) {
            hencky_vjp_from_eig(F, Fgi, Fe, beta, V, mu, lam, tb, Fb, Fgb);
            return false;
        }
        hencky_vjp_fp64(F, Fg, mu, lam, tb, Fb, Fgb);
        return true;
    }
};

// ---------------------------------------------------------------------------
// Herschel-Bulkley (Papanastasiou-regularised), rate dependent through C.
//   tau = kappa ln(Je) I + 2 eta(gdot) D,  D = sym(C),  gdot = sqrt(2 D:D + eps^2)
//   eta = K gdot^(n-1) + tau_y (1 - exp(-m gdot)) / gdot
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ void hb_stress(const R F[9], const R Fg[9], const R C[9], const ModelParams<R>& P,
                                          R tau[9]) {
    R Je = det3(F) / det3(Fg);
    R D[9];
    sym(C, D);
    R gdot = d_sqrt(R(2) * frob(D, D) + P.eps * P.eps);
    R eta = P.K * d_pow(gdot, P.n - R(1)) + P.tau_y * (R(1) - d_exp(-P.m * gdot)) / gdot;
    R vol = P.kappa * d_log(Je);
#pragma unroll
    for (int i = 0; i < 9; ++i) tau[i] = R(2) * eta * D[i] + ((i % 4 == 0) ? vol : R(0));
}
template <typename R>
__device__ __forceinline__ void hb_vjp(const R F[9], const R Fg[9], const R C[9], const ModelParams<R>& P,
                                       const R tau_bar[9], R Fb[9], R Fgb[9], R Cb[9]) {
    R tb[9];
    sym(tau_bar, tb);
    R tr = tb[0] + tb[4] + tb[8];
    R Fi[9], Fgi[9];
    inv3(F, Fi);
    inv3(Fg, Fgi);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            Fb[3 * i + j] = P.kappa * tr * Fi[3 * j + i];
            Fgb[3 * i + j] = -P.kappa * tr * Fgi[3 * j + i];
        }
    R D[9];
    sym(C, D);
    R gdot = d_sqrt(R(2) * frob(D, D) + P.eps * P.eps);
    R e = d_exp(-P.m * gdot);
    R eta = P.K * d_pow(gdot, P.n - R(1)) + P.tau_y * (R(1) - e) / gdot;
    R deta = P.K * (P.n - R(1)) * d_pow(gdot, P.n - R(2))
           + P.tau_y * ((P.m * e) * gdot - (R(1) - e)) / (gdot * gdot);
    R tbD = frob(tb, D);
    R k = R(4) * tbD * deta / gdot;
#pragma unroll
    for (int i = 0; i < 9; ++i) Cb[i] = R(2) * eta * tb[i] + k * D[i];
}

// ---------------------------------------------------------------------------
// Out-of-line Hencky VJP for the run-time model switch (the stand-alone VJP
// and the kernels over mixed or external scenes), so that its register demand
// does not inflate the allocation of the kernels that fuse it.  The FP64
// recompute of the stress is inline in every kernel, and so is the VJP's in
// the model-specialised reverse kernels: out of line, such a call passes its
// arrays through the local-memory stack and measured slower even on the rare
// path (reverse kernel 179.3 -> 186.2 ms, G2P 93.6 -> 96.7 ms per config-4
// trajectory).
// ---------------------------------------------------------------------------
template <typename R>
__device__ __noinline__ bool hencky_vjp_ool(const R* F, const R* Fg, R mu, R lam, float thresh, const R* tb, R* Fb,
                                            R* Fgb) {
    return Hencky<R>::vjp(F, Fg, mu, lam, thresh, tb, Fb, Fgb);
}
// ---------------------------------------------------------------------------
// Hencky with the eigendecomposition kept between the stress (before the P2G
// adjoint gather) and the VJP (after it): one eigensolve per particle in the
// reverse kernel.  keep = {beta[3], V[9], flag}; flag 1 means the FP32 stress
// went to FP64 and the VJP must do the same.
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ bool hencky_stress_keep(const R* F, const R* Fg, R mu, R lam, float thresh, R* tau,
                                                R* keep) {
    R Fgi[9], Fe[9], beta[3], V[9];
    hencky_eig(F, Fg, Fgi, Fe, beta, V);
    bool fp64 = false;
    if constexpr (sizeof(R) == 4) fp64 = sv_gap(beta) < thresh;
    if (fp64) {
        // the FP32 solve above already failed the gap test: straight to FP64
        if constexpr (sizeof(R) == 4) hencky_stress_fp64(F, Fg, mu, lam, tau);
    } else {
        hencky_tau_from_eig(beta, V, mu, lam, tau);
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) keep[i] = beta[i];
#pragma unroll
    for (int i = 0; i < 9; ++i) keep[3 + i] = V[i];
    keep[12] = fp64 ? R(1) : R(0);
    return fp64;
}
template <typename R>
__device__ __forceinline__ bool hencky_vjp_keep(const R* F, const R* Fg, R mu, R lam, float thresh, const R* tb,
                                             const R* keep, R* Fb, R* Fgb) {
    if constexpr (sizeof(R) == 4) {
        if (keep[12] != R(0)) {         // the stress went to FP64: so does the VJP
            hencky_vjp_fp64(F, Fg, mu, lam, tb, Fb, Fgb);
            return true;
        }
    }
    R Fgi[9], Fe[9], beta[3], V[9];
    inv3(Fg, Fgi);
    mm(F, Fgi, Fe);
#pragma unroll
    for (int i = 0; i < 3; ++i) beta[i] = keep[i];
#pragma unroll
    for (int i = 0; i < 9; ++i) V[i] = keep[3 + i];
    hencky_vjp_from_eig(F, Fgi, Fe, beta, V, mu, lam, tb, Fb, Fgb);
    return false;
}

// ---------------------------------------------------------------------------
// model dispatch.  Returns true when an FP32 Hencky evaluation went to FP64.
// The FP32 eigensolves are inlined; the out-of-line wrappers above carry the
// stand-alone Hencky VJP and the rare FP64 recomputes.
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ bool model_stress(const ModelParams<R>& P, float thresh, const R F[9], const R Fg[9],
                                             const R C[9], R tau[9]) {
    if (P.kind == MPM_MODEL_HENCKY) {
        // the eigensolve inline; only the rare FP32 -> FP64 recompute out of line
        R Fgi[9], Fe[9], beta[3], V[9];
        hencky_eig(F, Fg, Fgi, Fe, beta, V);
        if constexpr (sizeof(R) == 4) {
            if (sv_gap(beta) < thresh) {     // rare: straight to FP64, inline
                hencky_stress_fp64(F, Fg, P.mu, P.lam, tau);
                return true;
            }
        }
        hencky_tau_from_eig(beta, V, P.mu, P.lam, tau);
        return false;
    }
    if (P.kind == MPM_MODEL_HERSCHEL_BULKLEY) { hb_stress<R>(F, Fg, C, P, tau); return false; }
    nh_stress(F, Fg, P.mu, P.lam, tau);
    return false;
}
template <typename R>
__device__ __forceinline__ bool model_vjp(const ModelParams<R>& P, float thresh, const R F[9], const R Fg[9],
                                          const R C[9], const R tb[9], R Fb[9], R Fgb[9], R Cb[9]) {
    if (P.kind == MPM_MODEL_HERSCHEL_BULKLEY) { hb_vjp<R>(F, Fg, C, P, tb, Fb, Fgb, Cb); return false; }
#pragma unroll
    for (int i = 0; i < 9; ++i) Cb[i] = R(0);
    if (P.kind == MPM_MODEL_HENCKY) return hencky_vjp_ool<R>(F, Fg, P.mu, P.lam, thresh, tb, Fb, Fgb);
    nh_vjp(F, Fg, P.mu, P.lam, tb, Fb, Fgb);
    return false;
}

// Stress and VJP for the reverse kernel, sharing Hencky's eigendecomposition.
template <typename R>
__device__ __forceinline__ bool model_stress_keep(const ModelParams<R>& P, float thresh, const R F[9],
                                                  const R Fg[9], const R C[9], R tau[9], R keep[13]) {
    if (P.kind == MPM_MODEL_HENCKY) return hencky_stress_keep<R>(F, Fg, P.mu, P.lam, thresh, tau, keep);
    return model_stress(P, thresh, F, Fg, C, tau);
}
template <typename R>
__device__ __forceinline__ bool model_vjp_keep(const ModelParams<R>& P, float thresh, const R F[9], const R Fg[9],
                                               const R C[9], const R tb[9], const R keep[13], R Fb[9], R Fgb[9],
                                               R Cb[9]) {
    if (P.kind == MPM_MODEL_HENCKY) {
#pragma unroll
        for (int i = 0; i < 9; ++i) Cb[i] = R(0);
        return hencky_vjp_keep<R>(F, Fg, P.mu, P.lam, thresh, tb, keep, Fb, Fgb);
    }
    return model_vjp(P, thresh, F, Fg, C, tb, Fb, Fgb, Cb);
}

// ---------------------------------------------------------------------------
// Material-parameter gradients of one particle (no counterpart in the
// reference): g[0] = <tau_bar, d tau / d mu>, g[1] = <tau_bar, d tau / d lambda>.
//   neo-Hookean: d tau/d mu = Fe Fe^T - I,      d tau/d lambda = ln J I
//   Hencky:      d tau/d mu = V diag(ln beta) V^T, d tau/d lambda = 1/2 sum ln beta I
// (Hencky from the eigendecomposition kept for the VJP, keep = {beta, V, flag}).
// Herschel-Bulkley has no Lame parameters: zero.
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ void model_param_grad(const ModelParams<R>& P, const R F[9], const R Fg[9],
                                                 const R keep[13], const R tb[9], double g[2]) {
    g[0] = 0.0;
    g[1] = 0.0;
    const R tr = tb[0] + tb[4] + tb[8];
    if (P.kind == MPM_MODEL_NEOHOOKEAN) {
        R Fgi[9], Fe[9], b[9];
        inv3(Fg, Fgi);
        mm(F, Fgi, Fe);
        mmT(Fe, Fe, b);
        R s = 0;
#pragma unroll
        for (int i = 0; i < 9; ++i) s += tb[i] * (b[i] - ((i % 4 == 0) ? R(1) : R(0)));
        g[0] = (double)s;
        g[1] = (double)(d_log(det3(Fe)) * tr);
    } else if (P.kind == MPM_MODEL_HENCKY) {
        const R lb[3] = {d_log(keep[0]), d_log(keep[1]), d_log(keep[2])};
        const R* V = keep + 3;
        R s = 0;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            // (V^T tb V)_kk = sum_ij V_ik tb_ij V_jk
            R q = 0;
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) q += V[3 * i + k] * tb[3 * i + j] * V[3 * j + k];
            s += lb[k] * q;
        }
        g[0] = (double)s;
        g[1] = (double)(R(0.5) * (lb[0] + lb[1] + lb[2]) * tr);
    }
}

}  // namespace mpm
