// fem_math.cuh -- per-element Neo-Hookean math for the row-owner kernels.
//
// Shared by the assembly kernels and the element-level parity kernel, so the
// per-element hook and the assembled system run the same code.
//
// Reference semantics (paths relative to the SORS project root):
//   F = Ds Dm^-1 (tets, cpp/src/geometries/tetrahedron.cpp:152-169),
//   F_s = X^T G_s at 8 Gauss points +-1/sqrt(3) with weights 1/8 and the
//   5-tet undeformed volume (cpp/src/geometries/hexahedron.cpp:106-207),
//   Psi = mu/2 (tr F^T F - 3) - mu log J + lam/2 log^2 J,
//   P = mu F + (lam log J - mu) F^-T  (cpp/src/energies/neoHookean.cpp:14-72),
//   d2Psi/dF2 = mu I + lam g g^T + (lam log J - mu) dF^-T/dF (:75-128).
// With B = dF/dx the element Hessian block of vertices (v,w) is
//   V wq [ mu (d_v.d_w) I + lam a_v a_w^T - c a_w a_v^T ],  a = F^-T d,
// which equals B^T (d2Psi/dF2) B without forming the 9x9 or 9x12 matrices.
//
// SPD projection (no reference counterpart): the 9x9 d2Psi/dF2 has the
// analytic eigensystem of an isotropic energy (Smith, De Goes, Kim 2019,
// "Analytic Eigensystems for Isotropic Distortion Energies"): with
// F = U diag(s) V^T, twist modes U (e_i e_j^T - e_j e_i^T) V^T / sqrt2 with
// eigenvalue mu + (c/J) s_k, flip modes (e_i e_j^T + e_j e_i^T) with
// mu - (c/J) s_k, and three scaling modes U diag(y) V^T from the 3x3 matrix
// S_ii = mu + (mu + lam (1 - log J)) / s_i^2, S_ij = lam / (s_i s_j).
// Negative modes are removed as rank-1 corrections -lam_m (B^T e_m)(B^T e_m)^T.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace sors {

// ---------------------------------------------------------------------------
// small dense helpers (row-major 3x3)
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T det3(const T* a) {
    return a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
           a[2] * (a[3] * a[7] - a[4] * a[6]);
}

// cofactor matrix: cof[r][c]; F^-T = cof / det(F)
template <typename T>
__device__ __forceinline__ void cof3(const T* a, T* c) {
    c[0] = a[4] * a[8] - a[5] * a[7];
    c[1] = a[5] * a[6] - a[3] * a[8];
    c[2] = a[3] * a[7] - a[4] * a[6];
    c[3] = a[2] * a[7] - a[1] * a[8];
    c[4] = a[0] * a[8] - a[2] * a[6];
    c[5] = a[1] * a[6] - a[0] * a[7];
    c[6] = a[1] * a[5] - a[2] * a[4];
    c[7] = a[2] * a[3] - a[0] * a[5];
    c[8] = a[0] * a[4] - a[1] * a[3];
}

template <typename T>
__device__ __forceinline__ T tet_vol6(const T* a, const T* b, const T* c, const T* d) {
    T ab0 = b[0] - a[0], ab1 = b[1] - a[1], ab2 = b[2] - a[2];
    T ac0 = c[0] - a[0], ac1 = c[1] - a[1], ac2 = c[2] - a[2];
    T ad0 = d[0] - a[0], ad1 = d[1] - a[1], ad2 = d[2] - a[2];
    T cx = ac1 * ad2 - ac2 * ad1, cy = ac2 * ad0 - ac0 * ad2, cz = ac0 * ad1 - ac1 * ad0;
    return fabs(ab0 * cx + ab1 * cy + ab2 * cz);
}

// One Jacobi rotation zeroing a[p][q] of a symmetric 3x3; v accumulates columns.
template <typename T>
__device__ __forceinline__ void jrot(T* a, T* v, int p, int q) {
    T apq = a[p * 3 + q];
    if (apq == T(0)) return;
    T app = a[p * 3 + p], aqq = a[q * 3 + q];
    T theta = (aqq - app) / (T(2) * apq);
    T t = (theta >= T(0) ? T(1) : T(-1)) / (fabs(theta) + sqrt(theta * theta + T(1)));
    if (!(t == t)) return;  // theta overflowed: already diagonal to working precision
    T c = T(1) / sqrt(t * t + T(1)), s = t * c;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        T akp = a[k * 3 + p], akq = a[k * 3 + q];
        a[k * 3 + p] = c * akp - s * akq;
        a[k * 3 + q] = s * akp + c * akq;
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
        T apk = a[p * 3 + k], aqk = a[q * 3 + k];
        a[p * 3 + k] = c * apk - s * aqk;
        a[q * 3 + k] = s * apk + c * aqk;
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
        T vkp = v[k * 3 + p], vkq = v[k * 3 + q];
        v[k * 3 + p] = c * vkp - s * vkq;
        v[k * 3 + q] = s * vkp + c * vkq;
    }
}

// Symmetric 3x3 eigen-decomposition (cyclic Jacobi, bounded sweeps).
// a is destroyed; w = eigenvalues; v = eigenvectors as columns (row-major).
template <typename T>
__device__ void sym3_eig(T* a, T* w, T* v) {
#pragma unroll
    for (int k = 0; k < 9; k++) v[k] = (k % 4 == 0) ? T(1) : T(0);
    const T eps = sizeof(T) == 8 ? T(1e-30) : T(1e-14);
    for (int sweep = 0; sweep < 8; sweep++) {
        T off = a[1] * a[1] + a[2] * a[2] + a[5] * a[5];
        T dia = a[0] * a[0] + a[4] * a[4] + a[8] * a[8];
        if (off <= eps * dia) break;
        jrot(a, v, 0, 1);
        jrot(a, v, 0, 2);
        jrot(a, v, 1, 2);
    }
    w[0] = a[0]; w[1] = a[4]; w[2] = a[8];
}

// Swap eigenpairs a and b (a, b compile-time) when w[a] < w[b].
template <typename T, int A, int B>
__device__ __forceinline__ void eig_cswap(T* w, T* V) {
    if (w[A] < w[B]) {
        T t = w[A]; w[A] = w[B]; w[B] = t;
#pragma unroll
        for (int r = 0; r < 3; r++) { T u = V[r * 3 + A]; V[r * 3 + A] = V[r * 3 + B]; V[r * 3 + B] = u; }
    }
}

// Rotation-variant SVD of F with det(F) > 0: F = U diag(s) V^T, U, V rotations,
// s sorted descending.
template <typename T>
__device__ __forceinline__ void svd3_rv(const T* F, T* U, T* s, T* V) {
    T S[9];
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) S[r * 3 + c] = F[0 * 3 + r] * F[0 * 3 + c] + F[1 * 3 + r] * F[1 * 3 + c] +
                                                   F[2 * 3 + r] * F[2 * 3 + c];
    T w[3];
    sym3_eig(S, w, V);
    eig_cswap<T, 0, 1>(w, V);
    eig_cswap<T, 0, 2>(w, V);
    eig_cswap<T, 1, 2>(w, V);
    if (det3(V) < T(0)) { V[2] = -V[2]; V[5] = -V[5]; V[8] = -V[8]; }
    T B[9];  // B = F V
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) B[r * 3 + c] = F[r * 3 + 0] * V[0 * 3 + c] + F[r * 3 + 1] * V[1 * 3 + c] + F[r * 3 + 2] * V[2 * 3 + c];
    T n0 = sqrt(B[0] * B[0] + B[3] * B[3] + B[6] * B[6]);
    T u0[3] = {B[0] / n0, B[3] / n0, B[6] / n0};
    T d01 = u0[0] * B[1] + u0[1] * B[4] + u0[2] * B[7];
    T u1[3] = {B[1] - d01 * u0[0], B[4] - d01 * u0[1], B[7] - d01 * u0[2]};
    T n1 = sqrt(u1[0] * u1[0] + u1[1] * u1[1] + u1[2] * u1[2]);
    u1[0] /= n1; u1[1] /= n1; u1[2] /= n1;
    T u2[3] = {u0[1] * u1[2] - u0[2] * u1[1], u0[2] * u1[0] - u0[0] * u1[2], u0[0] * u1[1] - u0[1] * u1[0]};
    s[0] = n0;
    s[1] = u1[0] * B[1] + u1[1] * B[4] + u1[2] * B[7];
    s[2] = u2[0] * B[2] + u2[1] * B[5] + u2[2] * B[8];
#pragma unroll
    for (int r = 0; r < 3; r++) { U[r * 3 + 0] = u0[r]; U[r * 3 + 1] = u1[r]; U[r * 3 + 2] = u2[r]; }
}

// ---------------------------------------------------------------------------
// Eigen-modes of d2Psi/dF2 at one quadrature point, held in registers.
// Mode slots are fixed: twist/flip of pair m in {(0,1), (0,2), (1,2)} and
// three scaling modes; a slot whose eigenvalue is >= 0 is skipped.
// ---------------------------------------------------------------------------
template <typename T>
struct NhModes {
    T U[9], V[9];
    T lt[3], lf[3];   // twist / flip eigenvalues of pair m
    T ls[3];          // scaling eigenvalues
    T Y[9];           // scaling eigenvectors (columns)
    bool any;
};

// J > 0 required.  The scaling block S = mu I + D^-1 M D^-1 with
// M = (mu - lam log J) I + lam 1 1^T is >= mu I when mu - lam log J >= 0,
// so its eigen-solve is skipped then.
template <typename T>
__device__ __forceinline__ void nh_modes(const T* F, T J, T logJ, T mu, T lam, NhModes<T>& pm) {
    T s[3];
    svd3_rv(F, pm.U, s, pm.V);
    const T cj = (lam * logJ - mu) / J;
    // pair m = (0,1),(0,2),(1,2) uses the third singular value s[2], s[1], s[0]
    pm.lt[0] = mu + cj * s[2]; pm.lt[1] = mu + cj * s[1]; pm.lt[2] = mu + cj * s[0];
    pm.lf[0] = mu - cj * s[2]; pm.lf[1] = mu - cj * s[1]; pm.lf[2] = mu - cj * s[0];
    pm.ls[0] = pm.ls[1] = pm.ls[2] = T(1);
#pragma unroll
    for (int k = 0; k < 9; k++) pm.Y[k] = T(0);
    if (mu - lam * logJ < T(0)) {
        T S[9];
        const T base = mu + lam * (T(1) - logJ);
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) S[i * 3 + j] = (i == j) ? mu + base / (s[i] * s[i]) : lam / (s[i] * s[j]);
        sym3_eig(S, pm.ls, pm.Y);
    }
    pm.any = false;
#pragma unroll
    for (int m = 0; m < 3; m++) pm.any |= (pm.lt[m] < T(0)) | (pm.lf[m] < T(0)) | (pm.ls[m] < T(0));
}

// u = U y for the twist (sign -1) or flip (sign +1) mode of pair (I, JJ):
// y_I = dh_JJ / sqrt2, y_JJ = sign * dh_I / sqrt2.
template <typename T, int I, int JJ>
__device__ __forceinline__ void tf_vec(const T* U, const T* dh, T sign, T* u) {
    const T r2 = T(0.70710678118654752440);
    const T yi = dh[JJ] * r2, yj = sign * dh[I] * r2;
#pragma unroll
    for (int r = 0; r < 3; r++) u[r] = U[r * 3 + I] * yi + U[r * 3 + JJ] * yj;
}

template <typename T, int M>
__device__ __forceinline__ void sc_vec(const T* U, const T* Y, const T* dh, T* u) {
    const T y0 = Y[0 * 3 + M] * dh[0], y1 = Y[1 * 3 + M] * dh[1], y2 = Y[2 * 3 + M] * dh[2];
#pragma unroll
    for (int r = 0; r < 3; r++) u[r] = U[r * 3 + 0] * y0 + U[r * 3 + 1] * y1 + U[r * 3 + 2] * y2;
}

// blk (3x3) += coef * a b^T
template <typename T>
__device__ __forceinline__ void add_outer(T* blk, T coef, const T* a, const T* b) {
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
        for (int l = 0; l < 3; l++) blk[k * 3 + l] += coef * a[k] * b[l];
}

// ---------------------------------------------------------------------------
// One quadrature point's contribution to row v of the element Hessian and
// gradient.  d: shape gradients (NV x 3, FP64); x: current positions of the
// element's vertices (NV x 3); dvd = d[v].  wV = undeformed volume x
// quadrature weight.  blk: NV blocks of 9 accumulated in registers (+=);
// g: 3 values (+=).  All array indices are compile-time: v enters only
// through dvd.  Returns false when J <= 0.
// ---------------------------------------------------------------------------
template <typename HT, int NV, bool HESS>
__device__ __forceinline__ bool nh_qp_row(const double (&d)[NV][3], const double (&x)[NV][3], const double (&dvd)[3],
                                          double wV, double mu, double lam, bool project, double* g,
                                          HT (&blk)[NV * 9]) {
    double F[9];
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
            double acc = 0.0;
#pragma unroll
            for (int w = 0; w < NV; w++) acc += x[w][r] * d[w][c];
            F[r * 3 + c] = acc;
        }
    double C[9];
    cof3(F, C);
    const double J = F[0] * C[0] + F[1] * C[1] + F[2] * C[2];
    const double logJ = log(J);
    const double iJ = 1.0 / J;
    double G[9];
#pragma unroll
    for (int k = 0; k < 9; k++) G[k] = C[k] * iJ;
    const double cc = lam * logJ - mu;
    // gradient row v: wV * (mu F + c G) d_v
#pragma unroll
    for (int r = 0; r < 3; r++) {
        double pr = 0.0;
#pragma unroll
        for (int c = 0; c < 3; c++) pr += (mu * F[r * 3 + c] + cc * G[r * 3 + c]) * dvd[c];
        g[r] += wV * pr;
    }
    if (!(J > 0.0)) return false;
    if (!HESS) return true;
    HT Gh[9];
#pragma unroll
    for (int k = 0; k < 9; k++) Gh[k] = (HT)G[k];
    const HT dv[3] = {(HT)dvd[0], (HT)dvd[1], (HT)dvd[2]};
    HT av[3];
#pragma unroll
    for (int r = 0; r < 3; r++) av[r] = Gh[r * 3 + 0] * dv[0] + Gh[r * 3 + 1] * dv[1] + Gh[r * 3 + 2] * dv[2];
    const HT hmu = (HT)(wV * mu), hlam = (HT)(wV * lam), hc = (HT)(wV * cc);
#pragma unroll
    for (int w = 0; w < NV; w++) {
        const HT dw[3] = {(HT)d[w][0], (HT)d[w][1], (HT)d[w][2]};
        HT aw[3];
#pragma unroll
        for (int r = 0; r < 3; r++) aw[r] = Gh[r * 3 + 0] * dw[0] + Gh[r * 3 + 1] * dw[1] + Gh[r * 3 + 2] * dw[2];
        const HT dd = dv[0] * dw[0] + dv[1] * dw[1] + dv[2] * dw[2];
#pragma unroll
        for (int k = 0; k < 3; k++)
#pragma unroll
            for (int l = 0; l < 3; l++) {
                HT val = hlam * av[k] * aw[l] - hc * aw[k] * av[l];
                if (k == l) val += hmu * dd;
                blk[w * 9 + k * 3 + l] += val;
            }
    }
    if (project) {
        HT Fh[9];
#pragma unroll
        for (int k = 0; k < 9; k++) Fh[k] = (HT)F[k];
        NhModes<HT> pm;
        nh_modes<HT>(Fh, (HT)J, (HT)logJ, (HT)mu, (HT)lam, pm);
        if (pm.any) {
            const HT wv = (HT)wV;
            HT dhv[3];
#pragma unroll
            for (int c = 0; c < 3; c++) dhv[c] = pm.V[0 * 3 + c] * dv[0] + pm.V[1 * 3 + c] * dv[1] + pm.V[2 * 3 + c] * dv[2];
#pragma unroll
            for (int w = 0; w < NV; w++) {
                const HT dw[3] = {(HT)d[w][0], (HT)d[w][1], (HT)d[w][2]};
                HT dhw[3];
#pragma unroll
                for (int c = 0; c < 3; c++) dhw[c] = pm.V[0 * 3 + c] * dw[0] + pm.V[1 * 3 + c] * dw[1] + pm.V[2 * 3 + c] * dw[2];
                HT* b = blk + w * 9;
                HT uv[3], uw[3];
#define SORS_TF(M, I, JJ)                                      \
    if (pm.lt[M] < HT(0)) {                                    \
        tf_vec<HT, I, JJ>(pm.U, dhv, HT(-1), uv);              \
        tf_vec<HT, I, JJ>(pm.U, dhw, HT(-1), uw);              \
        add_outer(b, -pm.lt[M] * wv, uv, uw);                  \
    }                                                          \
    if (pm.lf[M] < HT(0)) {                                    \
        tf_vec<HT, I, JJ>(pm.U, dhv, HT(1), uv);               \
        tf_vec<HT, I, JJ>(pm.U, dhw, HT(1), uw);               \
        add_outer(b, -pm.lf[M] * wv, uv, uw);                  \
    }
                SORS_TF(0, 0, 1)
                SORS_TF(1, 0, 2)
                SORS_TF(2, 1, 2)
#undef SORS_TF
#define SORS_SC(M)                                             \
    if (pm.ls[M] < HT(0)) {                                    \
        sc_vec<HT, M>(pm.U, pm.Y, dhv, uv);                    \
        sc_vec<HT, M>(pm.U, pm.Y, dhw, uw);                    \
        add_outer(b, -pm.ls[M] * wv, uv, uw);                  \
    }
                SORS_SC(0)
                SORS_SC(1)
                SORS_SC(2)
#undef SORS_SC
            }
        }
    }
    return true;
}

// ---------------------------------------------------------------------------
// Stable Neo-Hookean (cpp/src/energies/stableNeoHookean.cpp, after Smith et al.
// 2018): Psi = mu/2 (I_C - 3) + lam/2 (J - alpha)^2 - mu/2 log(I_C + 1), with
// the reparameterised mu = 4/3 mu_L, lam = lam_L + 5/8 mu, alpha = 1 + 3/4 mu/lam
// (stableNeoHookean.cpp:10-15; mu and lam arrive already reparameterised).
// P = mu' F + c2 F^-T with mu' = mu (1 - 1/(I_C+1)), c2 = lam (J - alpha) J;
// dP/dF = mu' I + c1 g g^T + c2 M + c4 f f^T (g = vec F^-T, f = vec F,
// M = d F^-T / dF), c1 = lam (2J - alpha) J, c4 = 2 mu / (I_C+1)^2
// (stableNeoHookean.cpp:90-135).  It stays finite for inverted elements.
// In the rotation-variant SVD frame the twist / flip eigenvalues of pair (i,j)
// are mu' +- (c2/J) s_k and the stretch block is
// S_ij = mu' d_ij + c1/(s_i s_j) + c4 s_i s_j - c2 d_ij / s_i^2.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void snh_modes(const T* F, T J, T IC, T mu, T lam, T alpha, NhModes<T>& pm) {
    T s[3];
    svd3_rv(F, pm.U, s, pm.V);
    const T mup = mu * (T(1) - T(1) / (IC + T(1)));
    const T c2 = lam * (J - alpha) * J;
    const T c1 = lam * (T(2) * J - alpha) * J;
    const T c4 = T(2) * mu / ((IC + T(1)) * (IC + T(1)));
    const T cj = c2 / J;
    pm.lt[0] = mup + cj * s[2]; pm.lt[1] = mup + cj * s[1]; pm.lt[2] = mup + cj * s[0];
    pm.lf[0] = mup - cj * s[2]; pm.lf[1] = mup - cj * s[1]; pm.lf[2] = mup - cj * s[0];
    T S[9];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++)
            S[i * 3 + j] = c1 / (s[i] * s[j]) + c4 * s[i] * s[j] + ((i == j) ? mup - c2 / (s[i] * s[i]) : T(0));
    sym3_eig(S, pm.ls, pm.Y);
    pm.any = false;
#pragma unroll
    for (int m = 0; m < 3; m++) pm.any |= (pm.lt[m] < T(0)) | (pm.lf[m] < T(0)) | (pm.ls[m] < T(0));
}

// Row v of one quadrature point for the stable Neo-Hookean energy (same
// contract as nh_qp_row); returns false only for a degenerate F (J == 0).
template <typename HT, int NV, bool HESS>
__device__ __forceinline__ bool snh_qp_row(const double (&d)[NV][3], const double (&x)[NV][3], const double (&dvd)[3],
                                           double wV, double mu, double lam, bool project, double* g,
                                           HT (&blk)[NV * 9]) {
    double F[9];
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
            double acc = 0.0;
#pragma unroll
            for (int w = 0; w < NV; w++) acc += x[w][r] * d[w][c];
            F[r * 3 + c] = acc;
        }
    double C[9];
    cof3(F, C);
    const double J = F[0] * C[0] + F[1] * C[1] + F[2] * C[2];
    if (J == 0.0) return false;
    double IC = 0.0;
#pragma unroll
    for (int k = 0; k < 9; k++) IC += F[k] * F[k];
    const double alpha = 1.0 + 0.75 * mu / lam;
    const double iJ = 1.0 / J;
    double G[9];
#pragma unroll
    for (int k = 0; k < 9; k++) G[k] = C[k] * iJ;
    const double mup = mu * (1.0 - 1.0 / (IC + 1.0));
    const double c2 = lam * (J - alpha) * J;
#pragma unroll
    for (int r = 0; r < 3; r++) {
        double pr = 0.0;
#pragma unroll
        for (int c = 0; c < 3; c++) pr += (mup * F[r * 3 + c] + c2 * G[r * 3 + c]) * dvd[c];
        g[r] += wV * pr;
    }
    if (!HESS) return true;
    const double c1 = lam * (2.0 * J - alpha) * J;
    const double c4 = 2.0 * mu / ((IC + 1.0) * (IC + 1.0));
    HT Gh[9], Fh[9];
#pragma unroll
    for (int k = 0; k < 9; k++) { Gh[k] = (HT)G[k]; Fh[k] = (HT)F[k]; }
    const HT dv[3] = {(HT)dvd[0], (HT)dvd[1], (HT)dvd[2]};
    HT av[3], fv[3];
#pragma unroll
    for (int r = 0; r < 3; r++) {
        av[r] = Gh[r * 3 + 0] * dv[0] + Gh[r * 3 + 1] * dv[1] + Gh[r * 3 + 2] * dv[2];
        fv[r] = Fh[r * 3 + 0] * dv[0] + Fh[r * 3 + 1] * dv[1] + Fh[r * 3 + 2] * dv[2];
    }
    const HT hmu = (HT)(wV * mup), h1 = (HT)(wV * c1), h2 = (HT)(wV * c2), h4 = (HT)(wV * c4);
#pragma unroll
    for (int w = 0; w < NV; w++) {
        const HT dw[3] = {(HT)d[w][0], (HT)d[w][1], (HT)d[w][2]};
        HT aw[3], fw[3];
#pragma unroll
        for (int r = 0; r < 3; r++) {
            aw[r] = Gh[r * 3 + 0] * dw[0] + Gh[r * 3 + 1] * dw[1] + Gh[r * 3 + 2] * dw[2];
            fw[r] = Fh[r * 3 + 0] * dw[0] + Fh[r * 3 + 1] * dw[1] + Fh[r * 3 + 2] * dw[2];
        }
        const HT dd = dv[0] * dw[0] + dv[1] * dw[1] + dv[2] * dw[2];
#pragma unroll
        for (int k = 0; k < 3; k++)
#pragma unroll
            for (int l = 0; l < 3; l++) {
                HT val = h1 * av[k] * aw[l] - h2 * aw[k] * av[l] + h4 * fv[k] * fw[l];
                if (k == l) val += hmu * dd;
                blk[w * 9 + k * 3 + l] += val;
            }
    }
    if (project) {
        NhModes<HT> pm;
        snh_modes<HT>(Fh, (HT)J, (HT)IC, (HT)mu, (HT)lam, (HT)alpha, pm);
        if (pm.any) {
            const HT wv = (HT)wV;
            HT dhv[3];
#pragma unroll
            for (int c = 0; c < 3; c++) dhv[c] = pm.V[0 * 3 + c] * dv[0] + pm.V[1 * 3 + c] * dv[1] + pm.V[2 * 3 + c] * dv[2];
#pragma unroll
            for (int w = 0; w < NV; w++) {
                const HT dw[3] = {(HT)d[w][0], (HT)d[w][1], (HT)d[w][2]};
                HT dhw[3];
#pragma unroll
                for (int c = 0; c < 3; c++) dhw[c] = pm.V[0 * 3 + c] * dw[0] + pm.V[1 * 3 + c] * dw[1] + pm.V[2 * 3 + c] * dw[2];
                HT* b = blk + w * 9;
                HT uv[3], uw[3];
#define SORS_TF(M, I, JJ)                                      \
    if (pm.lt[M] < HT(0)) {                                    \
        tf_vec<HT, I, JJ>(pm.U, dhv, HT(-1), uv);              \
        tf_vec<HT, I, JJ>(pm.U, dhw, HT(-1), uw);              \
        add_outer(b, -pm.lt[M] * wv, uv, uw);                  \
    }                                                          \
    if (pm.lf[M] < HT(0)) {                                    \
        tf_vec<HT, I, JJ>(pm.U, dhv, HT(1), uv);               \
        tf_vec<HT, I, JJ>(pm.U, dhw, HT(1), uw);               \
        add_outer(b, -pm.lf[M] * wv, uv, uw);                  \
    }
                SORS_TF(0, 0, 1)
                SORS_TF(1, 0, 2)
                SORS_TF(2, 1, 2)
#undef SORS_TF
#define SORS_SC(M)                                             \
    if (pm.ls[M] < HT(0)) {                                    \
        sc_vec<HT, M>(pm.U, pm.Y, dhv, uv);                    \
        sc_vec<HT, M>(pm.U, pm.Y, dhw, uw);                    \
        add_outer(b, -pm.ls[M] * wv, uv, uw);                  \
    }
                SORS_SC(0)
                SORS_SC(1)
                SORS_SC(2)
#undef SORS_SC
            }
        }
    }
    return true;
}

// Stable Neo-Hookean energy density of one quadrature point (FP64).
__device__ __forceinline__ double snh_qp_energy(const double* F, double mu, double lam) {
    const double J = det3(F);
    double IC = 0.0;
#pragma unroll
    for (int k = 0; k < 9; k++) IC += F[k] * F[k];
    const double alpha = 1.0 + 0.75 * mu / lam;
    return 0.5 * mu * (IC - 3.0) + 0.5 * lam * (J - alpha) * (J - alpha) - 0.5 * mu * log(IC + 1.0);
}

// Energy density x weight of one quadrature point (FP64).
__device__ __forceinline__ double nh_qp_energy(const double* F, double mu, double lam) {
    double J = det3(F);
    double logJ = log(J);
    double tr = 0.0;
#pragma unroll
    for (int k = 0; k < 9; k++) tr += F[k] * F[k];
    return 0.5 * mu * (tr - 3.0) - mu * logJ + 0.5 * lam * logJ * logJ;
}

// ---------------------------------------------------------------------------
// SoftCon fibre term at one quadrature point (cpp/src/energies/softconMuscle.cpp).
// With u = F m = sum_w x_w s_w, s_w = d_w . m, l = |u| and r = (1 - e) / l the
// reference's gradient k (1 - r) u . du/dx (softconMuscle.cpp:56-73) is the
// gradient of k/2 (l - (1 - e))^2; this is the energy used here, with its exact
// Hessian: block (v,w) = k s_v s_w [u u^T / l^2 + c (I - u u^T / l^2)], c = 1 - r,
// clamped at 0 when the Hessian is projected (the u direction always has
// eigenvalue k).  mp = (m_x, m_y, m_z, k).
// ---------------------------------------------------------------------------
template <typename HT, int NV, bool HESS>
__device__ __forceinline__ void muscle_qp_row(const double (&d)[NV][3], const double (&x)[NV][3],
                                              const double (&dvd)[3], double wV, double4 mp, double eact,
                                              bool project, double* g, HT (&blk)[NV * 9]) {
    double s[NV];
    double u[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int w = 0; w < NV; w++) {
        s[w] = d[w][0] * mp.x + d[w][1] * mp.y + d[w][2] * mp.z;
#pragma unroll
        for (int r = 0; r < 3; r++) u[r] += x[w][r] * s[w];
    }
    const double l = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    const double rr = (1.0 - eact) / l;
    const double sv = dvd[0] * mp.x + dvd[1] * mp.y + dvd[2] * mp.z;
    const double gc = wV * mp.w * (1.0 - rr) * sv;
#pragma unroll
    for (int r = 0; r < 3; r++) g[r] += gc * u[r];
    if (!HESS) return;
    double c = 1.0 - rr;
    if (project && c < 0.0) c = 0.0;
    const double il2 = 1.0 / (l * l);
    HT M[9];
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
        for (int q = 0; q < 3; q++) M[k * 3 + q] = (HT)((1.0 - c) * u[k] * u[q] * il2 + (k == q ? c : 0.0));
    const double hv = wV * mp.w * sv;
#pragma unroll
    for (int w = 0; w < NV; w++) {
        const HT f = (HT)(hv * s[w]);
#pragma unroll
        for (int k = 0; k < 9; k++) blk[w * 9 + k] += f * M[k];
    }
}

// Energy density of the fibre term at one quadrature point: k/2 (|F m| - (1 - e))^2.
__device__ __forceinline__ double muscle_qp_energy(const double* F, double4 mp, double eact) {
    double u[3];
#pragma unroll
    for (int r = 0; r < 3; r++) u[r] = F[r * 3 + 0] * mp.x + F[r * 3 + 1] * mp.y + F[r * 3 + 2] * mp.z;
    const double l = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    const double t = l - (1.0 - eact);
    return 0.5 * mp.w * t * t;
}

// ---------------------------------------------------------------------------
// Element geometry: shape gradients d (NV x 3) at a quadrature point and the
// undeformed volume, from the undeformed vertex positions X (NV x 3).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double tet_shape(const double (*X)[3], double (*d)[3]) {
    double Dm[9];
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) Dm[r * 3 + c] = X[c][r] - X[3][r];
    double C[9];
    cof3(Dm, C);
    double det = Dm[0] * C[0] + Dm[1] * C[1] + Dm[2] * C[2];
    double id = 1.0 / det;
    // Dm^-1 = C^T / det; d_w (w < 3) = row w of Dm^-1 = column w of C / det
#pragma unroll
    for (int w = 0; w < 3; w++)
#pragma unroll
        for (int c = 0; c < 3; c++) d[w][c] = C[c * 3 + w] * id;
#pragma unroll
    for (int c = 0; c < 3; c++) d[3][c] = -(d[0][c] + d[1][c] + d[2][c]);
    return fabs(det) / 6.0;
}

__constant__ const double kHexRef[8][3] = {{1., -1., -1.}, {1., 1., -1.}, {-1., 1., -1.}, {-1., -1., -1.},
                                          {1., -1., 1.},  {1., 1., 1.},  {-1., 1., 1.},  {-1., -1., 1.}};

__device__ __forceinline__ double hex_volume(const double (*X)[3]) {
    const int T5[5][4] = {{0, 1, 3, 4}, {1, 2, 3, 6}, {1, 4, 5, 6}, {3, 4, 6, 7}, {1, 3, 4, 6}};
    double v = 0.0;
#pragma unroll
    for (int t = 0; t < 5; t++) v += tet_vol6(X[T5[t][0]], X[T5[t][1]], X[T5[t][2]], X[T5[t][3]]) / 6.0;
    return v;
}

// Shape-function gradients at Gauss point s (hexahedron.cpp:170-207).
__device__ __forceinline__ void hex_shape(const double (*X)[3], int s, double (*d)[3]) {
    const double r3 = 0.57735026918962576451;  // 1/sqrt(3)
    double qx = r3 * kHexRef[s][0], qy = r3 * kHexRef[s][1], qz = r3 * kHexRef[s][2];
    double hg[8][3];
#pragma unroll
    for (int i = 0; i < 8; i++) {
        double xi = kHexRef[i][0], yi = kHexRef[i][1], zi = kHexRef[i][2];
        hg[i][0] = 0.125 * (xi * (1 + yi * qy) * (1 + zi * qz));
        hg[i][1] = 0.125 * (yi * (1 + xi * qx) * (1 + zi * qz));
        hg[i][2] = 0.125 * (zi * (1 + xi * qx) * (1 + yi * qy));
    }
    double hF[9];
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
            double acc = 0.0;
#pragma unroll
            for (int i = 0; i < 8; i++) acc += X[i][r] * hg[i][c];
            hF[r * 3 + c] = acc;
        }
    double C[9];
    cof3(hF, C);
    double id = 1.0 / (hF[0] * C[0] + hF[1] * C[1] + hF[2] * C[2]);
    // G_s = hatG hatF^-1, hatF^-1[k][c] = C[c][k] / det
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int c = 0; c < 3; c++) d[i][c] = (hg[i][0] * C[c * 3 + 0] + hg[i][1] * C[c * 3 + 1] + hg[i][2] * C[c * 3 + 2]) * id;
}

}  // namespace sors
