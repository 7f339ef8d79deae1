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

// Rotation-variant SVD of F with det(F) > 0: F = U diag(s) V^T, U, V rotations.
template <typename T>
__device__ void svd3_rv(const T* F, T* U, T* s, T* V) {
    T S[9];
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) S[r * 3 + c] = F[0 * 3 + r] * F[0 * 3 + c] + F[1 * 3 + r] * F[1 * 3 + c] +
                                                   F[2 * 3 + r] * F[2 * 3 + c];
    T w[3];
    sym3_eig(S, w, V);
    // sort descending, permuting columns of V
    int o0 = 0, o1 = 1, o2 = 2, tmp;
    if (w[o0] < w[o1]) { tmp = o0; o0 = o1; o1 = tmp; }
    if (w[o0] < w[o2]) { tmp = o0; o0 = o2; o2 = tmp; }
    if (w[o1] < w[o2]) { tmp = o1; o1 = o2; o2 = tmp; }
    T Vs[9];
#pragma unroll
    for (int r = 0; r < 3; r++) { Vs[r * 3 + 0] = V[r * 3 + o0]; Vs[r * 3 + 1] = V[r * 3 + o1]; Vs[r * 3 + 2] = V[r * 3 + o2]; }
    if (det3(Vs) < T(0)) { Vs[2] = -Vs[2]; Vs[5] = -Vs[5]; Vs[8] = -Vs[8]; }
#pragma unroll
    for (int k = 0; k < 9; k++) V[k] = Vs[k];
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
// Projection data of one quadrature point: the negative modes of d2Psi/dF2
// expressed in the (U, V) frames.
// ---------------------------------------------------------------------------
template <typename T>
struct ProjModes {
    T U[9], V[9];
    int n;          // number of negative modes
    int kind[9];    // 0 twist, 1 flip, 2 scaling
    int pi[9], pj[9];
    T lam[9];
    T y[9][3];      // scaling eigenvector (kind 2)
};

// Returns the negative eigen-modes; J > 0 required.
template <typename T>
__device__ void nh_negative_modes(const T* F, T J, T logJ, T mu, T lam, ProjModes<T>& pm) {
    T s[3];
    svd3_rv(F, pm.U, s, pm.V);
    T c = lam * logJ - mu;
    pm.n = 0;
    const int PI[3] = {0, 0, 1}, PJ[3] = {1, 2, 2}, PK[3] = {2, 1, 0};
#pragma unroll
    for (int m = 0; m < 3; m++) {
        T lt = mu + (c / J) * s[PK[m]];
        T lf = mu - (c / J) * s[PK[m]];
        if (lt < T(0)) { int q = pm.n++; pm.kind[q] = 0; pm.pi[q] = PI[m]; pm.pj[q] = PJ[m]; pm.lam[q] = lt; }
        if (lf < T(0)) { int q = pm.n++; pm.kind[q] = 1; pm.pi[q] = PI[m]; pm.pj[q] = PJ[m]; pm.lam[q] = lf; }
    }
    T S[9];
    T base = mu + lam * (T(1) - logJ);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) S[i * 3 + j] = (i == j) ? mu + base / (s[i] * s[i]) : lam / (s[i] * s[j]);
    T w[3], Y[9];
    sym3_eig(S, w, Y);
#pragma unroll
    for (int m = 0; m < 3; m++)
        if (w[m] < T(0)) {
            int q = pm.n++;
            pm.kind[q] = 2; pm.lam[q] = w[m];
            pm.y[q][0] = Y[0 * 3 + m]; pm.y[q][1] = Y[1 * 3 + m]; pm.y[q][2] = Y[2 * 3 + m];
        }
}

// E_m (V^T d) for mode q, in the U frame.
template <typename T>
__device__ __forceinline__ void mode_apply(const ProjModes<T>& pm, int q, const T* dh, T* y) {
    const T r2 = T(0.70710678118654752440);
    int k = pm.kind[q];
    if (k == 2) {
        y[0] = pm.y[q][0] * dh[0]; y[1] = pm.y[q][1] * dh[1]; y[2] = pm.y[q][2] * dh[2];
    } else {
        int i = pm.pi[q], j = pm.pj[q];
        y[0] = y[1] = y[2] = T(0);
        y[i] = dh[j] * r2;
        y[j] = (k == 0 ? -dh[i] : dh[i]) * r2;
    }
}

// ---------------------------------------------------------------------------
// One quadrature point's contribution to row v of the element Hessian and
// gradient.  d: shape gradients (NV x 3, FP64); x: current positions of the
// element's vertices (NV x 3).  wV = undeformed volume x quadrature weight.
// blk: NV blocks of 9, accumulated (+=).  g: 3 values accumulated (+=).
// Returns false when J <= 0.
// ---------------------------------------------------------------------------
template <typename HT, int NV, bool HESS>
__device__ __forceinline__ bool nh_qp_row(const double (*d)[3], const double (*x)[3], int v, double wV,
                                          double mu, double lam, bool project, double* g, HT* blk) {
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
    double J = F[0] * C[0] + F[1] * C[1] + F[2] * C[2];
    double logJ = log(J);
    double iJ = 1.0 / J;
    double G[9];
#pragma unroll
    for (int k = 0; k < 9; k++) G[k] = C[k] * iJ;
    double cc = lam * logJ - mu;
    // gradient row v: wV * (mu F + c G) d_v
#pragma unroll
    for (int r = 0; r < 3; r++) {
        double pr = 0.0;
#pragma unroll
        for (int c = 0; c < 3; c++) pr += (mu * F[r * 3 + c] + cc * G[r * 3 + c]) * d[v][c];
        g[r] += wV * pr;
    }
    if (!(J > 0.0)) return false;
    if (!HESS) return true;
    // Hessian row blocks in HT precision
    HT Gh[9];
#pragma unroll
    for (int k = 0; k < 9; k++) Gh[k] = (HT)G[k];
    HT dv[3] = {(HT)d[v][0], (HT)d[v][1], (HT)d[v][2]};
    HT av[3];
#pragma unroll
    for (int r = 0; r < 3; r++) av[r] = Gh[r * 3 + 0] * dv[0] + Gh[r * 3 + 1] * dv[1] + Gh[r * 3 + 2] * dv[2];
    HT hmu = (HT)(wV * mu), hlam = (HT)(wV * lam), hc = (HT)(wV * cc);
#pragma unroll
    for (int w = 0; w < NV; w++) {
        HT dw[3] = {(HT)d[w][0], (HT)d[w][1], (HT)d[w][2]};
        HT aw[3];
#pragma unroll
        for (int r = 0; r < 3; r++) aw[r] = Gh[r * 3 + 0] * dw[0] + Gh[r * 3 + 1] * dw[1] + Gh[r * 3 + 2] * dw[2];
        HT dd = dv[0] * dw[0] + dv[1] * dw[1] + dv[2] * dw[2];
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
        ProjModes<HT> pm;
        nh_negative_modes<HT>(Fh, (HT)J, (HT)logJ, (HT)mu, (HT)lam, pm);
        if (pm.n > 0) {
            // dh_w = V^T d_w
            HT dhv[3];
#pragma unroll
            for (int c = 0; c < 3; c++) dhv[c] = pm.V[0 * 3 + c] * dv[0] + pm.V[1 * 3 + c] * dv[1] + pm.V[2 * 3 + c] * dv[2];
            HT wv = (HT)wV;
            for (int w = 0; w < NV; w++) {
                HT dw[3] = {(HT)d[w][0], (HT)d[w][1], (HT)d[w][2]};
                HT dhw[3];
#pragma unroll
                for (int c = 0; c < 3; c++) dhw[c] = pm.V[0 * 3 + c] * dw[0] + pm.V[1 * 3 + c] * dw[1] + pm.V[2 * 3 + c] * dw[2];
                HT Cm[9];
#pragma unroll
                for (int k = 0; k < 9; k++) Cm[k] = HT(0);
                for (int q = 0; q < pm.n; q++) {
                    HT yv[3], yw[3];
                    mode_apply(pm, q, dhv, yv);
                    mode_apply(pm, q, dhw, yw);
                    HT lm = -pm.lam[q] * wv;
#pragma unroll
                    for (int k = 0; k < 3; k++)
#pragma unroll
                        for (int l = 0; l < 3; l++) Cm[k * 3 + l] += lm * yv[k] * yw[l];
                }
                // blk += U Cm U^T
                HT T1[9];
#pragma unroll
                for (int k = 0; k < 3; k++)
#pragma unroll
                    for (int l = 0; l < 3; l++)
                        T1[k * 3 + l] = Cm[k * 3 + 0] * pm.U[l * 3 + 0] + Cm[k * 3 + 1] * pm.U[l * 3 + 1] + Cm[k * 3 + 2] * pm.U[l * 3 + 2];
#pragma unroll
                for (int k = 0; k < 3; k++)
#pragma unroll
                    for (int l = 0; l < 3; l++)
                        blk[w * 9 + k * 3 + l] += pm.U[k * 3 + 0] * T1[0 * 3 + l] + pm.U[k * 3 + 1] * T1[1 * 3 + l] + pm.U[k * 3 + 2] * T1[2 * 3 + l];
            }
        }
    }
    return true;
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
