/*
 * sors_oracle.c -- CPU restatement of the SORS implicit-Euler FEM step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle and the timed CPU
 * baseline ("port" kind).  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / reference arm may load it.  The product path
 * (sors_b200/, libsors_b200.so) never links or calls it.
 *
 * Parity pinning: the reference (SORS, C++17 + Eigen + OpenMP) cannot be built
 * here because its Eigen/OSQP submodules are empty.  This restatement follows
 * the reference sources line by line (citations below, paths relative to the
 * reference project root) and is pinned against the known-answer tests that
 * the reference ships in cpp/src/_test.cpp (see tests/golden/).
 *
 * Everything is FP64, like the reference.  Matrices are row-major.
 * DOF order is 3*vertex + component (cpp/src/energy.cpp:217-222).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_OK 0
#define ORC_ERR_INVERTED 2
#define ORC_ERR_NOT_CONVERGED 3
#define ORC_ERR_SINGULAR 4
#define ORC_ERR_ARG 5

/* material models */
#define ORC_MAT_NEOHOOKEAN 0
#define ORC_MAT_TEST_QUARTIC 1
#define ORC_MAT_STABLE_NEOHOOKEAN 2

/* ------------------------------------------------------------------------- */
/* 3x3 helpers (Eigen's fixed-size determinant()/inverse() use the cofactor   */
/* expansion; restated here).                                                */
/* ------------------------------------------------------------------------- */
static double det3(const double a[9]) {
    return a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
           a[2] * (a[3] * a[7] - a[4] * a[6]);
}

static void inv3(const double a[9], double out[9]) {
    double c00 = a[4] * a[8] - a[5] * a[7];
    double c01 = a[5] * a[6] - a[3] * a[8];
    double c02 = a[3] * a[7] - a[4] * a[6];
    double det = a[0] * c00 + a[1] * c01 + a[2] * c02;
    double id = 1.0 / det;
    out[0] = c00 * id;
    out[1] = (a[2] * a[7] - a[1] * a[8]) * id;
    out[2] = (a[1] * a[5] - a[2] * a[4]) * id;
    out[3] = c01 * id;
    out[4] = (a[0] * a[8] - a[2] * a[6]) * id;
    out[5] = (a[2] * a[3] - a[0] * a[5]) * id;
    out[6] = c02 * id;
    out[7] = (a[1] * a[6] - a[0] * a[7]) * id;
    out[8] = (a[0] * a[4] - a[1] * a[3]) * id;
}

static double tet_abs_volume(const double* a, const double* b, const double* c, const double* d) {
    /* cpp/src/geometries/tetrahedron.cpp:137-149: |ab . (ac x ad)| / 6 */
    double ab[3], ac[3], ad[3];
    for (int k = 0; k < 3; k++) { ab[k] = b[k] - a[k]; ac[k] = c[k] - a[k]; ad[k] = d[k] - a[k]; }
    double cx = ac[1] * ad[2] - ac[2] * ad[1];
    double cy = ac[2] * ad[0] - ac[0] * ad[2];
    double cz = ac[0] * ad[1] - ac[1] * ad[0];
    return fabs(ab[0] * cx + ab[1] * cy + ab[2] * cz) / 6.0;
}

/* ------------------------------------------------------------------------- */
/* Element geometry                                                          */
/* ------------------------------------------------------------------------- */

/* Tetrahedron constructor, cpp/src/geometries/tetrahedron.cpp:5-43.
 * X: 4x3 undeformed vertices.  B: 9x12 dF/dx (row-major), invDm: 3x3. */
int orc_tet_init(const double* X, double* B, double* invDm, double* vol) {
    double Dm[9];
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) Dm[r * 3 + c] = X[c * 3 + r] - X[3 * 3 + r];
    double inv[9];
    inv3(Dm, inv);
    if (invDm) memcpy(invDm, inv, sizeof(inv));
    /* blockMatrices: n = 3i+j -> unit matrix with 1 at (j,i); n = 9,10,11 ->
     * row (n-9) = (-1,-1,-1).  Each is multiplied by invDm and flattened
     * row-major into column n (tetrahedron.cpp:19-37). */
    for (int n = 0; n < 12; n++) {
        double M[9] = {0};
        if (n < 9) {
            int i = n / 3, j = n % 3;
            for (int c = 0; c < 3; c++) M[j * 3 + c] = inv[i * 3 + c];
        } else {
            int j = n - 9;
            for (int c = 0; c < 3; c++) M[j * 3 + c] = -(inv[0 * 3 + c] + inv[1 * 3 + c] + inv[2 * 3 + c]);
        }
        for (int f = 0; f < 9; f++) B[f * 12 + n] = M[f];
    }
    if (vol) *vol = tet_abs_volume(X + 0, X + 3, X + 6, X + 9);
    return ORC_OK;
}

/* Hexahedron constructor, cpp/src/geometries/hexahedron.cpp:106-207.
 * X: 8x3.  G: 8 quadrature points x (8x3) shape-function gradients.
 * B: 8 x (9x24) dF/dx.  vol: 5-tet split volume. */
static const double HEX_REF_NODES[8][3] = {
    {1., -1., -1.}, {1., 1., -1.}, {-1., 1., -1.}, {-1., -1., -1.},
    {1., -1., 1.},  {1., 1., 1.},  {-1., 1., 1.},  {-1., -1., 1.}};
static const int HEX_5TETS[5][4] = {{0, 1, 3, 4}, {1, 2, 3, 6}, {1, 4, 5, 6}, {3, 4, 6, 7}, {1, 3, 4, 6}};

int orc_hex_init(const double* X, double* G, double* B, double* vol) {
    const double s3 = 1.0 / sqrt(3.0);
    for (int s = 0; s < 8; s++) {
        double qx = s3 * HEX_REF_NODES[s][0], qy = s3 * HEX_REF_NODES[s][1], qz = s3 * HEX_REF_NODES[s][2];
        double hatG[8][3];
        for (int i = 0; i < 8; i++) {
            double xi = HEX_REF_NODES[i][0], yi = HEX_REF_NODES[i][1], zi = HEX_REF_NODES[i][2];
            hatG[i][0] = 0.125 * (xi * (1 + yi * qy) * (1 + zi * qz));
            hatG[i][1] = 0.125 * (yi * (1 + xi * qx) * (1 + zi * qz));
            hatG[i][2] = 0.125 * (zi * (1 + xi * qx) * (1 + yi * qy));
        }
        /* hatF = X^T hatG (hexahedron.cpp:203) */
        double hatF[9] = {0};
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) {
                double acc = 0;
                for (int i = 0; i < 8; i++) acc += X[i * 3 + r] * hatG[i][c];
                hatF[r * 3 + c] = acc;
            }
        double hinv[9];
        inv3(hatF, hinv);
        /* G_s = (hatF^{-T} hatG^T)^T = hatG hatF^{-1}  (hexahedron.cpp:204) */
        double* Gs = G ? G + s * 24 : NULL;
        double gl[24];
        for (int i = 0; i < 8; i++)
            for (int c = 0; c < 3; c++) {
                double acc = 0;
                for (int k = 0; k < 3; k++) acc += hatG[i][k] * hinv[k * 3 + c];
                gl[i * 3 + c] = acc;
            }
        if (Gs) memcpy(Gs, gl, sizeof(gl));
        /* dF/dx: column 3i+j = flatten_rowmajor(E(j,i) * G_s) -> row j = G_s row i
         * (hexahedron.cpp:145-167) */
        if (B) {
            double* Bs = B + s * 9 * 24;
            memset(Bs, 0, sizeof(double) * 9 * 24);
            for (int i = 0; i < 8; i++)
                for (int j = 0; j < 3; j++)
                    for (int c = 0; c < 3; c++) Bs[(j * 3 + c) * 24 + (3 * i + j)] = gl[i * 3 + c];
        }
    }
    if (vol) {
        double v = 0;
        for (int t = 0; t < 5; t++)
            v += tet_abs_volume(X + 3 * HEX_5TETS[t][0], X + 3 * HEX_5TETS[t][1], X + 3 * HEX_5TETS[t][2],
                                X + 3 * HEX_5TETS[t][3]);
        *vol = v;
    }
    return ORC_OK;
}

/* ------------------------------------------------------------------------- */
/* Symmetric eigen-decomposition (cyclic Jacobi) for the SPD projection.     */
/* The reference has no projection (cpp/src/energies/neoHookean.cpp:75-128);  */
/* this is the CPU restatement of the projection added on top: eigenvalues   */
/* of the 9x9 dP/dF below zero are clamped to zero.                          */
/* ------------------------------------------------------------------------- */
static void jacobi_eig(int n, double* A /* n*n, destroyed */, double* w, double* V) {
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) V[i * n + j] = (i == j) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0, tot = 0;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                tot += A[i * n + j] * A[i * n + j];
                if (i != j) off += A[i * n + j] * A[i * n + j];
            }
        if (off <= 1e-32 * tot || off == 0.0) break;
        for (int p = 0; p < n - 1; p++)
            for (int q = p + 1; q < n; q++) {
                double apq = A[p * n + q];
                if (apq == 0.0) continue;
                double app = A[p * n + p], aqq = A[q * n + q];
                double theta = (aqq - app) / (2.0 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < n; k++) {
                    double akp = A[k * n + p], akq = A[k * n + q];
                    A[k * n + p] = c * akp - s * akq;
                    A[k * n + q] = s * akp + c * akq;
                }
                for (int k = 0; k < n; k++) {
                    double apk = A[p * n + k], aqk = A[q * n + k];
                    A[p * n + k] = c * apk - s * aqk;
                    A[q * n + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; k++) {
                    double vkp = V[k * n + p], vkq = V[k * n + q];
                    V[k * n + p] = c * vkp - s * vkq;
                    V[k * n + q] = s * vkp + c * vkq;
                }
            }
    }
    for (int i = 0; i < n; i++) w[i] = A[i * n + i];
}

static void project_psd(double* A9 /* 9x9 in/out */) {
    double W[81], w[9], V[81];
    memcpy(W, A9, sizeof(W));
    jacobi_eig(9, W, w, V);
    for (int i = 0; i < 9; i++)
        for (int j = 0; j < 9; j++) {
            double acc = 0;
            for (int k = 0; k < 9; k++) {
                double lk = w[k] > 0 ? w[k] : 0.0;
                acc += V[i * 9 + k] * lk * V[j * 9 + k];
            }
            A9[i * 9 + j] = acc;
        }
}

/* ------------------------------------------------------------------------- */
/* Neo-Hookean material, cpp/src/energies/neoHookean.cpp                     */
/* ------------------------------------------------------------------------- */
static void lame(double E, double nu, double* mu, double* lam) {
    /* neoHookean.cpp:10-11 */
    *lam = (E * nu) / ((1 + nu) * (1 - 2 * nu));
    *mu = E / (2 * (1 + nu));
}

/* stableNeoHookean.cpp:10-15 */
static void lame_material(double E, double nu, int material, double* mu, double* lam) {
    lame(E, nu, mu, lam);
    if (material == ORC_MAT_STABLE_NEOHOOKEAN) {
        *mu *= 4.0 / 3.0;
        *lam += 5.0 / 8.0 * (*mu);
    }
}

/* neoHookean.cpp:14-41 */
static double nh_energy(const double* F, int nqp, double mu, double lam) {
    double e = 0;
    double w = 1.0 / nqp;
    for (int s = 0; s < nqp; s++) {
        const double* f = F + 9 * s;
        double J = det3(f);
        double logJ = log(J);
        double tr = 0;
        for (int k = 0; k < 9; k++) tr += f[k] * f[k];
        e += (0.5 * mu * (tr - 3) - mu * logJ + 0.5 * lam * logJ * logJ) * w;
    }
    return e;
}

/* neoHookean.cpp:43-72; B: nqp x (9 x ncol) */
static void nh_gradient(const double* F, const double* B, int nqp, int ncol, double mu, double lam, double* g) {
    double w = 1.0 / nqp;
    for (int c = 0; c < ncol; c++) g[c] = 0;
    for (int s = 0; s < nqp; s++) {
        const double* f = F + 9 * s;
        double inv[9];
        inv3(f, inv);
        double J = det3(f), logJ = log(J);
        double dEdF[9];
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++)  /* flat(FinvT)[3r+c] = inv[c][r] */
                dEdF[r * 3 + c] = mu * f[r * 3 + c] + (lam * logJ - mu) * inv[c * 3 + r];
        const double* Bs = B + (size_t)s * 9 * ncol;
        for (int c = 0; c < ncol; c++) {
            double acc = 0;
            for (int k = 0; k < 9; k++) acc += dEdF[k] * Bs[k * ncol + c];
            g[c] += acc * w;
        }
    }
}

/* neoHookean.cpp:75-128 (+ optional projection of the 9x9 dP/dF).
 * Returns ORC_ERR_INVERTED when J <= 0 (neoHookean.cpp:98-101). */
static int nh_hessian(const double* F, const double* B, int nqp, int ncol, double mu, double lam, int project,
                      double* H) {
    double w = 1.0 / nqp;
    for (int i = 0; i < ncol * ncol; i++) H[i] = 0;
    double* T = (double*)malloc(sizeof(double) * 9 * ncol);
    int status = ORC_OK;
    for (int s = 0; s < nqp; s++) {
        const double* f = F + 9 * s;
        double inv[9], G[9];
        inv3(f, inv);
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) G[r * 3 + c] = inv[c * 3 + r];
        double J = det3(f);
        if (J <= 0) { status = ORC_ERR_INVERTED; break; }
        double logJ = log(J);
        double cc = lam * logJ - mu;
        /* FinvTGrad column i=3a+b = rowmajor(-G E_ab^T G): entry (p,q) = -G[p][b] G[a][q] */
        double A[81];
        for (int p = 0; p < 3; p++)
            for (int q = 0; q < 3; q++)
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++) {
                        int row = p * 3 + q, col = a * 3 + b;
                        double m = -G[p * 3 + b] * G[a * 3 + q];
                        double v = lam * G[row] * G[col] + cc * m;
                        if (row == col) v += mu;
                        A[row * 9 + col] = v;
                    }
        if (project) project_psd(A);
        const double* Bs = B + (size_t)s * 9 * ncol;
        /* (A^T B)^T B = B^T A B */
        for (int r = 0; r < 9; r++)
            for (int c = 0; c < ncol; c++) {
                double acc = 0;
                for (int k = 0; k < 9; k++) acc += A[k * 9 + r] * Bs[k * ncol + c];
                T[r * ncol + c] = acc;
            }
        for (int i = 0; i < ncol; i++)
            for (int j = 0; j < ncol; j++) {
                double acc = 0;
                for (int k = 0; k < 9; k++) acc += T[k * ncol + i] * Bs[k * ncol + j];
                H[i * ncol + j] += acc * w;
            }
    }
    free(T);
    return status;
}

/* Stable Neo-Hookean, cpp/src/energies/stableNeoHookean.cpp.  mu, lam arrive
 * reparameterised (:10-15): mu_s = 4/3 mu, lam_s = lam + 5/8 mu_s; alpha =
 * 1 + 3/4 mu_s / lam_s.  Energy :18-45, gradient :48-83, Hessian :86-140. */
static double snh_energy(const double* F, int nqp, double mu, double lam) {
    double e = 0, w = 1.0 / nqp, alpha = 1 + 0.75 * mu / lam;
    for (int s = 0; s < nqp; s++) {
        const double* f = F + 9 * s;
        double J = det3(f), IC = 0;
        for (int k = 0; k < 9; k++) IC += f[k] * f[k];
        e += (0.5 * mu * (IC - 3) + 0.5 * lam * (J - alpha) * (J - alpha) - 0.5 * mu * log(IC + 1)) * w;
    }
    return e;
}

static void snh_gradient(const double* F, const double* B, int nqp, int ncol, double mu, double lam, double* g) {
    double w = 1.0 / nqp, alpha = 1 + 0.75 * mu / lam;
    for (int c = 0; c < ncol; c++) g[c] = 0;
    for (int s = 0; s < nqp; s++) {
        const double* f = F + 9 * s;
        double inv[9], J = det3(f), IC = 0;
        inv3(f, inv);
        for (int k = 0; k < 9; k++) IC += f[k] * f[k];
        double dEdF[9];
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++)
                dEdF[r * 3 + c] = mu * f[r * 3 + c] + lam * (J - alpha) * J * inv[c * 3 + r] - mu * f[r * 3 + c] / (IC + 1);
        const double* Bs = B + (size_t)s * 9 * ncol;
        for (int c = 0; c < ncol; c++) {
            double acc = 0;
            for (int k = 0; k < 9; k++) acc += dEdF[k] * Bs[k * ncol + c];
            g[c] += acc * w;
        }
    }
}

static int snh_hessian(const double* F, const double* B, int nqp, int ncol, double mu, double lam, int project,
                       double* H) {
    double w = 1.0 / nqp, alpha = 1 + 0.75 * mu / lam;
    for (int i = 0; i < ncol * ncol; i++) H[i] = 0;
    double* T = (double*)malloc(sizeof(double) * 9 * ncol);
    for (int s = 0; s < nqp; s++) {
        const double* f = F + 9 * s;
        double inv[9], G[9], J = det3(f), IC = 0;
        inv3(f, inv);
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) G[r * 3 + c] = inv[c * 3 + r];
        for (int k = 0; k < 9; k++) IC += f[k] * f[k];
        double A[81];
        for (int p = 0; p < 3; p++)
            for (int q = 0; q < 3; q++)
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++) {
                        int row = p * 3 + q, col = a * 3 + b;
                        double m = -G[p * 3 + b] * G[a * 3 + q];
                        double v = (2 * J - alpha) * lam * J * G[row] * G[col] + lam * (J - alpha) * J * m +
                                   2 * mu * f[row] * f[col] / ((IC + 1) * (IC + 1));
                        if (row == col) v += mu - mu / (IC + 1);
                        A[row * 9 + col] = v;
                    }
        if (project) project_psd(A);
        const double* Bs = B + (size_t)s * 9 * ncol;
        for (int r = 0; r < 9; r++)
            for (int c = 0; c < ncol; c++) {
                double acc = 0;
                for (int k = 0; k < 9; k++) acc += A[k * 9 + r] * Bs[k * ncol + c];
                T[r * ncol + c] = acc;
            }
        for (int i = 0; i < ncol; i++)
            for (int j = 0; j < ncol; j++) {
                double acc = 0;
                for (int k = 0; k < 9; k++) acc += T[k * ncol + i] * Bs[k * ncol + j];
                H[i * ncol + j] += acc * w;
            }
    }
    free(T);
    return ORC_OK;
}

/* ------------------------------------------------------------------------- */
/* Element evaluation (Element::compute_energy, Tetrahedron/Hexahedron::      */
/* compute_gradient/hessian): material value x undeformed volume.            */
/* element.h:40-58, tetrahedron.cpp:99-134, hexahedron.cpp:68-103            */
/* ------------------------------------------------------------------------- */
typedef struct {
    int nv, nqp, ncol;
    double vol;
    double B[8 * 9 * 24]; /* big enough for hex */
    double Dinv[9];       /* tet only */
    double G[8 * 24];     /* hex only */
} ElemGeom;

static void elem_geom(int nv, const double* X, ElemGeom* g) {
    g->nv = nv;
    g->ncol = 3 * nv;
    if (nv == 4) {
        g->nqp = 1;
        orc_tet_init(X, g->B, g->Dinv, &g->vol);
    } else {
        g->nqp = 8;
        orc_hex_init(X, g->G, g->B, &g->vol);
    }
}

static void elem_F(const ElemGeom* g, const double* x, double* F) {
    if (g->nv == 4) {
        /* tetrahedron.cpp:152-169: F = Ds invDm */
        double Ds[9];
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) Ds[r * 3 + c] = x[c * 3 + r] - x[9 + r];
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) {
                double acc = 0;
                for (int k = 0; k < 3; k++) acc += Ds[r * 3 + k] * g->Dinv[k * 3 + c];
                F[r * 3 + c] = acc;
            }
    } else {
        /* hexahedron.cpp:133-142: F_s = X^T G_s */
        for (int s = 0; s < 8; s++)
            for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++) {
                    double acc = 0;
                    for (int i = 0; i < 8; i++) acc += x[i * 3 + r] * g->G[s * 24 + i * 3 + c];
                    F[s * 9 + r * 3 + c] = acc;
                }
    }
}

/* Material models (ORC_MAT_*): 0 = Neo-Hookean; 1 = the reference's mock
 * "Testahedron" quartic energy sum x^2(x^2-0.5) over the element's
 * coordinates, which is not scaled by the volume (cpp/src/_test.cpp:8-66);
 * 2 = stable Neo-Hookean. */

/* SoftCon fibre term of one element (cpp/src/energies/softconMuscle.cpp:12-132):
 * stiffness k, fibre direction m, activation e of the element's muscle group. */
typedef struct { double k, m[3], e; } OrcMuscle;
/* form 0: the reference's energy k/2 |(1-r) F m| = k/2 |l-(1-e)| (:30-31) and its
 * Hessian, whose second term sums d(Fm)_a/dx over a before the outer product
 * (:115-127).  form 1: the energy k/2 (l-(1-e))^2, of which the reference's
 * gradient (:56-73) is the gradient, and its exact Hessian (eigenvalue k along
 * F m, k (1-r) across it; the latter clamped at 0 when projecting). */
#define ORC_MUSCLE_REFERENCE 0
#define ORC_MUSCLE_CONSISTENT 1

/* Adds the fibre term (not yet scaled by the volume) to psi / grad / hess. */
static void muscle_eval(const ElemGeom* g, const double* F, const OrcMuscle* mm, int form, int project,
                        double* psi, double* grad, double* hess) {
    int n = g->ncol;
    double w = 1.0 / g->nqp;
    double Bm[3][24];
    for (int s = 0; s < g->nqp; s++) {
        const double* f = F + 9 * s;
        const double* Bs = g->B + (size_t)s * 9 * n;
        double u[3];
        for (int a = 0; a < 3; a++) u[a] = f[a * 3] * mm->m[0] + f[a * 3 + 1] * mm->m[1] + f[a * 3 + 2] * mm->m[2];
        double l = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        double r = (1 - mm->e) / l;
        /* Bm_a(i) = sum_c m_c dF_ac/dx_i */
        for (int a = 0; a < 3; a++)
            for (int i = 0; i < n; i++) {
                double acc = 0;
                for (int c = 0; c < 3; c++) acc += mm->m[c] * Bs[(a * 3 + c) * n + i];
                Bm[a][i] = acc;
            }
        if (psi) {
            double t = l - (1 - mm->e);
            *psi += (form == ORC_MUSCLE_REFERENCE ? 0.5 * mm->k * fabs(t) : 0.5 * mm->k * t * t) * w;
        }
        if (grad)
            for (int i = 0; i < n; i++)
                grad[i] += mm->k * (1 - r) * (u[0] * Bm[0][i] + u[1] * Bm[1][i] + u[2] * Bm[2][i]) * w;
        if (hess) {
            if (form == ORC_MUSCLE_REFERENCE) {
                for (int i = 0; i < n; i++) {
                    double p1i = u[0] * Bm[0][i] + u[1] * Bm[1][i] + u[2] * Bm[2][i];
                    double p2i = Bm[0][i] + Bm[1][i] + Bm[2][i];
                    for (int j = 0; j < n; j++) {
                        double p1j = u[0] * Bm[0][j] + u[1] * Bm[1][j] + u[2] * Bm[2][j];
                        double p2j = Bm[0][j] + Bm[1][j] + Bm[2][j];
                        hess[i * n + j] += mm->k * (r / (l * l) * p1i * p1j + (1 - r) * p2i * p2j) * w;
                    }
                }
            } else {
                double c = 1 - r;
                if (project && c < 0) c = 0;
                double M[9];
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++) M[a * 3 + b] = (1 - c) * u[a] * u[b] / (l * l) + (a == b ? c : 0.0);
                for (int i = 0; i < n; i++)
                    for (int j = 0; j < n; j++) {
                        double acc = 0;
                        for (int a = 0; a < 3; a++)
                            for (int b = 0; b < 3; b++) acc += M[a * 3 + b] * Bm[a][i] * Bm[b][j];
                        hess[i * n + j] += mm->k * acc * w;
                    }
            }
        }
    }
}

static int elem_eval_geom(const ElemGeom* g, int material, const double* x, double mu, double lam, int project,
                          const OrcMuscle* mm, int mform, double* psi, double* grad, double* hess) {
    int n = g->ncol;
    if (material == ORC_MAT_TEST_QUARTIC) {
        if (psi) {
            double e = 0;
            for (int k = 0; k < n; k++) e += x[k] * x[k] * (x[k] * x[k] - 0.5);
            *psi = e;
        }
        if (grad)
            for (int k = 0; k < n; k++) grad[k] = (2 * x[k] - 1) * (2 * x[k] + 1) * x[k];
        if (hess) {
            for (int k = 0; k < n * n; k++) hess[k] = 0;
            for (int k = 0; k < n; k++) hess[k * n + k] = 12 * x[k] * x[k] - 1;
        }
        return ORC_OK;
    }
    double F[72];
    elem_F(g, x, F);
    int st = ORC_OK;
    if (material == ORC_MAT_STABLE_NEOHOOKEAN) {
        if (psi) *psi = snh_energy(F, g->nqp, mu, lam);
        if (grad) snh_gradient(F, g->B, g->nqp, n, mu, lam, grad);
        if (hess) st = snh_hessian(F, g->B, g->nqp, n, mu, lam, project, hess);
    } else {
        if (psi) *psi = nh_energy(F, g->nqp, mu, lam);
        if (grad) nh_gradient(F, g->B, g->nqp, n, mu, lam, grad);
        if (hess) st = nh_hessian(F, g->B, g->nqp, n, mu, lam, project, hess);
    }
    if (mm) muscle_eval(g, F, mm, mform, project, psi, grad, hess);
    if (psi) *psi *= g->vol;
    if (grad)
        for (int k = 0; k < n; k++) grad[k] *= g->vol;
    if (hess)
        for (int k = 0; k < n * n; k++) hess[k] *= g->vol;
    return st;
}

/* Public element hooks (parity fixtures). */
int orc_elem_eval(int nv, const double* X, const double* x, double youngs, double nu, int project, double* psi,
                  double* grad, double* hess) {
    ElemGeom g;
    elem_geom(nv, X, &g);
    double mu, lam;
    lame(youngs, nu, &mu, &lam);
    return elem_eval_geom(&g, ORC_MAT_NEOHOOKEAN, x, mu, lam, project, NULL, 0, psi, grad, hess);
}

/* Neo-Hookean + SoftCon fibre element (form: ORC_MUSCLE_*). */
int orc_elem_eval_muscle(int nv, const double* X, const double* x, double youngs, double nu, double k,
                         const double* m, double act, int form, int project, double* psi, double* grad,
                         double* hess) {
    ElemGeom g;
    elem_geom(nv, X, &g);
    double mu, lam;
    lame(youngs, nu, &mu, &lam);
    OrcMuscle mm = {k, {m[0], m[1], m[2]}, act};
    return elem_eval_geom(&g, ORC_MAT_NEOHOOKEAN, x, mu, lam, project, &mm, form, psi, grad, hess);
}

/* Element hook with a material model (ORC_MAT_*). */
int orc_elem_eval_material(int nv, const double* X, const double* x, double youngs, double nu, int material,
                           int project, double* psi, double* grad, double* hess) {
    ElemGeom g;
    elem_geom(nv, X, &g);
    double mu, lam;
    lame_material(youngs, nu, material, &mu, &lam);
    return elem_eval_geom(&g, material, x, mu, lam, project, NULL, 0, psi, grad, hess);
}

/* Batched element evaluation over a mesh (OpenMP).  Outputs per element:
 * psi[E], grad[E*3nv], hess[E*(3nv)^2] (any may be NULL). */
int orc_elem_eval_batch(int nv, int ne, const double* Xn, const int32_t* conn, const double* xn,
                        const double* youngs, const double* nu, int project, double* psi, double* grad,
                        double* hess) {
    int n = 3 * nv;
    int status = ORC_OK;
#pragma omp parallel for schedule(static)
    for (int e = 0; e < ne; e++) {
        double X[24], x[24];
        for (int j = 0; j < nv; j++)
            for (int k = 0; k < 3; k++) {
                X[j * 3 + k] = Xn[3 * conn[e * nv + j] + k];
                x[j * 3 + k] = xn[3 * conn[e * nv + j] + k];
            }
        ElemGeom g;
        elem_geom(nv, X, &g);
        double mu, lam;
        lame(youngs[e], nu[e], &mu, &lam);
        int st = elem_eval_geom(&g, ORC_MAT_NEOHOOKEAN, x, mu, lam, project, NULL, 0, psi ? psi + e : NULL,
                                grad ? grad + (size_t)e * n : NULL, hess ? hess + (size_t)e * n * n : NULL);
        if (st != ORC_OK) {
#pragma omp atomic write
            status = st;
        }
    }
    return status;
}

/* Projection hook: A9 in/out (9x9). */
void orc_project_psd9(double* A9) { project_psd(A9); }

/* ------------------------------------------------------------------------- */
/* Sparse matrices: triplets -> CSR with duplicate summation                 */
/* (Eigen::SparseMatrix::setFromTriplets semantics)                          */
/* ------------------------------------------------------------------------- */
typedef struct {
    int n;
    int64_t nnz;
    int64_t* rowptr;
    int32_t* col;
    double* val;
} Csr;

static void csr_free(Csr* m) {
    free(m->rowptr); free(m->col); free(m->val);
    memset(m, 0, sizeof(*m));
}

static int cmp_pair(const void* a, const void* b) {
    const int32_t* x = (const int32_t*)a;
    const int32_t* y = (const int32_t*)b;
    return (x[0] > y[0]) - (x[0] < y[0]);
}

typedef struct { int32_t col; int32_t pad; double v; } ColVal;
static int cmp_colval(const void* a, const void* b) {
    const ColVal* x = (const ColVal*)a;
    const ColVal* y = (const ColVal*)b;
    return (x->col > y->col) - (x->col < y->col);
}

static void csr_from_triplets(int n, int64_t nt, const int32_t* ti, const int32_t* tj, const double* tv, Csr* out) {
    int64_t* cnt = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
    for (int64_t t = 0; t < nt; t++) cnt[ti[t] + 1]++;
    for (int i = 0; i < n; i++) cnt[i + 1] += cnt[i];
    ColVal* buf = (ColVal*)malloc(sizeof(ColVal) * (size_t)(nt ? nt : 1));
    int64_t* pos = (int64_t*)malloc(sizeof(int64_t) * (size_t)n);
    for (int i = 0; i < n; i++) pos[i] = cnt[i];
    for (int64_t t = 0; t < nt; t++) {
        int64_t p = pos[ti[t]]++;
        buf[p].col = tj[t];
        buf[p].v = tv[t];
    }
    out->n = n;
    out->rowptr = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
    int64_t total = 0;
    /* first pass: sort each row and count unique */
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : total)
    for (int i = 0; i < n; i++) {
        int64_t a = cnt[i], b = cnt[i + 1];
        qsort(buf + a, (size_t)(b - a), sizeof(ColVal), cmp_colval);
        int64_t u = 0;
        for (int64_t p = a; p < b; p++)
            if (p == a || buf[p].col != buf[p - 1].col) u++;
        out->rowptr[i + 1] = u;
        total += u;
    }
    for (int i = 0; i < n; i++) out->rowptr[i + 1] += out->rowptr[i];
    out->nnz = out->rowptr[n];
    out->col = (int32_t*)malloc(sizeof(int32_t) * (size_t)(out->nnz ? out->nnz : 1));
    out->val = (double*)malloc(sizeof(double) * (size_t)(out->nnz ? out->nnz : 1));
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < n; i++) {
        int64_t a = cnt[i], b = cnt[i + 1];
        int64_t q = out->rowptr[i] - 1;
        for (int64_t p = a; p < b; p++) {
            if (p == a || buf[p].col != buf[p - 1].col) {
                q++;
                out->col[q] = buf[p].col;
                out->val[q] = buf[p].v;
            } else {
                out->val[q] += buf[p].v;
            }
        }
    }
    free(buf); free(pos); free(cnt);
    (void)cmp_pair;
}

/* ------------------------------------------------------------------------- */
/* Sparse LDL^T (up-looking, elimination-tree based; the published algorithm */
/* of T. A. Davis, "Algorithm 849: A concise sparse Cholesky factorization    */
/* package", ACM TOMS 31(4), 2005).  Stands in for Eigen::SimplicialLDLT,     */
/* which reads the lower triangle of its input (cpp/src/solver.cpp:65,82-84). */
/* Fill-reducing ordering: coordinate nested dissection on the node graph.   */
/* ------------------------------------------------------------------------- */
typedef struct {
    int n;
    int32_t* perm;  /* new -> old */
    int32_t* iperm; /* old -> new */
    int64_t* Lp;
    int32_t* Li;
    double* Lx;
    double* D;
    int32_t* parent;
    int64_t* lnz;
    int analyzed;
} Ldl;

static void ldl_free(Ldl* f) {
    free(f->perm); free(f->iperm); free(f->Lp); free(f->Li); free(f->Lx); free(f->D); free(f->parent); free(f->lnz);
    memset(f, 0, sizeof(*f));
}

/* Symmetric matrix in full CSR, built from the lower triangle of the input:
 * C(i,j) = A(max(i,j), min(i,j)), then permuted: Cp(a,b) = C(perm[a], perm[b]). */
static void sym_lower_permuted(const Csr* A, const int32_t* iperm, Csr* out) {
    int n = A->n;
    int64_t nl = 0;
    for (int i = 0; i < n; i++)
        for (int64_t p = A->rowptr[i]; p < A->rowptr[i + 1]; p++)
            if (A->col[p] <= i) nl++;
    int64_t nt = 2 * nl;
    int32_t* ti = (int32_t*)malloc(sizeof(int32_t) * (size_t)nt);
    int32_t* tj = (int32_t*)malloc(sizeof(int32_t) * (size_t)nt);
    double* tv = (double*)malloc(sizeof(double) * (size_t)nt);
    int64_t t = 0;
    for (int i = 0; i < n; i++)
        for (int64_t p = A->rowptr[i]; p < A->rowptr[i + 1]; p++) {
            int j = A->col[p];
            if (j > i) continue;
            ti[t] = iperm[i]; tj[t] = iperm[j]; tv[t] = A->val[p]; t++;
            if (j != i) { ti[t] = iperm[j]; tj[t] = iperm[i]; tv[t] = A->val[p]; t++; }
        }
    csr_from_triplets(n, t, ti, tj, tv, out);
    free(ti); free(tj); free(tv);
}

static void ldl_symbolic(const Csr* C, Ldl* f) {
    int n = C->n;
    int32_t* flag = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    f->parent = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    f->lnz = (int64_t*)malloc(sizeof(int64_t) * (size_t)n);
    f->Lp = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n + 1));
    for (int k = 0; k < n; k++) {
        f->parent[k] = -1;
        flag[k] = k;
        f->lnz[k] = 0;
        for (int64_t p = C->rowptr[k]; p < C->rowptr[k + 1]; p++) {
            int i = C->col[p];
            if (i < k) {
                for (; flag[i] != k; i = f->parent[i]) {
                    if (f->parent[i] == -1) f->parent[i] = k;
                    f->lnz[i]++;
                    flag[i] = k;
                }
            }
        }
    }
    f->Lp[0] = 0;
    for (int k = 0; k < n; k++) f->Lp[k + 1] = f->Lp[k] + f->lnz[k];
    free(f->Li); free(f->Lx);
    f->Li = (int32_t*)malloc(sizeof(int32_t) * (size_t)(f->Lp[n] ? f->Lp[n] : 1));
    f->Lx = (double*)malloc(sizeof(double) * (size_t)(f->Lp[n] ? f->Lp[n] : 1));
    f->D = (double*)malloc(sizeof(double) * (size_t)n);
    free(flag);
    f->analyzed = 1;
}

static int ldl_numeric(const Csr* C, Ldl* f) {
    int n = C->n;
    double* Y = (double*)calloc((size_t)n, sizeof(double));
    int32_t* pattern = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int32_t* flag = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int st = ORC_OK;
    for (int k = 0; k < n; k++) {
        Y[k] = 0.0;
        int top = n;
        flag[k] = k;
        f->lnz[k] = 0;
        for (int64_t p = C->rowptr[k]; p < C->rowptr[k + 1]; p++) {
            int i = C->col[p];
            if (i > k) continue;
            Y[i] += C->val[p];
            int len = 0;
            for (; flag[i] != k; i = f->parent[i]) {
                pattern[len++] = i;
                flag[i] = k;
            }
            while (len > 0) pattern[--top] = pattern[--len];
        }
        f->D[k] = Y[k];
        Y[k] = 0.0;
        for (; top < n; top++) {
            int i = pattern[top];
            double yi = Y[i];
            Y[i] = 0.0;
            int64_t p2 = f->Lp[i] + f->lnz[i];
            for (int64_t p = f->Lp[i]; p < p2; p++) Y[f->Li[p]] -= f->Lx[p] * yi;
            double lki = yi / f->D[i];
            f->D[k] -= lki * yi;
            f->Li[p2] = k;
            f->Lx[p2] = lki;
            f->lnz[i]++;
        }
        if (f->D[k] == 0.0) { st = ORC_ERR_SINGULAR; break; }
    }
    free(Y); free(pattern); free(flag);
    return st;
}

static void ldl_solve(const Ldl* f, double* x /* in: b (original order), out: solution */) {
    int n = f->n;
    double* y = (double*)malloc(sizeof(double) * (size_t)n);
    for (int k = 0; k < n; k++) y[k] = x[f->perm[k]];
    for (int j = 0; j < n; j++)
        for (int64_t p = f->Lp[j]; p < f->Lp[j + 1]; p++) y[f->Li[p]] -= f->Lx[p] * y[j];
    for (int j = 0; j < n; j++) y[j] /= f->D[j];
    for (int j = n - 1; j >= 0; j--)
        for (int64_t p = f->Lp[j]; p < f->Lp[j + 1]; p++) y[j] -= f->Lx[p] * y[f->Li[p]];
    for (int k = 0; k < n; k++) x[f->perm[k]] = y[k];
    free(y);
}

/* Nested dissection on the node graph by coordinate bisection. */
typedef struct {
    const int64_t* adjp;
    const int32_t* adj;
    const double* X;
    int32_t* mark;   /* partition labels */
    int32_t* out;
    int nout;
} NdCtx;

static int cmp_key_idx(const void* a, const void* b) {
    const double* x = (const double*)a;
    const double* y = (const double*)b;
    return (x[0] > y[0]) - (x[0] < y[0]);
}

static void nd_recurse(NdCtx* c, int32_t* nodes, int n, int label) {
    if (n <= 96) {
        for (int i = 0; i < n; i++) c->out[c->nout++] = nodes[i];
        return;
    }
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int i = 0; i < n; i++)
        for (int k = 0; k < 3; k++) {
            double v = c->X[3 * nodes[i] + k];
            if (v < lo[k]) lo[k] = v;
            if (v > hi[k]) hi[k] = v;
        }
    int ax = 0;
    for (int k = 1; k < 3; k++)
        if (hi[k] - lo[k] > hi[ax] - lo[ax]) ax = k;
    double* key = (double*)malloc(sizeof(double) * 2 * (size_t)n);
    for (int i = 0; i < n; i++) { key[2 * i] = c->X[3 * nodes[i] + ax]; key[2 * i + 1] = (double)nodes[i]; }
    qsort(key, (size_t)n, 2 * sizeof(double), cmp_key_idx);
    int half = n / 2;
    int la = 2 * label + 1, lb = 2 * label + 2;
    for (int i = 0; i < n; i++) c->mark[(int)key[2 * i + 1]] = (i < half) ? la : lb;
    /* separator: nodes of part A adjacent to part B */
    int32_t* A = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int32_t* Bn = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int32_t* S = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int na = 0, nb = 0, ns = 0;
    for (int i = 0; i < n; i++) {
        int v = (int)key[2 * i + 1];
        if (c->mark[v] == lb) { Bn[nb++] = v; continue; }
        int sep = 0;
        for (int64_t p = c->adjp[v]; p < c->adjp[v + 1]; p++)
            if (c->mark[c->adj[p]] == lb) { sep = 1; break; }
        if (sep) S[ns++] = v; else A[na++] = v;
    }
    for (int i = 0; i < ns; i++) c->mark[S[i]] = -1;
    free(key);
    if (na == 0 || nb == 0) {
        for (int i = 0; i < na; i++) c->out[c->nout++] = A[i];
        for (int i = 0; i < nb; i++) c->out[c->nout++] = Bn[i];
    } else {
        nd_recurse(c, A, na, la);
        nd_recurse(c, Bn, nb, lb);
    }
    for (int i = 0; i < ns; i++) c->out[c->nout++] = S[i];
    free(A); free(Bn); free(S);
}

/* ------------------------------------------------------------------------- */
/* Global system (Energy<3,E>), cpp/src/energy.cpp + cpp/src/integrator.cpp  */
/* ------------------------------------------------------------------------- */
#define SCHEME_BE 0
#define SCHEME_CN 1
#define METHOD_NEWTON 0
#define METHOD_LINESEARCH 1
#define METHOD_FROZEN 2
#define METHOD_SQP 3

typedef struct {
    int nv, N, E, ndof;
    double* X;     /* N*3 */
    int32_t* conn; /* E*nv */
    double* mu;
    double* lam;
    ElemGeom* geom;
    double* mass;  /* 3N, per DOF (energy.cpp:176-189) */
    double grav[3];
    double alpha;
    int scheme, method, project, material;
    int* mask;      /* 3N */
    double* mval;   /* 3N */
    int has_neumann;
    /* pressure force (cpp/src/forces/pressureForce.cpp) */
    int n_faces, face_nv;
    int32_t* faces;
    int32_t* face_group;
    int has_pressure;
    int has_vertex_force;
    /* SoftCon fibre terms: group per element (-1 none), k, direction; activation per group */
    int32_t* mgroup;
    double* mk;
    double* mdir;
    double* mact;
    int n_mgroups, muscle_form;
    /* integrator state (integrator.h:109-117) */
    double* qPrev;
    double* vPrev;
    double* gPrev;
    double* gPrevTmp;
    /* node adjacency for the ordering */
    int64_t* adjp;
    int32_t* adj;
    Ldl ldl;
    int nthreads;
    double settings_dt;
    int settings_substeps;
    int cfl;
    int last_newton_iters;
} OrcSystem;

static void build_node_adjacency(OrcSystem* s) {
    int N = s->N, nv = s->nv;
    int64_t ne = (int64_t)s->E * nv * (nv - 1);
    int32_t* ti = (int32_t*)malloc(sizeof(int32_t) * (size_t)(ne ? ne : 1));
    int32_t* tj = (int32_t*)malloc(sizeof(int32_t) * (size_t)(ne ? ne : 1));
    double* tv = (double*)malloc(sizeof(double) * (size_t)(ne ? ne : 1));
    int64_t t = 0;
    for (int e = 0; e < s->E; e++)
        for (int a = 0; a < nv; a++)
            for (int b = 0; b < nv; b++) {
                if (a == b) continue;
                ti[t] = s->conn[e * nv + a]; tj[t] = s->conn[e * nv + b]; tv[t] = 1.0; t++;
            }
    Csr m;
    csr_from_triplets(N, t, ti, tj, tv, &m);
    s->adjp = m.rowptr;
    s->adj = m.col;
    free(m.val);
    free(ti); free(tj); free(tv);
}

OrcSystem* orc_create(int nv, int N, const double* X, int E, const int32_t* conn, const double* rho,
                      const double* youngs, const double* nu, const double* grav, double alpha, int scheme,
                      int method, int project, int material, int nthreads) {
    OrcSystem* s = (OrcSystem*)calloc(1, sizeof(OrcSystem));
    s->nv = nv; s->N = N; s->E = E; s->ndof = 3 * N;
    s->X = (double*)malloc(sizeof(double) * 3 * (size_t)N);
    memcpy(s->X, X, sizeof(double) * 3 * (size_t)N);
    s->conn = (int32_t*)malloc(sizeof(int32_t) * (size_t)E * nv);
    memcpy(s->conn, conn, sizeof(int32_t) * (size_t)E * nv);
    s->mu = (double*)malloc(sizeof(double) * (size_t)E);
    s->lam = (double*)malloc(sizeof(double) * (size_t)E);
    s->geom = (ElemGeom*)malloc(sizeof(ElemGeom) * (size_t)(E ? E : 1));
    s->mass = (double*)calloc(3 * (size_t)N, sizeof(double));
    s->nthreads = nthreads > 0 ? nthreads : 1;
#ifdef _OPENMP
    omp_set_dynamic(0);
    omp_set_num_threads(s->nthreads);  /* energy.cpp:195-196 */
#endif
#pragma omp parallel for schedule(static)
    for (int e = 0; e < E; e++) {
        double Xe[24];
        for (int j = 0; j < nv; j++)
            for (int k = 0; k < 3; k++) Xe[j * 3 + k] = X[3 * conn[e * nv + j] + k];
        elem_geom(nv, Xe, &s->geom[e]);
        lame_material(youngs[e], nu[e], material, &s->mu[e], &s->lam[e]);
    }
    /* lumped mass, energy.cpp:176-189: element mass rho*V split equally */
    for (int e = 0; e < E; e++) {
        double m = rho[e] * s->geom[e].vol;
        for (int j = 0; j < nv; j++)
            for (int k = 0; k < 3; k++) s->mass[3 * conn[e * nv + j] + k] += m / nv;
    }
    for (int k = 0; k < 3; k++) s->grav[k] = grav[k];
    s->alpha = alpha;
    s->scheme = scheme;
    s->method = method;
    s->project = project;
    s->material = material;
    s->mask = (int*)calloc(3 * (size_t)N, sizeof(int));
    s->mval = (double*)calloc(3 * (size_t)N, sizeof(double));
    /* integrator.h:155-161: qPrev = undeformed vertices, vPrev = gPrev = 0 */
    s->qPrev = (double*)malloc(sizeof(double) * 3 * (size_t)N);
    memcpy(s->qPrev, X, sizeof(double) * 3 * (size_t)N);
    s->vPrev = (double*)calloc(3 * (size_t)N, sizeof(double));
    s->gPrev = (double*)calloc(3 * (size_t)N, sizeof(double));
    s->gPrevTmp = (double*)calloc(3 * (size_t)N, sizeof(double));
    s->settings_substeps = 1;
    build_node_adjacency(s);
    return s;
}

void orc_destroy(OrcSystem* s) {
    free(s->mgroup); free(s->mk); free(s->mdir); free(s->mact);
    if (!s) return;
    free(s->X); free(s->conn); free(s->mu); free(s->lam); free(s->geom); free(s->mass);
    free(s->mask); free(s->mval); free(s->faces); free(s->face_group);
    free(s->qPrev); free(s->vPrev); free(s->gPrev); free(s->gPrevTmp);
    free(s->adjp); free(s->adj);
    ldl_free(&s->ldl);
    free(s);
}

void orc_set_neumann(OrcSystem* s, const int32_t* mask, const double* val) {
    for (int i = 0; i < s->ndof; i++) { s->mask[i] = mask[i]; s->mval[i] = val[i]; }
    s->has_neumann = 1;
}

void orc_set_pressure(OrcSystem* s, int nfaces, int fnv, const int32_t* faces, const int32_t* groups) {
    free(s->faces); free(s->face_group);
    s->n_faces = nfaces; s->face_nv = fnv;
    s->faces = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nfaces * fnv + 1));
    s->face_group = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nfaces + 1));
    memcpy(s->faces, faces, sizeof(int32_t) * (size_t)nfaces * fnv);
    memcpy(s->face_group, groups, sizeof(int32_t) * (size_t)nfaces);
    s->has_pressure = 1;
}

void orc_set_vertex_force(OrcSystem* s, int enabled) { s->has_vertex_force = enabled; }
void orc_set_step_settings(OrcSystem* s, double dt, int substeps, int cfl) {
    s->settings_dt = dt; s->settings_substeps = substeps; s->cfl = cfl;
}
void orc_set_method(OrcSystem* s, int method) { s->method = method; }

void orc_set_initial_deformation(OrcSystem* s, const double* q) {
    memcpy(s->qPrev, q, sizeof(double) * (size_t)s->ndof);
}
void orc_set_initial_velocity(OrcSystem* s, const double* v) {
    memcpy(s->vPrev, v, sizeof(double) * (size_t)s->ndof);
}
void orc_get_state(OrcSystem* s, double* qPrev, double* vPrev, double* gPrev) {
    if (qPrev) memcpy(qPrev, s->qPrev, sizeof(double) * (size_t)s->ndof);
    if (vPrev) memcpy(vPrev, s->vPrev, sizeof(double) * (size_t)s->ndof);
    if (gPrev) memcpy(gPrev, s->gPrev, sizeof(double) * (size_t)s->ndof);
}
void orc_get_mass(OrcSystem* s, double* m) { memcpy(m, s->mass, sizeof(double) * (size_t)s->ndof); }
int orc_last_newton_iters(OrcSystem* s) { return s->last_newton_iters; }

static void gather_elem(const OrcSystem* s, const double* q, int e, double* x) {
    for (int j = 0; j < s->nv; j++)
        for (int k = 0; k < 3; k++) x[j * 3 + k] = q[3 * s->conn[e * s->nv + j] + k];
}

/* The element's fibre term, or NULL (element.h:50-53 looks the activation up
 * under the energy's name, "softconMuscle", by the element's muscle group). */
static const OrcMuscle* elem_muscle(const OrcSystem* s, int e, OrcMuscle* mm) {
    if (!s->mgroup || s->mgroup[e] < 0) return NULL;
    mm->k = s->mk[e];
    for (int c = 0; c < 3; c++) mm->m[c] = s->mdir[3 * (size_t)e + c];
    mm->e = s->mact[s->mgroup[e]];
    return mm;
}

void orc_set_muscles(OrcSystem* s, const int32_t* group, const double* k, const double* dir, int n_groups,
                     int form) {
    free(s->mgroup); free(s->mk); free(s->mdir); free(s->mact);
    s->mgroup = (int32_t*)malloc(sizeof(int32_t) * (size_t)(s->E ? s->E : 1));
    s->mk = (double*)malloc(sizeof(double) * (size_t)(s->E ? s->E : 1));
    s->mdir = (double*)malloc(sizeof(double) * 3 * (size_t)(s->E ? s->E : 1));
    s->mact = (double*)calloc((size_t)(n_groups > 0 ? n_groups : 1), sizeof(double));
    memcpy(s->mgroup, group, sizeof(int32_t) * (size_t)s->E);
    memcpy(s->mk, k, sizeof(double) * (size_t)s->E);
    memcpy(s->mdir, dir, sizeof(double) * 3 * (size_t)s->E);
    s->n_mgroups = n_groups;
    s->muscle_form = form;
}

void orc_set_muscle_act(OrcSystem* s, const double* act) {
    if (s->mact) memcpy(s->mact, act, sizeof(double) * (size_t)s->n_mgroups);
}

/* pressureForce.cpp:14-56.  act: pressure per group. */
static void pressure_force(const OrcSystem* s, const double* q, const double* act, double* f) {
    for (int f_ = 0; f_ < s->n_faces; f_++) {
        const int32_t* face = s->faces + f_ * s->face_nv;
        double area[3] = {0, 0, 0};
        const double* x0 = q + 3 * face[0];
        const double* x1 = q + 3 * face[1];
        const double* x2 = q + 3 * face[2];
        if (s->face_nv == 3) {
            double v1[3], v2[3];
            for (int k = 0; k < 3; k++) { v1[k] = x1[k] - x0[k]; v2[k] = x2[k] - x0[k]; }
            area[0] = 0.5 * (v1[1] * v2[2] - v1[2] * v2[1]);
            area[1] = 0.5 * (v1[2] * v2[0] - v1[0] * v2[2]);
            area[2] = 0.5 * (v1[0] * v2[1] - v1[1] * v2[0]);
        } else {
            const double* x3 = q + 3 * face[3];
            double v1[3], v2[3], v3[3], v4[3];
            for (int k = 0; k < 3; k++) {
                v1[k] = x1[k] - x0[k]; v2[k] = x3[k] - x0[k];
                v3[k] = x3[k] - x2[k]; v4[k] = x1[k] - x2[k];
            }
            area[0] = 0.5 * (v1[1] * v2[2] - v1[2] * v2[1]);
            area[1] = 0.5 * (v1[2] * v2[0] - v1[0] * v2[2]);
            area[2] = 0.5 * (v1[0] * v2[1] - v1[1] * v2[0]);
            area[0] += 0.5 * (v3[1] * v4[2] - v3[2] * v4[1]);
            area[1] += 0.5 * (v3[2] * v4[0] - v3[0] * v4[2]);
            area[2] += 0.5 * (v3[0] * v4[1] - v3[1] * v4[0]);
        }
        double p = act[s->face_group[f_]];
        for (int j = 0; j < s->face_nv; j++)
            for (int k = 0; k < 3; k++) f[3 * face[j] + k] += -p * area[k] / s->face_nv;
    }
}

/* skew(b - a): hessX for triangle vertex with opposite edge (a -> b)
 * (pressureForce.cpp:76-90) */
static void skew_of(const double* a, const double* b, double* M) {
    double d0 = b[0] - a[0], d1 = b[1] - a[1], d2 = b[2] - a[2];
    M[0] = 0;   M[1] = -d2; M[2] = d1;
    M[3] = d2;  M[4] = 0;   M[5] = -d0;
    M[6] = -d1; M[7] = d0;  M[8] = 0;
}

/* pressureForce.cpp:59-186: triplets (row, col, value) appended. */
static int64_t pressure_triplets(const OrcSystem* s, const double* q, const double* act, int32_t* ti, int32_t* tj,
                                 double* tv) {
    int64_t t = 0;
    int fnv = s->face_nv;
    for (int f_ = 0; f_ < s->n_faces; f_++) {
        const int32_t* face = s->faces + f_ * fnv;
        double hess[4][9];
        if (fnv == 3) {
            const double* x0 = q + 3 * face[0];
            const double* x1 = q + 3 * face[1];
            const double* x2 = q + 3 * face[2];
            skew_of(x1, x2, hess[0]);
            skew_of(x2, x0, hess[1]);
            skew_of(x0, x1, hess[2]);
        } else {
            const double* qx0 = q + 3 * face[0];
            const double* qx1 = q + 3 * face[1];
            const double* qx2 = q + 3 * face[2];
            const double* qx3 = q + 3 * face[3];
            /* triangle 1: (x0, x1, x3) -> hess[0], hess[1], hess[3]; hess[2] = 0 */
            skew_of(qx1, qx3, hess[0]);
            skew_of(qx3, qx0, hess[1]);
            for (int k = 0; k < 9; k++) hess[2][k] = 0;
            skew_of(qx0, qx1, hess[3]);
            /* triangle 2: (x2, x3, x1): hessX2 (new) replaces, hessX3/hessX1 accumulate */
            double h2[9], h3[9], h1[9];
            skew_of(qx3, qx1, h2);   /* x0=quadx2,x1=quadx3,x2=quadx1: skew(x2-x1) = skew(qx1-qx3) */
            skew_of(qx1, qx2, h3);   /* skew(x0 - x2) with x0=qx2, x2=qx1 */
            skew_of(qx2, qx3, h1);   /* skew(x1 - x0) with x1=qx3, x0=qx2 */
            for (int k = 0; k < 9; k++) {
                hess[1][k] += h1[k];
                hess[2][k] = h2[k];
                hess[3][k] += h3[k];
            }
        }
        double p = act[s->face_group[f_]];
        for (int j = 0; j < fnv; j++)
            for (int k = 0; k < fnv; k++)
                for (int l = 0; l < 3; l++)
                    for (int m = 0; m < 3; m++) {
                        ti[t] = 3 * face[j] + l;
                        tj[t] = 3 * face[k] + m;
                        tv[t] = p / 6 * hess[k][l * 3 + m];
                        t++;
                    }
    }
    return t;
}

static void external_forces(const OrcSystem* s, const double* q, const double* pressure_act, const double* vforce,
                            double* f) {
    memset(f, 0, sizeof(double) * (size_t)s->ndof);
    if (s->has_pressure && pressure_act) pressure_force(s, q, pressure_act, f);
    if (s->has_vertex_force && vforce)
        for (int i = 0; i < s->ndof; i++) f[i] += vforce[i]; /* vertexForce.cpp:4-8 */
}

/* integrator.cpp:3-42 */
static double integrate_energy(const OrcSystem* s, const double* q, double dt, double eint) {
    int n = s->ndof;
    double grav = 0;
    for (int i = 0; i < n; i++) grav += s->mass[i] * q[i] * s->grav[i % 3];
    grav = -grav;
    if (dt == 0) return grav + eint;
    double ke = 0, de = 0;
    for (int i = 0; i < n; i++) {
        double v, a;
        if (s->scheme == SCHEME_BE) v = (q[i] - s->qPrev[i]) / dt;
        else v = 2 * (q[i] - s->qPrev[i]) / dt - s->vPrev[i];
        a = (v - s->vPrev[i]) / dt;
        ke += s->mass[i] * a * a;
        de += s->mass[i] * v * v;
    }
    if (s->scheme == SCHEME_BE) {
        ke = 0.5 * ke * dt * dt;
        de = 0.5 * s->alpha * dt * de;
    } else {
        ke = 0.5 * ke * dt * dt / 2;
        de = 0.25 * s->alpha * dt * de;
    }
    return ke + grav + de + eint;
}

/* energy.cpp:208-248 */
double orc_energy(OrcSystem* s, const double* q, double dt, const double* pressure_act, const double* vforce) {
    double e = 0;
#pragma omp parallel for reduction(+ : e) schedule(static)
    for (int el = 0; el < s->E; el++) {
        double x[24], psi;
        gather_elem(s, q, el, x);
        OrcMuscle mm;
        elem_eval_geom(&s->geom[el], s->material, x, s->mu[el], s->lam[el], 0, elem_muscle(s, el, &mm),
                       s->muscle_form, &psi, NULL, NULL);
        e += psi;
    }
    if (s->has_pressure || s->has_vertex_force) {
        double* f = (double*)malloc(sizeof(double) * (size_t)s->ndof);
        external_forces(s, q, pressure_act, vforce, f);
        double w = 0;
        for (int i = 0; i < s->ndof; i++) w += f[i] * (q[i] - s->qPrev[i]);
        e += w;
        free(f);
    }
    return integrate_energy(s, q, dt, e);
}

static int sqp_mode(const OrcSystem* s) { return s->method == METHOD_SQP; }

/* energy.cpp:252-308 + integrator.cpp:45-84 */
void orc_gradient(OrcSystem* s, const double* q, double dt, const double* pressure_act, const double* vforce,
                  double* g) {
    int n = s->ndof, nv = s->nv, ncol = 3 * nv;
    memset(g, 0, sizeof(double) * (size_t)n);
    double* ge = (double*)malloc(sizeof(double) * (size_t)s->E * ncol);
#pragma omp parallel for schedule(static)
    for (int el = 0; el < s->E; el++) {
        double x[24];
        gather_elem(s, q, el, x);
        OrcMuscle mm;
        elem_eval_geom(&s->geom[el], s->material, x, s->mu[el], s->lam[el], 0, elem_muscle(s, el, &mm),
                       s->muscle_form, NULL, ge + (size_t)el * ncol, NULL);
    }
    for (int el = 0; el < s->E; el++)
        for (int j = 0; j < nv; j++)
            for (int k = 0; k < 3; k++) {
                int d = 3 * s->conn[el * nv + j] + k;
                if (sqp_mode(s) || s->mask[d] == 0) g[d] += ge[(size_t)el * ncol + 3 * j + k];
            }
    free(ge);
    if (s->has_pressure || s->has_vertex_force) {
        double* f = (double*)malloc(sizeof(double) * (size_t)n);
        external_forces(s, q, pressure_act, vforce, f);
        for (int i = 0; i < n; i++) g[i] -= f[i];
        free(f);
    }
    /* integrate_gradient */
    if (dt == 0) {
        for (int i = 0; i < n; i++) g[i] += -s->mass[i] * s->grav[i % 3];
    } else {
        memcpy(s->gPrevTmp, g, sizeof(double) * (size_t)n);
        for (int i = 0; i < n; i++) {
            double v;
            if (s->scheme == SCHEME_BE) v = (q[i] - s->qPrev[i]) / dt;
            else v = 2 * (q[i] - s->qPrev[i]) / dt - s->vPrev[i];
            double kin = s->mass[i] * ((v - s->vPrev[i]) / dt);
            double damp = s->alpha * s->mass[i] * v;
            double grav = -s->mass[i] * s->grav[i % 3];
            double inert = kin + grav + damp;
            if (s->scheme == SCHEME_BE) g[i] = inert + g[i];
            else g[i] = inert + 0.5 * (g[i] + s->gPrev[i]);
        }
    }
    /* Neumann override only for "minimize_newton" (energy.cpp:299-306) */
    if (s->method == METHOD_NEWTON && s->has_neumann) {
        for (int i = 0; i < n; i++)
            if (s->mask[i] == 1) g[i] = -(s->qPrev[i] + dt * s->mval[i] - q[i]);
    }
}

/* energy.cpp:312-390 + integrator.cpp:87-126.  Returns the CSR in *out. */
static int hessian_csr(OrcSystem* s, const double* q, double dt, const double* pressure_act, Csr* out) {
    int n = s->ndof, nv = s->nv, ncol = 3 * nv;
    int64_t nel = (int64_t)s->E * ncol * ncol;
    int64_t nfaceT = (s->has_pressure && pressure_act) ? (int64_t)s->n_faces * s->face_nv * s->face_nv * 9 : 0;
    int64_t ntot = nel + nfaceT + n;
    int32_t* ti = (int32_t*)malloc(sizeof(int32_t) * (size_t)ntot);
    int32_t* tj = (int32_t*)malloc(sizeof(int32_t) * (size_t)ntot);
    double* tv = (double*)malloc(sizeof(double) * (size_t)ntot);
    int status = ORC_OK;
    double cscale = (s->scheme == SCHEME_CN && dt != 0) ? 0.5 : 1.0;
#pragma omp parallel
    {
        double* He = (double*)malloc(sizeof(double) * (size_t)ncol * ncol);
#pragma omp for schedule(static)
        for (int el = 0; el < s->E; el++) {
            double x[24];
            gather_elem(s, q, el, x);
            OrcMuscle mm;
            int st = elem_eval_geom(&s->geom[el], s->material, x, s->mu[el], s->lam[el], s->project,
                                    elem_muscle(s, el, &mm), s->muscle_form, NULL, NULL, He);
            if (st != ORC_OK) {
#pragma omp atomic write
                status = st;
            }
            int64_t base = (int64_t)el * ncol * ncol;
            for (int j = 0; j < nv; j++)
                for (int k = 0; k < 3; k++)
                    for (int m = 0; m < nv; m++)
                        for (int l = 0; l < 3; l++) {
                            int64_t t = base + (int64_t)(j * 3 + k) * ncol + m * 3 + l;
                            int r = 3 * s->conn[el * nv + j] + k, c = 3 * s->conn[el * nv + m] + l;
                            if (sqp_mode(s) || (s->mask[r] == 0 && s->mask[c] == 0)) {
                                ti[t] = r; tj[t] = c; tv[t] = He[(j * 3 + k) * ncol + m * 3 + l] * cscale;
                            } else {
                                ti[t] = 0; tj[t] = 0; tv[t] = 0.0; /* default Triplet (0,0,0) */
                            }
                        }
        }
        free(He);
    }
    int64_t t = nel;
    if (nfaceT) {
        int64_t t0 = t;
        int64_t nf = pressure_triplets(s, q, pressure_act, ti + t0, tj + t0, tv + t0);
        for (int64_t k = t0; k < t0 + nf; k++) {
            /* only in "minimize_newton" and with both DOFs unmasked (energy.cpp:371) */
            if (!(s->method == METHOD_NEWTON && s->mask[ti[k]] == 0 && s->mask[tj[k]] == 0)) {
                ti[k] = 0; tj[k] = 0; tv[k] = 0.0;
            } else {
                tv[k] *= cscale;
            }
        }
        t += nf;
    }
    /* integrate_hessian: diagonal inertia (integrator.cpp:94-121) */
    if (dt != 0) {
        for (int i = 0; i < n; i++) {
            ti[t] = i; tj[t] = i;
            if (s->scheme == SCHEME_BE) tv[t] = s->mass[i] / (dt * dt) + s->alpha * s->mass[i] / dt;
            else tv[t] = 2 * s->mass[i] / (dt * dt) + 2 * s->alpha * s->mass[i] / dt;
            t++;
        }
    }
    csr_from_triplets(n, t, ti, tj, tv, out);
    free(ti); free(tj); free(tv);
    /* Neumann: diag = 1 (energy.cpp:381-388); coeffRef inserts when absent */
    if (s->method == METHOD_NEWTON && s->has_neumann) {
        for (int i = 0; i < n; i++) {
            if (s->mask[i] != 1) continue;
            int found = 0;
            for (int64_t p = out->rowptr[i]; p < out->rowptr[i + 1]; p++)
                if (out->col[p] == i) { out->val[p] = 1.0; found = 1; break; }
            if (!found) {
                /* rebuild with an inserted diagonal (rare: isolated masked DOF) */
                int64_t nn = out->nnz + 1;
                int32_t* ti2 = (int32_t*)malloc(sizeof(int32_t) * (size_t)nn);
                int32_t* tj2 = (int32_t*)malloc(sizeof(int32_t) * (size_t)nn);
                double* tv2 = (double*)malloc(sizeof(double) * (size_t)nn);
                int64_t u = 0;
                for (int r = 0; r < n; r++)
                    for (int64_t p = out->rowptr[r]; p < out->rowptr[r + 1]; p++) {
                        ti2[u] = r; tj2[u] = out->col[p]; tv2[u] = out->val[p]; u++;
                    }
                ti2[u] = i; tj2[u] = i; tv2[u] = 1.0; u++;
                csr_free(out);
                csr_from_triplets(n, u, ti2, tj2, tv2, out);
                free(ti2); free(tj2); free(tv2);
            }
        }
    }
    return status;
}

/* Dense export of the Hessian (small meshes, tests).  H: ndof x ndof. */
int orc_hessian_dense(OrcSystem* s, const double* q, double dt, const double* pressure_act, double* H) {
    Csr m;
    int st = hessian_csr(s, q, dt, pressure_act, &m);
    int n = s->ndof;
    memset(H, 0, sizeof(double) * (size_t)n * n);
    for (int i = 0; i < n; i++)
        for (int64_t p = m.rowptr[i]; p < m.rowptr[i + 1]; p++) H[(size_t)i * n + m.col[p]] = m.val[p];
    csr_free(&m);
    return st;
}

/* CSR export: call with NULL buffers to get nnz, then with buffers. */
int orc_hessian_csr(OrcSystem* s, const double* q, double dt, const double* pressure_act, int64_t* nnz,
                    int64_t* rowptr, int32_t* col, double* val) {
    Csr m;
    int st = hessian_csr(s, q, dt, pressure_act, &m);
    *nnz = m.nnz;
    if (rowptr) memcpy(rowptr, m.rowptr, sizeof(int64_t) * (size_t)(m.n + 1));
    if (col) memcpy(col, m.col, sizeof(int32_t) * (size_t)m.nnz);
    if (val) memcpy(val, m.val, sizeof(double) * (size_t)m.nnz);
    csr_free(&m);
    return st;
}

static void ensure_ordering(OrcSystem* s) {
    if (s->ldl.perm) return;
    int N = s->N, n = s->ndof;
    NdCtx c;
    c.adjp = s->adjp; c.adj = s->adj; c.X = s->X;
    c.mark = (int32_t*)calloc((size_t)N, sizeof(int32_t));
    c.out = (int32_t*)malloc(sizeof(int32_t) * (size_t)N);
    c.nout = 0;
    int32_t* nodes = (int32_t*)malloc(sizeof(int32_t) * (size_t)N);
    for (int i = 0; i < N; i++) nodes[i] = i;
    nd_recurse(&c, nodes, N, 0);
    s->ldl.n = n;
    s->ldl.perm = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    s->ldl.iperm = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    for (int a = 0; a < N; a++)
        for (int k = 0; k < 3; k++) s->ldl.perm[3 * a + k] = 3 * c.out[a] + k;
    for (int a = 0; a < n; a++) s->ldl.iperm[s->ldl.perm[a]] = a;
    free(c.mark); free(c.out); free(nodes);
}

/* Factor H (lower triangle, as SimplicialLDLT) and solve H dx = rhs. */
static int ldl_factor_solve(OrcSystem* s, const Csr* H, double* rhs_inout) {
    ensure_ordering(s);
    Csr C;
    sym_lower_permuted(H, s->ldl.iperm, &C);
    /* The symbolic analysis depends on the pattern; recompute every call
     * (patterns can change with masks), as SimplicialLDLT::compute does. */
    free(s->ldl.parent); free(s->ldl.lnz); free(s->ldl.Lp); free(s->ldl.D);
    s->ldl.parent = NULL; s->ldl.lnz = NULL; s->ldl.Lp = NULL; s->ldl.D = NULL;
    ldl_symbolic(&C, &s->ldl);
    int st = ldl_numeric(&C, &s->ldl);
    csr_free(&C);
    if (st != ORC_OK) return st;
    ldl_solve(&s->ldl, rhs_inout);
    return ORC_OK;
}

static double norm2(const double* v, int n) {
    double a = 0;
    for (int i = 0; i < n; i++) a += v[i] * v[i];
    return sqrt(a);
}

static int has_nan(const double* v, int n) {
    for (int i = 0; i < n; i++)
        if (v[i] != v[i]) return 1;
    return 0;
}

#define MAX_ITER 100      /* cpp/headers/common.h:21 */
#define DX_TOL 1e-9       /* cpp/headers/common.h:25 */

/* solver.cpp:56-105 */
static int minimize_newton(OrcSystem* s, double* x, double dt, const double* pact, const double* vforce) {
    int n = s->ndof;
    double* g = (double*)malloc(sizeof(double) * (size_t)n);
    int converged = 0, st = ORC_OK, it;
    for (it = 0; it < MAX_ITER; it++) {
        orc_gradient(s, x, dt, pact, vforce, g);
        Csr H;
        st = hessian_csr(s, x, dt, pact, &H);
        if (st != ORC_OK) { csr_free(&H); break; }
        for (int i = 0; i < n; i++) g[i] = -g[i];
        st = ldl_factor_solve(s, &H, g);
        csr_free(&H);
        if (st != ORC_OK) break;
        for (int i = 0; i < n; i++) x[i] += g[i];
        if (has_nan(g, n)) break;
        if (norm2(g, n) < DX_TOL) { converged = 1; break; }
    }
    s->last_newton_iters = it + 1;
    free(g);
    if (st != ORC_OK) return st;
    return converged ? ORC_OK : ORC_ERR_NOT_CONVERGED;
}

/* solver.cpp:201-264 (Armijo backtracking: alpha0 = 1, beta = 0.5, c = 0.1) */
static int minimize_newton_linesearch(OrcSystem* s, double* x, double dt, const double* pact, const double* vforce) {
    int n = s->ndof;
    double* g = (double*)malloc(sizeof(double) * (size_t)n);
    double* dx = (double*)malloc(sizeof(double) * (size_t)n);
    double* xnew = (double*)malloc(sizeof(double) * (size_t)n);
    double* xprev = (double*)malloc(sizeof(double) * (size_t)n);
    memcpy(xprev, x, sizeof(double) * (size_t)n);
    int converged = 0, st = ORC_OK, it;
    for (it = 0; it < MAX_ITER; it++) {
        orc_gradient(s, x, dt, pact, vforce, g);
        Csr H;
        st = hessian_csr(s, x, dt, pact, &H);
        if (st != ORC_OK) { csr_free(&H); break; }
        for (int i = 0; i < n; i++) dx[i] = -g[i];
        st = ldl_factor_solve(s, &H, dx);
        csr_free(&H);
        if (st != ORC_OK) break;
        double alpha = 1.0;
        double gdx = 0;
        for (int i = 0; i < n; i++) gdx += g[i] * dx[i];
        for (int ls = 0; ls < 200; ls++) {
            for (int i = 0; i < n; i++) xnew[i] = x[i] + alpha * dx[i];
            double enew = orc_energy(s, xnew, dt, pact, vforce);
            double e = orc_energy(s, x, dt, pact, vforce);
            if (enew <= e + 0.1 * alpha * gdx) { memcpy(x, xnew, sizeof(double) * (size_t)n); break; }
            alpha *= 0.5;
        }
        for (int i = 0; i < n; i++) { dx[i] = x[i] - xprev[i]; xprev[i] = x[i]; }
        if (has_nan(dx, n)) break;
        if (norm2(dx, n) < DX_TOL) { converged = 1; break; }
    }
    s->last_newton_iters = it + 1;
    free(g); free(dx); free(xnew); free(xprev);
    if (st != ORC_OK) return st;
    return converged ? ORC_OK : ORC_ERR_NOT_CONVERGED;
}

/* solver.cpp:268-296 */
static int minimize_frozen(OrcSystem* s, double* x, double dt, const double* pact, const double* vforce) {
    int n = s->ndof;
    Csr H;
    int st = hessian_csr(s, x, dt, pact, &H);
    if (st != ORC_OK) { csr_free(&H); return st; }
    ensure_ordering(s);
    Csr C;
    sym_lower_permuted(&H, s->ldl.iperm, &C);
    free(s->ldl.parent); free(s->ldl.lnz); free(s->ldl.Lp); free(s->ldl.D);
    ldl_symbolic(&C, &s->ldl);
    st = ldl_numeric(&C, &s->ldl);
    csr_free(&C); csr_free(&H);
    if (st != ORC_OK) return st;
    double* g = (double*)malloc(sizeof(double) * (size_t)n);
    int it;
    for (it = 0; it < MAX_ITER; it++) {
        orc_gradient(s, x, dt, pact, vforce, g);
        for (int i = 0; i < n; i++) g[i] = -g[i];
        ldl_solve(&s->ldl, g);
        for (int i = 0; i < n; i++) x[i] += g[i];
        if (norm2(g, n) < DX_TOL) break;
    }
    s->last_newton_iters = it + 1;
    free(g);
    return ORC_OK; /* the reference only prints on non-convergence */
}

/* integrator.h:86-90 */
void orc_update_state(OrcSystem* s, const double* q, double dt) {
    int n = s->ndof;
    for (int i = 0; i < n; i++) {
        double v;
        if (s->scheme == SCHEME_BE) v = (q[i] - s->qPrev[i]) / dt;
        else v = 2 * (q[i] - s->qPrev[i]) / dt - s->vPrev[i];
        s->vPrev[i] = v;
    }
    memcpy(s->qPrev, q, sizeof(double) * (size_t)n);
    memcpy(s->gPrev, s->gPrevTmp, sizeof(double) * (size_t)n);
}

/* solver.cpp:300-331 */
static double cfl_timestep(OrcSystem* s, const double* q, double dt) {
    double vmax = 0;
    for (int i = 0; i < s->ndof; i++) if (fabs(s->vPrev[i]) > vmax) vmax = fabs(s->vPrev[i]);
    double lmin = -1;
    for (int e = 0; e < s->E; e++) {
        double x[24];
        gather_elem(s, q, e, x);
        for (int i = 0; i < s->nv; i++)
            for (int j = i + 1; j < s->nv; j++) {
                double d0 = x[i * 3] - x[j * 3], d1 = x[i * 3 + 1] - x[j * 3 + 1], d2 = x[i * 3 + 2] - x[j * 3 + 2];
                double l = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
                if (lmin < 0 || l < lmin) lmin = l;
            }
    }
    double dtc = lmin / vmax;
    return dtc < dt ? dtc : dt;
}

/* solver.cpp:5-44.  q in/out. */
int orc_step(OrcSystem* s, double* q, double dt, int substeps, const double* pact, const double* vforce) {
    if (dt == 0.0) dt = s->settings_dt;
    if (substeps == 0) substeps = s->settings_substeps;
    if (s->cfl) {
        double dtc = cfl_timestep(s, q, dt);
        substeps = (int)ceil(dt / dtc);
    }
    double dts = dt / substeps;
    int st = ORC_OK;
    for (int j = 0; j < substeps; j++) {
        if (s->method == METHOD_NEWTON) st = minimize_newton(s, q, dts, pact, vforce);
        else if (s->method == METHOD_LINESEARCH) st = minimize_newton_linesearch(s, q, dts, pact, vforce);
        else if (s->method == METHOD_FROZEN) st = minimize_frozen(s, q, dts, pact, vforce);
        else st = ORC_ERR_ARG;
        if (st != ORC_OK) return st;
        orc_update_state(s, q, dts);
    }
    return st;
}

/* One minimisation without update_state (Solver::minimize_*), q in/out. */
int orc_minimize(OrcSystem* s, double* q, double dt, const double* pact, const double* vforce) {
    if (s->method == METHOD_NEWTON) return minimize_newton(s, q, dt, pact, vforce);
    if (s->method == METHOD_LINESEARCH) return minimize_newton_linesearch(s, q, dt, pact, vforce);
    if (s->method == METHOD_FROZEN) return minimize_frozen(s, q, dt, pact, vforce);
    return ORC_ERR_ARG;
}

/* Linear solve hook for tests: solves H x = b with the oracle's LDL^T. */
int orc_solve_with_hessian(OrcSystem* s, const double* q, double dt, const double* pact, double* b_inout) {
    Csr H;
    int st = hessian_csr(s, q, dt, pact, &H);
    if (st == ORC_OK) st = ldl_factor_solve(s, &H, b_inout);
    csr_free(&H);
    return st;
}

/* Number of nonzeros of the last L factor (diagnostics). */
int64_t orc_last_lnz(OrcSystem* s) { return s->ldl.Lp ? s->ldl.Lp[s->ldl.n] : 0; }

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
