// kernels.cu -- sm_100a kernels of the implicit-Euler FEM step.
//
// Assembly is row-owner: one warp owns one block-row (node) of the 3x3-block
// CSR Hessian.  Its lanes evaluate the incident (element, local vertex) pairs
// into shared memory, then sum them into the row's slots through the fixed
// slot-item lists built at mesh load.  Every Hessian value and gradient entry
// is written exactly once, by one warp, in a fixed order: no atomics, no
// colouring, bit-reproducible.
//
// Reductions are deterministic two-stage sums (per-block partials in fixed
// grid order, summed by the last block to finish).
#include <cuda_runtime.h>
#include <stdint.h>

#include "fem_math.cuh"
#include "sors_internal.h"

namespace sors {

std::atomic<long long> g_kernel_launches{0};
static inline void counted(int n = 1) { g_kernel_launches.fetch_add(n, std::memory_order_relaxed); }

// ---------------------------------------------------------------------------
// deterministic reductions
// ---------------------------------------------------------------------------
template <int NS>
__device__ __forceinline__ void warp_sum(double (&v)[NS]) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int s = 0; s < NS; s++) v[s] += __shfl_xor_sync(0xffffffffu, v[s], o);
}

// Block sum of NS values (fixed order: lanes, then warps); every thread gets
// the totals.  sh: 32 x NS shared doubles.
template <int NS>
__device__ __forceinline__ void block_sum(double (&v)[NS], double (*sh)[NS]) {
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
    warp_sum<NS>(v);
    if (l == 0)
#pragma unroll
        for (int s = 0; s < NS; s++) sh[w][s] = v[s];
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int s = 0; s < NS; s++) v[s] = (l < nw) ? sh[l][s] : 0.0;
        warp_sum<NS>(v);
        if (l == 0)
#pragma unroll
            for (int s = 0; s < NS; s++) sh[0][s] = v[s];
    }
    __syncthreads();
#pragma unroll
    for (int s = 0; s < NS; s++) v[s] = sh[0][s];
}

// Block sum of v into partials[blockIdx.x*NS + s]; then the last block to
// arrive sums all partials in grid order and returns true with totals in tot.
template <int NS>
__device__ bool reduce_grid(double (&v)[NS], double* partials, unsigned* counter, double (&tot)[NS]) {
    __shared__ double sh[32][NS];
    __shared__ bool am_last;
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
    warp_sum<NS>(v);
    if (l == 0)
#pragma unroll
        for (int s = 0; s < NS; s++) sh[w][s] = v[s];
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int s = 0; s < NS; s++) v[s] = (l < nw) ? sh[l][s] : 0.0;
        warp_sum<NS>(v);
        if (l == 0) {
#pragma unroll
            for (int s = 0; s < NS; s++) partials[blockIdx.x * NS + s] = v[s];
            __threadfence();
            unsigned t = atomicAdd(counter, 1u);
            am_last = (t == gridDim.x - 1);
        }
    }
    __syncthreads();
    if (!am_last) return false;
    __threadfence();
    double a[NS];
#pragma unroll
    for (int s = 0; s < NS; s++) a[s] = 0.0;
    const volatile double* vp = partials;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
#pragma unroll
        for (int s = 0; s < NS; s++) a[s] += vp[b * NS + s];
    warp_sum<NS>(a);
    __syncthreads();
    if (l == 0)
#pragma unroll
        for (int s = 0; s < NS; s++) sh[w][s] = a[s];
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int s = 0; s < NS; s++) a[s] = (l < nw) ? sh[l][s] : 0.0;
        warp_sum<NS>(a);
        if (l == 0)
#pragma unroll
            for (int s = 0; s < NS; s++) sh[0][s] = a[s];
    }
    __syncthreads();
#pragma unroll
    for (int s = 0; s < NS; s++) tot[s] = sh[0][s];
    if (threadIdx.x == 0) *counter = 0u;
    return true;
}

// Largest grid the launchers of this thread use (0: none below the defaults).
// The library sets it from the calling handle's settings on every entry, so
// captured graphs carry the grid of the handle that captured them.
thread_local int t_grid_cap = 0;
void set_grid_cap(int blocks) { t_grid_cap = blocks > 0 ? blocks : 0; }

static inline long long cap_grid(long long b) {
    if (t_grid_cap > 0 && b > t_grid_cap) b = t_grid_cap;
    return b < 1 ? 1 : b;
}

// Streaming multiprocessors of the current device (looked up once per device).
static int sm_count() {
    static std::atomic<int> cache[kMaxDevices];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) dev = 0;
    int n = cache[dev].load(std::memory_order_relaxed);
    if (n <= 0) {
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
        cache[dev].store(n, std::memory_order_relaxed);
    }
    return n;
}

static inline int red_grid(long long n, int per_thread = 1) {
    long long b = (n + (long long)kRedThreads * per_thread - 1) / ((long long)kRedThreads * per_thread);
    if (b < 1) b = 1;
    if (b > kRedBlocks) b = kRedBlocks;
    return (int)cap_grid(b);
}

// ---------------------------------------------------------------------------
// element row evaluation shared by the assembly and the parity hook
// ---------------------------------------------------------------------------
// Tets read their shape gradients d_0..d_2 and volume from tsh (10 doubles per
// element, written once by k_tet_shapes; d_3 = -(d_0 + d_1 + d_2)); hexes
// recompute theirs from the undeformed positions at every quadrature point.
template <typename HT, int NV, bool HESS, bool SNH = false>
__device__ __forceinline__ bool elem_row(const double* __restrict__ Xg, const double* __restrict__ qg,
                                         const int* __restrict__ conn, const double2* __restrict__ mat,
                                         const double* __restrict__ tsh, const MuscleArgs& mus, int e, int v,
                                         int material, bool project, double* g, HT (&blk)[NV * 9]) {
    double X[NV][3], x[NV][3];
#pragma unroll
    for (int w = 0; w < NV; w++) {
        const int n = __ldg(conn + (size_t)e * NV + w);
#pragma unroll
        for (int r = 0; r < 3; r++) {
            if (NV != 4) X[w][r] = __ldg(Xg + 3 * (size_t)n + r);
            x[w][r] = qg[3 * (size_t)n + r];
        }
    }
#pragma unroll
    for (int k = 0; k < NV * 9; k++) blk[k] = HT(0);
    if (material == 1) {
        // quartic test element of the reference (cpp/src/_test.cpp:31-66)
#pragma unroll
        for (int w = 0; w < NV; w++)
            if (w == v) {
#pragma unroll
                for (int r = 0; r < 3; r++) {
                    const double xv = x[w][r];
                    g[r] += (2 * xv - 1) * (2 * xv + 1) * xv;
                    if (HESS) blk[w * 9 + r * 3 + r] = (HT)(12 * xv * xv - 1);
                }
            }
        return true;
    }
    const double2 m = __ldg(mat + e);
    const int grp = mus.group ? __ldg(mus.group + e) : -1;
    double4 mp = make_double4(0.0, 0.0, 0.0, 0.0);
    double eact = 0.0;
    if (grp >= 0) { mp = mus.param[e]; eact = __ldg(mus.act + grp); }
    bool ok = true;
    double d[NV][3];
    double dv[3];
    if (NV == 4) {
        const double2* ts = reinterpret_cast<const double2*>(tsh + (size_t)e * 10);
        double t[10];
#pragma unroll
        for (int k = 0; k < 5; k++) {
            const double2 u = __ldg(ts + k);
            t[2 * k] = u.x; t[2 * k + 1] = u.y;
        }
#pragma unroll
        for (int c = 0; c < 3; c++) {
            d[0][c] = t[c]; d[1][c] = t[3 + c]; d[2][c] = t[6 + c];
            d[3][c] = -(t[c] + t[3 + c] + t[6 + c]);
        }
        const double V = t[9];
#pragma unroll
        for (int w = 0; w < NV; w++)
            if (w == v) { dv[0] = d[w][0]; dv[1] = d[w][1]; dv[2] = d[w][2]; }
        ok = SNH ? snh_qp_row<HT, NV, HESS>(d, x, dv, V, m.x, m.y, project, g, blk)
                 : nh_qp_row<HT, NV, HESS>(d, x, dv, V, m.x, m.y, project, g, blk);
        if (grp >= 0) muscle_qp_row<HT, NV, HESS>(d, x, dv, V, mp, eact, project, g, blk);
    } else {
        const double V = hex_volume((const double(*)[3])X) * 0.125;
        for (int s = 0; s < 8; s++) {
            hex_shape((const double(*)[3])X, s, (double(*)[3])d);
#pragma unroll
            for (int w = 0; w < NV; w++)
                if (w == v) { dv[0] = d[w][0]; dv[1] = d[w][1]; dv[2] = d[w][2]; }
            ok &= SNH ? snh_qp_row<HT, NV, HESS>(d, x, dv, V, m.x, m.y, project, g, blk)
                      : nh_qp_row<HT, NV, HESS>(d, x, dv, V, m.x, m.y, project, g, blk);
            if (grp >= 0) muscle_qp_row<HT, NV, HESS>(d, x, dv, V, mp, eact, project, g, blk);
        }
    }
    return ok;
}

// Energy of element e (element.h:40-58): volume x quadrature mean of the
// Neo-Hookean density plus the fibre term where the element has one.
template <int NV>
__device__ __forceinline__ double elem_energy(const double* __restrict__ Xg, const double* __restrict__ qg,
                                              const int* __restrict__ conn, const double2* __restrict__ mat,
                                              const MuscleArgs& mus, int e, int material) {
    double X[NV][3], x[NV][3];
#pragma unroll
    for (int w = 0; w < NV; w++) {
        const int n = __ldg(conn + (size_t)e * NV + w);
#pragma unroll
        for (int r = 0; r < 3; r++) { X[w][r] = __ldg(Xg + 3 * (size_t)n + r); x[w][r] = qg[3 * (size_t)n + r]; }
    }
    if (material == 1) {
        double out = 0.0;
#pragma unroll
        for (int w = 0; w < NV; w++)
#pragma unroll
            for (int r = 0; r < 3; r++) out += x[w][r] * x[w][r] * (x[w][r] * x[w][r] - 0.5);
        return out;
    }
    const double2 m = __ldg(mat + e);
    const int grp = mus.group ? __ldg(mus.group + e) : -1;
    double4 mp = make_double4(0.0, 0.0, 0.0, 0.0);
    double eact = 0.0;
    if (grp >= 0) { mp = mus.param[e]; eact = __ldg(mus.act + grp); }
    double d[NV][3], F[9];
    const int nqp = (NV == 4) ? 1 : 8;
    const double V = (NV == 4) ? 0.0 : hex_volume((const double(*)[3])X);
    double Vt = 0.0, acc = 0.0;
    for (int s = 0; s < nqp; s++) {
        if (NV == 4) Vt = tet_shape((const double(*)[3])X, (double(*)[3])d);
        else hex_shape((const double(*)[3])X, s, (double(*)[3])d);
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) {
                double t = 0.0;
#pragma unroll
                for (int w = 0; w < NV; w++) t += x[w][r] * d[w][c];
                F[r * 3 + c] = t;
            }
        double qe = material == 2 ? snh_qp_energy(F, m.x, m.y) : nh_qp_energy(F, m.x, m.y);
        if (grp >= 0) qe += muscle_qp_energy(F, mp, eact);
        acc += (NV == 4) ? qe : qe * 0.125;
    }
    return (NV == 4 ? Vt : V) * acc;
}

// Per-element adjoint contractions for the parameter gradients of one step.
// out[e]     = lam_e . g_e^NH: the Neo-Hookean element gradient is proportional
//              to Young's modulus (mu and lambda are, neoHookean.cpp:10-11);
// out[E + e] = lam_e . d g_e^fibre / d e: with g_v = wV k (1 - (1-e)/l) u s_v,
//              d/de gives wV k u s_v / l.
template <int NV>
__global__ void k_adjoint_elem(int E, const double* __restrict__ Xg, const double* __restrict__ qg,
                               const int* __restrict__ conn, const double2* __restrict__ mat, MuscleArgs mus,
                               int material, const double* __restrict__ lam, double* __restrict__ out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    double X[NV][3], x[NV][3], L[NV][3];
#pragma unroll
    for (int w = 0; w < NV; w++) {
        const int n = __ldg(conn + (size_t)e * NV + w);
#pragma unroll
        for (int r = 0; r < 3; r++) {
            X[w][r] = __ldg(Xg + 3 * (size_t)n + r);
            x[w][r] = qg[3 * (size_t)n + r];
            L[w][r] = lam[3 * (size_t)n + r];
        }
    }
    const double2 m = __ldg(mat + e);
    const int grp = mus.group ? __ldg(mus.group + e) : -1;
    double4 mp = make_double4(0.0, 0.0, 0.0, 0.0);
    if (grp >= 0) mp = mus.param[e];
    double d[NV][3];
    const int nqp = (NV == 4) ? 1 : 8;
    const double Vh = (NV == 4) ? 0.0 : hex_volume((const double(*)[3])X) * 0.125;
    double acc_nh = 0.0, acc_mu = 0.0;
    for (int s = 0; s < nqp; s++) {
        double wV;
        if (NV == 4) wV = tet_shape((const double(*)[3])X, (double(*)[3])d);
        else { hex_shape((const double(*)[3])X, s, (double(*)[3])d); wV = Vh; }
        double F[9], LD[9];
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) {
                double t = 0.0, u = 0.0;
#pragma unroll
                for (int w = 0; w < NV; w++) { t += x[w][r] * d[w][c]; u += L[w][r] * d[w][c]; }
                F[r * 3 + c] = t;
                LD[r * 3 + c] = u;
            }
        double C[9];
        cof3(F, C);
        const double J = F[0] * C[0] + F[1] * C[1] + F[2] * C[2];
        // P = a F + b cof(F): Neo-Hookean a = mu, b = (lam log J - mu) / J;
        // stable Neo-Hookean a = mu (1 - 1/(I_C+1)), b = lam (J - alpha)
        double pa, pb;
        if (material == 2) {
            double IC = 0.0;
#pragma unroll
            for (int k = 0; k < 9; k++) IC += F[k] * F[k];
            pa = m.x * (1.0 - 1.0 / (IC + 1.0));
            pb = m.y * (J - (1.0 + 0.75 * m.x / m.y));
        } else {
            pa = m.x;
            pb = (m.y * log(J) - m.x) / J;
        }
        double pd = 0.0;
#pragma unroll
        for (int k = 0; k < 9; k++) pd += (pa * F[k] + pb * C[k]) * LD[k];
        acc_nh += wV * pd;
        if (grp >= 0) {
            double u[3], ls[3];
#pragma unroll
            for (int r = 0; r < 3; r++) {
                u[r] = F[r * 3 + 0] * mp.x + F[r * 3 + 1] * mp.y + F[r * 3 + 2] * mp.z;
                ls[r] = LD[r * 3 + 0] * mp.x + LD[r * 3 + 1] * mp.y + LD[r * 3 + 2] * mp.z;
            }
            const double l = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
            acc_mu += wV * mp.w * (u[0] * ls[0] + u[1] * ls[1] + u[2] * ls[2]) / l;
        }
    }
    out[e] = acc_nh;
    out[(size_t)E + e] = acc_mu;
}

void launch_adjoint_elem(int E, int nv, const double* X, const double* q, const int* conn, const double2* mat,
                         const MuscleArgs& mus, int material, const double* lam, double* out, cudaStream_t st) {
    if (E == 0) return;
    const int threads = 128, blocks = (E + threads - 1) / threads;
    if (nv == 4) k_adjoint_elem<4><<<blocks, threads, 0, st>>>(E, X, q, conn, mat, mus, material, lam, out);
    else k_adjoint_elem<8><<<blocks, threads, 0, st>>>(E, X, q, conn, mat, mus, material, lam, out);
    counted();
}

// Per-tet shape gradients d_0..d_2 (rows of Dm^-1) and undeformed volume,
// computed once at mesh load (tetrahedron.cpp:11-15, :137-149).
__global__ void k_tet_shapes(int E, const double* __restrict__ Xg, const int* __restrict__ conn,
                             double* __restrict__ out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    double X[4][3], d[4][3];
#pragma unroll
    for (int w = 0; w < 4; w++) {
        const int n = conn[(size_t)e * 4 + w];
#pragma unroll
        for (int r = 0; r < 3; r++) X[w][r] = Xg[3 * (size_t)n + r];
    }
    const double V = tet_shape((const double(*)[3])X, (double(*)[3])d);
    double* o = out + (size_t)e * 10;
#pragma unroll
    for (int w = 0; w < 3; w++)
#pragma unroll
        for (int c = 0; c < 3; c++) o[w * 3 + c] = d[w][c];
    o[9] = V;
}

void launch_tet_shapes(int E, const double* X, const int* conn, double* out, cudaStream_t st) {
    if (E == 0) return;
    k_tet_shapes<<<(E + 127) / 128, 128, 0, st>>>(E, X, conn, out);
    counted();
}

// ---------------------------------------------------------------------------
// Row-owner assembly of gradient rows and Hessian block-rows.
// ---------------------------------------------------------------------------
// Row v of tet e written straight into the warp's staging buffer (dst = 4
// blocks of 9): the same terms as elem_row + nh_qp_row / snh_qp_row +
// muscle_qp_row, rearranged for registers: F accumulates while the vertices
// load, and each block is finished (base terms, projection corrections,
// fibre term) and stored before the next is formed.
template <typename HT, bool HESS, bool SNH, bool PROJ>
__device__ __forceinline__ bool tet_row_stage(const AsmArgs<HT>& a, int e, int v, double* g, HT* dst) {
    const double2* ts = reinterpret_cast<const double2*>(a.tshape + (size_t)e * 10);
    double t[10];
#pragma unroll
    for (int k = 0; k < 5; k++) {
        const double2 u = __ldg(ts + k);
        t[2 * k] = u.x; t[2 * k + 1] = u.y;
    }
    // d_w = t[3w .. 3w+2] for w < 3, d_3 = -(d_0 + d_1 + d_2)
    auto dcomp = [&](int w, int c) -> double {
        return w < 3 ? t[3 * w + c] : -(t[c] + t[3 + c] + t[6 + c]);
    };
    const double V = t[9];
    double F[9];
#pragma unroll
    for (int k = 0; k < 9; k++) F[k] = 0.0;
#pragma unroll
    for (int w = 0; w < 4; w++) {
        const int n = __ldg(a.conn + (size_t)e * 4 + w);
#pragma unroll
        for (int r = 0; r < 3; r++) {
            const double xr = a.q[3 * (size_t)n + r];
#pragma unroll
            for (int c = 0; c < 3; c++) F[r * 3 + c] += xr * dcomp(w, c);
        }
    }
    double dv[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        double acc = 0.0;
#pragma unroll
        for (int w = 0; w < 4; w++)
            if (w == v) acc = dcomp(w, c);
        dv[c] = acc;
    }
    const double2 m = __ldg(a.mat + e);
    const int grp = a.mus.group ? __ldg(a.mus.group + e) : -1;
    double C[9];
    cof3(F, C);
    const double J = F[0] * C[0] + F[1] * C[1] + F[2] * C[2];
    // an inverted element still gets the reference's gradient row (NaN or inf
    // as log J and 1/J give); the caller reports it through `ok`
    const double iJ = 1.0 / J;
    double IC = 0.0;
    if (SNH) {
#pragma unroll
        for (int k = 0; k < 9; k++) IC += F[k] * F[k];
    }
    const double alpha = SNH ? 1.0 + 0.75 * m.x / m.y : 0.0;
    const double logJ = SNH ? 0.0 : log(J);
    // P = pa F + pb G with G = C / J
    const double pa = SNH ? m.x * (1.0 - 1.0 / (IC + 1.0)) : m.x;
    const double pb = SNH ? m.y * (J - alpha) * J : (m.y * logJ - m.x);
#pragma unroll
    for (int r = 0; r < 3; r++) {
        double pr = 0.0;
#pragma unroll
        for (int c = 0; c < 3; c++) pr += (pa * F[r * 3 + c] + pb * C[r * 3 + c] * iJ) * dv[c];
        g[r] += V * pr;
    }
    // fibre term (muscle_qp_row)
    double4 mp = make_double4(0.0, 0.0, 0.0, 0.0);
    double mu_u[3] = {0.0, 0.0, 0.0}, mu_c = 0.0, mu_hv = 0.0, mu_il2 = 0.0;
    if (grp >= 0) {
        mp = a.mus.param[e];
        const double eact = __ldg(a.mus.act + grp);
#pragma unroll
        for (int r = 0; r < 3; r++) mu_u[r] = F[r * 3 + 0] * mp.x + F[r * 3 + 1] * mp.y + F[r * 3 + 2] * mp.z;
        const double l = sqrt(mu_u[0] * mu_u[0] + mu_u[1] * mu_u[1] + mu_u[2] * mu_u[2]);
        const double rr = (1.0 - eact) / l;
        const double sv = dv[0] * mp.x + dv[1] * mp.y + dv[2] * mp.z;
        const double gc = V * mp.w * (1.0 - rr) * sv;
#pragma unroll
        for (int r = 0; r < 3; r++) g[r] += gc * mu_u[r];
        mu_c = 1.0 - rr;
        if (PROJ && mu_c < 0.0) mu_c = 0.0;
        mu_il2 = 1.0 / (l * l);
        mu_hv = V * mp.w * sv;
    }
    const bool ok = SNH ? (J != 0.0) : (J > 0.0);
    if (!HESS) return ok;
    if (!ok) {
#pragma unroll
        for (int k = 0; k < 36; k++) dst[k] = HT(0);
        return false;
    }
    HT Gh[9], Fh[9];
#pragma unroll
    for (int k = 0; k < 9; k++) { Gh[k] = (HT)(C[k] * iJ); Fh[k] = (HT)F[k]; }
    const HT dvh[3] = {(HT)dv[0], (HT)dv[1], (HT)dv[2]};
    HT av[3], fv[3];
#pragma unroll
    for (int r = 0; r < 3; r++) {
        av[r] = Gh[r * 3 + 0] * dvh[0] + Gh[r * 3 + 1] * dvh[1] + Gh[r * 3 + 2] * dvh[2];
        fv[r] = Fh[r * 3 + 0] * dvh[0] + Fh[r * 3 + 1] * dvh[1] + Fh[r * 3 + 2] * dvh[2];
    }
    // coefficients: block(v,w)[k][l] = hmu dd d_kl + h1 av_k aw_l - h2 aw_k av_l + h4 fv_k fw_l
    const HT hmu = (HT)(V * pa);
    const HT h1 = (HT)(SNH ? V * m.y * (2.0 * J - alpha) * J : V * m.y);
    const HT h2 = (HT)(V * pb);
    const HT h4 = (HT)(SNH ? V * 2.0 * m.x / ((IC + 1.0) * (IC + 1.0)) : 0.0);
    NhModes<HT> pm;
    HT dhv[3];
    if (PROJ) {
        if (SNH) snh_modes<HT>(Fh, (HT)J, (HT)IC, (HT)m.x, (HT)m.y, (HT)alpha, pm);
        else nh_modes<HT>(Fh, (HT)J, (HT)logJ, (HT)m.x, (HT)m.y, pm);
#pragma unroll
        for (int c = 0; c < 3; c++) dhv[c] = pm.V[0 * 3 + c] * dvh[0] + pm.V[1 * 3 + c] * dvh[1] + pm.V[2 * 3 + c] * dvh[2];
    }
#pragma unroll
    for (int w = 0; w < 4; w++) {
        const HT dw[3] = {(HT)dcomp(w, 0), (HT)dcomp(w, 1), (HT)dcomp(w, 2)};
        HT aw[3], fw[3];
#pragma unroll
        for (int r = 0; r < 3; r++) {
            aw[r] = Gh[r * 3 + 0] * dw[0] + Gh[r * 3 + 1] * dw[1] + Gh[r * 3 + 2] * dw[2];
            fw[r] = Fh[r * 3 + 0] * dw[0] + Fh[r * 3 + 1] * dw[1] + Fh[r * 3 + 2] * dw[2];
        }
        const HT dd = dvh[0] * dw[0] + dvh[1] * dw[1] + dvh[2] * dw[2];
        HT b[9];
#pragma unroll
        for (int k = 0; k < 3; k++)
#pragma unroll
            for (int l = 0; l < 3; l++) {
                HT val = h1 * av[k] * aw[l] - h2 * aw[k] * av[l];
                if (SNH) val += h4 * fv[k] * fw[l];
                if (k == l) val += hmu * dd;
                b[k * 3 + l] = val;
            }
        if (PROJ && pm.any) {
            const HT wv = (HT)V;
            HT dhw[3];
#pragma unroll
            for (int c = 0; c < 3; c++) dhw[c] = pm.V[0 * 3 + c] * dw[0] + pm.V[1 * 3 + c] * dw[1] + pm.V[2 * 3 + c] * dw[2];
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
        if (grp >= 0) {
            const double sw = dcomp(w, 0) * mp.x + dcomp(w, 1) * mp.y + dcomp(w, 2) * mp.z;
            const HT f = (HT)(mu_hv * sw);
#pragma unroll
            for (int k = 0; k < 3; k++)
#pragma unroll
                for (int l = 0; l < 3; l++)
                    b[k * 3 + l] += f * (HT)((1.0 - mu_c) * mu_u[k] * mu_u[l] * mu_il2 + (k == l ? mu_c : 0.0));
        }
#pragma unroll
        for (int k = 0; k < 9; k++) dst[w * 9 + k] = b[k];
    }
    return true;
}

// Tet rows of the exact Neo-Hookean Hessian: FP32 at 3 blocks per SM (80
// registers, a few hundred bytes of spills) measured 18 % faster than 2 blocks
// at 128 registers, and FP64 fits 2 blocks (128 registers, no spills; 156
// unbounded); the projected and stable variants spill more and keep 2 / 1.
template <typename HT, int NV, bool SNH, bool PROJ>
__global__ void __launch_bounds__(256, NV == 4 ? (sizeof(HT) == 4 ? ((SNH || PROJ) ? 2 : 3) : ((SNH || PROJ) ? 1 : 2)) : 1)
    k_assemble(AsmArgs<HT> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    HT* stage = reinterpret_cast<HT*>(smem_raw) + (size_t)warp * a.stage_per_warp;
    for (int row = blockIdx.x * wpb + warp; row < a.N; row += gridDim.x * wpb) {
        const int p0 = a.pair_ptr[row];
        const int np = a.pair_ptr[row + 1] - p0;
        double g[3] = {0.0, 0.0, 0.0};
        bool ok = true;
        for (int k = lane; k < np; k += 32) {
            const int ev = __ldg(a.pair_ev + p0 + k);
            const int e = ev >> 3, v = ev & 7;
            if (NV == 4) {
                HT* dst = stage + (size_t)k * 36;
                if (a.material == 1) {
                    // quartic test element of the reference (cpp/src/_test.cpp:31-66)
#pragma unroll
                    for (int t = 0; t < 36; t++) dst[t] = HT(0);
                    const int n = __ldg(a.conn + (size_t)e * 4 + v);
#pragma unroll
                    for (int r = 0; r < 3; r++) {
                        const double xv = a.q[3 * (size_t)n + r];
                        g[r] += (2 * xv - 1) * (2 * xv + 1) * xv;
                        dst[v * 9 + r * 3 + r] = (HT)(12 * xv * xv - 1);
                    }
                } else if (a.want_hess) {
                    ok &= (PROJ ? tet_row_stage<HT, true, SNH, true>(a, e, v, g, dst)
                                : tet_row_stage<HT, true, SNH, false>(a, e, v, g, dst));
                } else {
                    ok &= tet_row_stage<HT, false, SNH, false>(a, e, v, g, dst);
                }
                continue;
            }
            HT blk[NV * 9];
            if (a.want_hess) {
                ok &= elem_row<HT, NV, true, SNH>(a.X, a.q, a.conn, a.mat, a.tshape, a.mus, e, v, a.material, a.project != 0, g, blk);
                HT* dst = stage + (size_t)k * NV * 9;
#pragma unroll
                for (int t = 0; t < NV * 9; t++) dst[t] = blk[t];
            } else {
                ok &= elem_row<HT, NV, false, SNH>(a.X, a.q, a.conn, a.mat, a.tshape, a.mus, e, v, a.material, false, g, blk);
            }
        }
        if (!ok) atomicOr(a.status, kFlagInverted);
        warp_sum<3>(g);
        const unsigned mrow = a.node_mask[row];
        if (lane < 3) {
            double gv = (lane == 0) ? g[0] : (lane == 1 ? g[1] : g[2]);
            if (a.apply_mask && ((mrow >> lane) & 1u)) gv = 0.0;
            a.g_int[3 * (size_t)row + lane] = gv;
        }
        if (a.want_hess) {
            __syncwarp();
            const int b0 = a.row_ptr[row];
            const int nb = a.row_ptr[row + 1] - b0;
            const double md = a.inertia_coef * a.mass[row];
            for (int t = lane; t < nb * 9; t += 32) {
                const int s = t / 9, rc = t - s * 9, r = rc / 3, c = rc - r * 3;
                const int bg = b0 + s;
                const int i0 = __ldg(a.slot_item_ptr + bg), i1 = __ldg(a.slot_item_ptr + bg + 1);
                HT acc = HT(0);
                for (int it = i0; it < i1; ++it) acc += stage[(int)__ldg(a.slot_items + it) * 9 + rc];
                const int j = __ldg(a.col + bg);
                const unsigned mcol = a.node_mask[j];
                const bool rmask = (mrow >> r) & 1u;
                double val = (double)acc * a.hscale;
                if (a.apply_mask && (rmask || ((mcol >> c) & 1u))) val = 0.0;
                if (j == row && r == c) {
                    val += md;
                    if (a.neumann_override && rmask) val = 1.0;
                }
                a.H[hval(bg, rc, a.nnzb)] = (HT)val;
            }
            __syncwarp();
        }
    }
}

// ---------------------------------------------------------------------------
// Element-owner tet assembly over node chunks (exact Neo-Hookean and stable
// Neo-Hookean Hessians).  One block per chunk of nearby nodes:
//   A. each element incident to the chunk is evaluated once (F, cofactor, J,
//      log J and P in FP64, as tet_row_stage) into a Hessian generator in
//      shared memory, and V P d_v is stored for every vertex v the chunk owns;
//   B. one thread per CSR block of the chunk's rows sums the block's items in
//      their fixed order, expanding block (v, w) of element e from its
//      generator:  hmu (d_v . d_w) I + h1 a_v a_w^T - h2 a_w a_v^T
//      [+ h4 f_v f_w^T], a_v = F^-T d_v, f_v = F d_v (the same terms, in the
//      same Hessian type, as the row-owner kernel), and writes it once;
//   C. one thread per row sums its gradient pairs in their fixed order.
// No atomics, a fixed order everywhere: bit-reproducible.
// ---------------------------------------------------------------------------
constexpr int kChunkThreads = 256;

// generator fields per element: hmu, h1, h2, a_v (12), d_v . d_w (10, v <= w);
// stable Neo-Hookean adds h4 and f_v (12)
template <bool SNH>
struct ChunkGen {
    static constexpr int kA = 3, kDD = 15, kH4 = 25, kF = 26;
    static constexpr int kFields = SNH ? 38 : 25;
};

__device__ __forceinline__ int dd_index(int v, int w) {
    // v <= w: (0,0..3) -> 0..3, (1,1..3) -> 4..6, (2,2..3) -> 7..8, (3,3) -> 9
    return v * 4 - (v * (v - 1)) / 2 + (w - v);
}

ChunkLimits chunk_limits(int hsize, int material) {
    const bool snh = material == 2;
    if (hsize == 4) return snh ? ChunkLimits{64, 384, 1152} : ChunkLimits{64, 512, 1536};
    return snh ? ChunkLimits{32, 192, 576} : ChunkLimits{32, 256, 768};
}

// Shared memory of one chunk block: the gradient pairs (3 doubles per pair),
// the element generators, and the chunk's row table.
size_t chunk_region_bytes(int hsize, int material, int max_pairs) {
    (void)max_pairs;
    const ChunkLimits l = chunk_limits(hsize, material);
    return ((size_t)l.pairs * 3 * sizeof(double) + 15) / 16 * 16;
}

size_t chunk_smem_bytes(int hsize, int material, int max_pairs) {
    const ChunkLimits l = chunk_limits(hsize, material);
    const int nf = material == 2 ? ChunkGen<true>::kFields : ChunkGen<false>::kFields;
    return chunk_region_bytes(hsize, material, max_pairs) + (size_t)nf * l.elems * hsize +
           (size_t)(5 * l.rows + 2) * sizeof(int);
}

// Hessian generator and gradient rows of one tet (the element math of the
// chunked assembly): out.grad(v, r, x) receives V (P d_v)_r for the vertices
// out.wants(v), out.gen(f, x) generator field f.  Returns false for an
// inverted element (J <= 0; J == 0 for stable Neo-Hookean), whose generator is
// zero.
template <typename HT, bool SNH, typename Sink>
__device__ __forceinline__ bool tet_generator(const AsmArgs<HT>& a, int e, bool want_hess, Sink& out) {
    using G = ChunkGen<SNH>;
    const double2* ts = reinterpret_cast<const double2*>(a.tshape + (size_t)e * 10);
    double t[10];
#pragma unroll
    for (int k = 0; k < 5; k++) {
        const double2 u = __ldg(ts + k);
        t[2 * k] = u.x; t[2 * k + 1] = u.y;
    }
    const int4 cn = __ldg(reinterpret_cast<const int4*>(a.conn) + e);
    const int nodes[4] = {cn.x, cn.y, cn.z, cn.w};
    double d[4][3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        d[0][c] = t[c]; d[1][c] = t[3 + c]; d[2][c] = t[6 + c];
        d[3][c] = -(t[c] + t[3 + c] + t[6 + c]);
    }
    const double V = t[9];
    double F[9];
#pragma unroll
    for (int k = 0; k < 9; k++) F[k] = 0.0;
#pragma unroll
    for (int w = 0; w < 4; w++) {
#pragma unroll
        for (int r = 0; r < 3; r++) {
            const double xr = a.q[3 * (size_t)nodes[w] + r];
#pragma unroll
            for (int c = 0; c < 3; c++) F[r * 3 + c] += xr * d[w][c];
        }
    }
    const double2 m = __ldg(a.mat + e);
    double C[9];
    cof3(F, C);
    const double J = F[0] * C[0] + F[1] * C[1] + F[2] * C[2];
    const double iJ = 1.0 / J;
    double IC = 0.0;
    if (SNH) {
#pragma unroll
        for (int k = 0; k < 9; k++) IC += F[k] * F[k];
    }
    const double alpha = SNH ? 1.0 + 0.75 * m.x / m.y : 0.0;
    const double logJ = SNH ? 0.0 : log(J);
    const double pa = SNH ? m.x * (1.0 - 1.0 / (IC + 1.0)) : m.x;
    const double pb = SNH ? m.y * (J - alpha) * J : (m.y * logJ - m.x);
    double P[9];
#pragma unroll
    for (int k = 0; k < 9; k++) P[k] = pa * F[k] + pb * C[k] * iJ;
#pragma unroll
    for (int v = 0; v < 4; v++) {
        if (!out.wants(v)) continue;
#pragma unroll
        for (int r = 0; r < 3; r++) {
            double pr = 0.0;
#pragma unroll
            for (int c = 0; c < 3; c++) pr += P[r * 3 + c] * d[v][c];
            out.grad(v, r, V * pr);
        }
    }
    const bool eok = SNH ? (J != 0.0) : (J > 0.0);
    if (!want_hess) return eok;
    if (!eok) {
#pragma unroll
        for (int f = 0; f < G::kFields; f++) out.gen(f, HT(0));
        return false;
    }
    HT Gh[9], dh[4][3];
#pragma unroll
    for (int k = 0; k < 9; k++) Gh[k] = (HT)(C[k] * iJ);
#pragma unroll
    for (int v = 0; v < 4; v++)
#pragma unroll
        for (int c = 0; c < 3; c++) dh[v][c] = (HT)d[v][c];
    out.gen(0, (HT)(V * pa));
    out.gen(1, (HT)(SNH ? V * m.y * (2.0 * J - alpha) * J : V * m.y));
    out.gen(2, (HT)(V * pb));
#pragma unroll
    for (int v = 0; v < 4; v++)
#pragma unroll
        for (int r = 0; r < 3; r++)
            out.gen((G::kA + v * 3 + r), Gh[r * 3 + 0] * dh[v][0] + Gh[r * 3 + 1] * dh[v][1] + Gh[r * 3 + 2] * dh[v][2]);
#pragma unroll
    for (int v = 0; v < 4; v++)
#pragma unroll
        for (int w = v; w < 4; w++)
            out.gen((G::kDD + dd_index(v, w)), dh[v][0] * dh[w][0] + dh[v][1] * dh[w][1] + dh[v][2] * dh[w][2]);
    if (SNH) {
        out.gen(G::kH4, (HT)(V * 2.0 * m.x / ((IC + 1.0) * (IC + 1.0))));
        HT Fh[9];
#pragma unroll
        for (int k = 0; k < 9; k++) Fh[k] = (HT)F[k];
#pragma unroll
        for (int v = 0; v < 4; v++)
#pragma unroll
            for (int r = 0; r < 3; r++)
                out.gen((G::kF + v * 3 + r), Fh[r * 3 + 0] * dh[v][0] + Fh[r * 3 + 1] * dh[v][1] + Fh[r * 3 + 2] * dh[v][2]);
    }
    return true;
}

template <typename HT>
struct SmemGenSink {
    HT* g;
    int EM, s;
    double* gslot;
    unsigned short slots[4];
    __device__ __forceinline__ bool wants(int v) const { return slots[v] != 0xffff; }
    __device__ __forceinline__ void grad(int v, int r, double x) { gslot[3 * slots[v] + r] = x; }
    __device__ __forceinline__ void gen(int f, HT x) { g[f * EM + s] = x; }
};

template <typename HT>
struct GlobalGenSink {
    HT* rec;
    double* gr;
    __device__ __forceinline__ bool wants(int) const { return true; }
    __device__ __forceinline__ void grad(int v, int r, double x) { gr[3 * v + r] = x; }
    __device__ __forceinline__ void gen(int f, HT x) { rec[f] = x; }
};

// Record stride of the element generators in memory (fields padded to 16 bytes).
template <typename HT, bool SNH>
__host__ __device__ constexpr int chunk_gen_stride() {
    return (ChunkGen<SNH>::kFields * (int)sizeof(HT) + 15) / 16 * 16 / (int)sizeof(HT);
}

// Pass 1 of the two-pass chunked assembly: every tet once, one thread each.
template <typename HT, bool SNH>
__global__ void __launch_bounds__(128) k_tet_gen(AsmArgs<HT> a, int E) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    GlobalGenSink<HT> sink{reinterpret_cast<HT*>(a.ch.gen) + (size_t)e * chunk_gen_stride<HT, SNH>(),
                           a.ch.gradg + (size_t)e * 12};
    if (!tet_generator<HT, SNH>(a, e, a.want_hess != 0, sink)) atomicOr(a.status, kFlagInverted);
}

template <typename HT, bool SNH, bool FROMGEN>
__global__ void __launch_bounds__(kChunkThreads, 2) k_assemble_chunk(AsmArgs<HT> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using G = ChunkGen<SNH>;
    const int EM = a.ch.elems_max;
    double* gslot = reinterpret_cast<double*>(smem_raw);
    HT* gen = reinterpret_cast<HT*>(smem_raw + a.ch.region_bytes);
    int* srow = reinterpret_cast<int*>(gen + (size_t)G::kFields * EM);
    int* srp0 = srow + a.ch.rows_max;
    int* spair0 = srp0 + a.ch.rows_max;
    int* sblk0 = spair0 + a.ch.rows_max + 1;
    int* sdiag = sblk0 + a.ch.rows_max + 1;  // position of the diagonal block in each row
    const int chunk = blockIdx.x;
    const int r0 = __ldg(a.ch.ch_ptr + chunk), nr = __ldg(a.ch.ch_ptr + chunk + 1) - r0;
    const int e0 = __ldg(a.ch.ch_eptr + chunk), ne = __ldg(a.ch.ch_eptr + chunk + 1) - e0;
    const int lane = threadIdx.x & 31;
    // chunk rows: node id, first CSR block, and chunk-local pair / block offsets
    if (threadIdx.x < 32) {
        int pacc = 0, bacc = 0;
        for (int base = 0; base < nr; base += 32) {
            const int p = base + lane;
            int r = 0, rp = 0, np = 0, nb = 0;
            if (p < nr) {
                r = __ldg(a.ch.ch_rows + r0 + p);
                np = __ldg(a.pair_ptr + r + 1) - __ldg(a.pair_ptr + r);
                rp = __ldg(a.row_ptr + r);
                nb = __ldg(a.row_ptr + r + 1) - rp;
            }
            int ip = np, ib = nb;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int tp = __shfl_up_sync(0xffffffffu, ip, o), tb = __shfl_up_sync(0xffffffffu, ib, o);
                if (lane >= o) { ip += tp; ib += tb; }
            }
            if (p < nr) {
                srow[p] = r; srp0[p] = rp; spair0[p] = pacc + ip - np; sblk0[p] = bacc + ib - nb;
                sdiag[p] = __ldg(a.diag_slot + r) - rp;
            }
            pacc += __shfl_sync(0xffffffffu, ip, 31);
            bacc += __shfl_sync(0xffffffffu, ib, 31);
        }
        if (lane == 0) { spair0[nr] = pacc; sblk0[nr] = bacc; }
    }
    // A. element generators and gradient pairs (evaluated here, or loaded
    // from the records of k_tet_gen)
    bool ok = true;
    for (int s = threadIdx.x; s < ne; s += blockDim.x) {
        const int e = __ldg(a.ch.ch_elems + e0 + s);
        const ushort4 sl = a.ch.ch_eslot[e0 + s];
        const unsigned short slots[4] = {sl.x, sl.y, sl.z, sl.w};
        if (FROMGEN) {
            const HT* rec = reinterpret_cast<const HT*>(a.ch.gen) + (size_t)e * chunk_gen_stride<HT, SNH>();
            const double* gr = a.ch.gradg + (size_t)e * 12;
#pragma unroll
            for (int v = 0; v < 4; v++) {
                if (slots[v] == 0xffff) continue;
#pragma unroll
                for (int r = 0; r < 3; r++) gslot[3 * slots[v] + r] = __ldg(gr + 3 * v + r);
            }
            if (a.want_hess)
#pragma unroll
                for (int f = 0; f < G::kFields; f++) gen[f * EM + s] = __ldg(rec + f);
        } else {
            SmemGenSink<HT> sink{gen, EM, s, gslot, {slots[0], slots[1], slots[2], slots[3]}};
            ok &= tet_generator<HT, SNH>(a, e, a.want_hess != 0, sink);
        }
    }
    if (!ok) atomicOr(a.status, kFlagInverted);
    __syncthreads();
    // C. gradient rows
    for (int p = threadIdx.x; p < nr; p += blockDim.x) {
        const int row = srow[p];
        double g0 = 0.0, g1 = 0.0, g2 = 0.0;
        for (int k = spair0[p]; k < spair0[p + 1]; k++) {
            g0 += gslot[3 * k]; g1 += gslot[3 * k + 1]; g2 += gslot[3 * k + 2];
        }
        const unsigned mrow = a.node_mask[row];
        if (a.apply_mask) {
            if (mrow & 1u) g0 = 0.0;
            if (mrow & 2u) g1 = 0.0;
            if (mrow & 4u) g2 = 0.0;
        }
        a.g_int[3 * (size_t)row + 0] = g0;
        a.g_int[3 * (size_t)row + 1] = g1;
        a.g_int[3 * (size_t)row + 2] = g2;
    }
    if (!a.want_hess) return;
    // B. Hessian blocks, one thread per block, the chunk's diagonal blocks
    // first: a diagonal block sums one item per incident pair (about four
    // times an off-diagonal block's), so grouping them keeps warps balanced.
    // Diagonal items use the symmetric form hmu (d_v . d_v) I + (h1 - h2) a_v a_v^T
    // [+ h4 f_v f_v^T].
    const int total = sblk0[nr];
    for (int lb = threadIdx.x; lb < total; lb += blockDim.x) {
        int pos, bg, kb;
        const bool diag = lb < nr;
        if (diag) {
            pos = lb;
            kb = sdiag[pos];
            bg = srp0[pos] + kb;
        } else {
            const int j = lb - nr;  // j-th off-diagonal block of the chunk
            int lo = 0, hi = nr - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (sblk0[mid] - mid <= j) lo = mid; else hi = mid - 1;
            }
            pos = lo;
            const int k = j - (sblk0[pos] - pos);
            kb = k + (k >= sdiag[pos] ? 1 : 0);
            bg = srp0[pos] + kb;
        }
        const int row = srow[pos];
        const int i0 = __ldg(a.slot_item_ptr + bg), i1 = __ldg(a.slot_item_ptr + bg + 1);
        HT acc[9];
#pragma unroll
        for (int k = 0; k < 9; k++) acc[k] = HT(0);
        if (diag) {
            for (int it = i0; it < i1; ++it) {
                const unsigned item = __ldg(a.ch.items + it);
                const int es = (int)(item >> 4), v = (item >> 2) & 3;
                const HT hmu = gen[0 * EM + es], c1 = gen[1 * EM + es] - gen[2 * EM + es];
                const HT dd = gen[(G::kDD + dd_index(v, v)) * EM + es];
                HT av[3], fv[3] = {HT(0), HT(0), HT(0)};
#pragma unroll
                for (int k = 0; k < 3; k++) av[k] = gen[(G::kA + v * 3 + k) * EM + es];
                HT h4 = HT(0);
                if (SNH) {
                    h4 = gen[G::kH4 * EM + es];
#pragma unroll
                    for (int k = 0; k < 3; k++) fv[k] = gen[(G::kF + v * 3 + k) * EM + es];
                }
#pragma unroll
                for (int k = 0; k < 3; k++)
#pragma unroll
                    for (int l = k; l < 3; l++) {
                        HT val = c1 * av[k] * av[l];
                        if (SNH) val += h4 * fv[k] * fv[l];
                        if (k == l) val += hmu * dd;
                        acc[k * 3 + l] += val;
                    }
            }
            acc[3] = acc[1]; acc[6] = acc[2]; acc[7] = acc[5];
        } else {
            for (int it = i0; it < i1; ++it) {
                const unsigned item = __ldg(a.ch.items + it);
                const int es = (int)(item >> 4), v = (item >> 2) & 3, w = item & 3;
                const HT hmu = gen[0 * EM + es], h1 = gen[1 * EM + es], h2 = gen[2 * EM + es];
                const HT dd = gen[(G::kDD + (v <= w ? dd_index(v, w) : dd_index(w, v))) * EM + es];
                HT av[3], aw[3];
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    av[k] = gen[(G::kA + v * 3 + k) * EM + es];
                    aw[k] = gen[(G::kA + w * 3 + k) * EM + es];
                }
                HT h4 = HT(0), fv[3] = {HT(0), HT(0), HT(0)}, fw[3] = {HT(0), HT(0), HT(0)};
                if (SNH) {
                    h4 = gen[G::kH4 * EM + es];
#pragma unroll
                    for (int k = 0; k < 3; k++) {
                        fv[k] = gen[(G::kF + v * 3 + k) * EM + es];
                        fw[k] = gen[(G::kF + w * 3 + k) * EM + es];
                    }
                }
#pragma unroll
                for (int k = 0; k < 3; k++)
#pragma unroll
                    for (int l = 0; l < 3; l++) {
                        HT val = h1 * av[k] * aw[l] - h2 * aw[k] * av[l];
                        if (SNH) val += h4 * fv[k] * fw[l];
                        if (k == l) val += hmu * dd;
                        acc[k * 3 + l] += val;
                    }
            }
        }
        const int j = __ldg(a.col + bg);
        const unsigned mrow = a.node_mask[row], mcol = a.node_mask[j];
        const double md = a.inertia_coef * a.mass[row];
#pragma unroll
        for (int rc = 0; rc < 9; rc++) {
            const int r = rc / 3, c = rc - 3 * (rc / 3);
            const bool rmask = (mrow >> r) & 1u;
            double val = (double)acc[rc] * a.hscale;
            if (a.apply_mask && (rmask || ((mcol >> c) & 1u))) val = 0.0;
            if (j == row && r == c) {
                val += md;
                if (a.neumann_override && rmask) val = 1.0;
            }
            a.H[hval(bg, rc, a.nnzb)] = (HT)val;
        }
    }
}

// Raises a kernel's dynamic shared-memory limit to `smem` once per device
// (the attribute is per device; `done` remembers the largest size set on each).
template <typename K>
static void set_smem_limit(K kernel, size_t smem, std::atomic<int>* done) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) dev = 0;
    if (done[dev].load(std::memory_order_relaxed) >= (int)smem) return;
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int cur = done[dev].load(std::memory_order_relaxed);
    while (cur < (int)smem && !done[dev].compare_exchange_weak(cur, (int)smem)) {
    }
}

template <typename HT, bool SNH>
static void launch_assemble_chunk(const AsmArgs<HT>& a, cudaStream_t st) {
    static std::atomic<int> limit[2][kMaxDevices];
    const size_t smem = a.ch.smem_bytes;
    if (a.ch.gen) {
        // two passes: every element once, then the chunks load its records
        k_tet_gen<HT, SNH><<<(a.E + 127) / 128, 128, 0, st>>>(a, a.E);
        auto k = k_assemble_chunk<HT, SNH, true>;
        set_smem_limit(k, smem, limit[1]);
        k<<<a.ch.nchunks, kChunkThreads, smem, st>>>(a);
        counted(2);
    } else {
        auto k = k_assemble_chunk<HT, SNH, false>;
        set_smem_limit(k, smem, limit[0]);
        k<<<a.ch.nchunks, kChunkThreads, smem, st>>>(a);
        counted();
    }
}

// ---------------------------------------------------------------------------
// Element-owner hex assembly in two passes.
// Pass 1 (k_hex_tiles): one warp per hex, four lanes per Gauss point s (all
// 32 lanes busy).  The four lanes of s each compute the shape gradients d_s
// (hexahedron.cpp:170-207), F and the scalar terms; each then writes its own
// rows i = part, part + 4, part + 8 of P_s and of the 9x9 dP/dF A_s (exact
// Neo-Hookean or stable Neo-Hookean terms hmu I + h1 g g^T - h2 G_rc' G_r'c
// [+ h4 f f^T], the SPD projection's corrections -lambda_m vec(Q_m) vec(Q_m)^T
// for the negative modes of the analytic eigensystem, and the fibre term)
// into shared memory.  The 36 upper 3x3 blocks block(v,w) = sum_s wV d_sv^T
// A_s d_sw are then formed through T_sw = A_s (I x d_sw) (27 values per
// (s, w), 216 per s on the 32 lanes): block(v,w)[k][l] = sum_s wV sum_i
// d_sv[i] T_sw[k,i][l], 108 (block, k) rows on the 32 lanes, accumulated in
// registers over s.  That is 13k multiply-adds per hex instead of the 47k of
// d_v^T A_s d_w per block.  24 lanes write the gradient rows; both go to the
// element's tile.
// Pass 2 (k_hex_gather): one warp per row, a lane per CSR block, sums the
// block's items from the tiles (transposed for v > w) in slot order.
// ---------------------------------------------------------------------------
constexpr int kHexWarps = 4;

__device__ __forceinline__ int hex_upper(int v, int w) {  // v <= w
    return v * 8 - (v * (v - 1)) / 2 + (w - v);
}

// v[i] for a lane-dependent i in [0, 9) without local memory
template <typename T>
__device__ __forceinline__ T pick9(const T (&v)[9], int i) {
    T r = v[0];
#pragma unroll
    for (int k = 1; k < 9; k++) r = (i == k) ? v[k] : r;
    return r;
}

template <typename HT>
struct HexWarpMem {
    double X[8][3], x[8][3];
    double d[8][8][3];
    double P[8][9];
    HT A[8][81];
    HT T[2][216];                            // T_sw, double-buffered over s
    float dh[sizeof(HT) == 4 ? 8 : 1][8][3]; // FP32 copy of d for the block phase (FP32 tiles only)
    double wV;
};

template <typename HT>
__device__ __forceinline__ HT hex_d(const HexWarpMem<HT>& W, int s, int w, int j) {
    if constexpr (sizeof(HT) == 4) return W.dh[s][w][j];
    else return W.d[s][w][j];
}

template <typename HT, bool SNH, bool PROJ>
__global__ void __launch_bounds__(32 * kHexWarps) k_hex_tiles(AsmArgs<HT> a, int E) {
    __shared__ HexWarpMem<HT> wm[kHexWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    HexWarpMem<HT>& W = wm[warp];
    const int s = lane >> 2, part = lane & 3;
    // this lane's (block, k) rows of the block phase: t = lane + 32 u < 108
    int bv[4], bw[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
        const int t = lane + 32 * u;
        int v = 0, rem = t < 108 ? t / 3 : 0;
        while (rem >= 8 - v) { rem -= 8 - v; v++; }
        bv[u] = v;
        bw[u] = v + rem;
    }
    bool ok = true;
    for (int e = blockIdx.x * kHexWarps + warp; e < E; e += gridDim.x * kHexWarps) {
        if (lane < 24) {
            const int v = lane / 3, r = lane - 3 * (lane / 3);
            const int n = __ldg(a.conn + (size_t)e * 8 + v);
            W.X[v][r] = __ldg(a.X + 3 * (size_t)n + r);
            W.x[v][r] = a.q[3 * (size_t)n + r];
        }
        __syncwarp();
        {
            if (lane == 0) W.wV = hex_volume((const double(*)[3])W.X) * 0.125;
            double d[8][3];
            hex_shape((const double(*)[3])W.X, s, d);
            double F[9];
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    double acc = 0.0;
#pragma unroll
                    for (int w = 0; w < 8; w++) acc += W.x[w][r] * d[w][c];
                    F[r * 3 + c] = acc;
                }
            // this lane stores d_s of vertices 2 part and 2 part + 1
#pragma unroll
            for (int w = 0; w < 8; w++)
                if ((w >> 1) == part)
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        W.d[s][w][c] = d[w][c];
                        if constexpr (sizeof(HT) == 4) W.dh[s][w][c] = (float)d[w][c];
                    }
            const double2 m = __ldg(a.mat + e);
            double C[9];
            cof3(F, C);
            const double J = F[0] * C[0] + F[1] * C[1] + F[2] * C[2];
            const double iJ = 1.0 / J;
            double G[9];
#pragma unroll
            for (int k = 0; k < 9; k++) G[k] = C[k] * iJ;
            double IC = 0.0;
            if (SNH)
#pragma unroll
                for (int k = 0; k < 9; k++) IC += F[k] * F[k];
            const double alpha = SNH ? 1.0 + 0.75 * m.x / m.y : 0.0;
            const double logJ = SNH ? 0.0 : log(J);
            const double hmu = SNH ? m.x * (1.0 - 1.0 / (IC + 1.0)) : m.x;
            const double h2 = SNH ? m.y * (J - alpha) * J : (m.y * logJ - m.x);
            const double h1 = SNH ? m.y * (2.0 * J - alpha) * J : m.y;
            const double h4 = SNH ? 2.0 * m.x / ((IC + 1.0) * (IC + 1.0)) : 0.0;
            const bool qok = SNH ? (J != 0.0) : (J > 0.0);
            ok &= qok;
            // fibre term (softconMuscle.cpp, in its consistent squared form)
            const int grp = a.mus.group ? __ldg(a.mus.group + e) : -1;
            double4 mp = make_double4(0.0, 0.0, 0.0, 0.0);
            double u[3] = {0.0, 0.0, 0.0}, rr = 0.0, il2 = 0.0;
            if (grp >= 0) {
                mp = a.mus.param[e];
                const double eact = __ldg(a.mus.act + grp);
#pragma unroll
                for (int r = 0; r < 3; r++) u[r] = F[r * 3 + 0] * mp.x + F[r * 3 + 1] * mp.y + F[r * 3 + 2] * mp.z;
                const double l = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
                rr = (1.0 - eact) / l;
                il2 = 1.0 / (l * l);
            }
            const double mv[3] = {mp.x, mp.y, mp.z};
            // rows i = part, part + 4, part + 8 of P_s and A_s
#pragma unroll
            for (int ii = 0; ii < 3; ii++) {
                const int i = part + 4 * ii;
                if (i >= 9) break;
                const int r = i / 3, c = i - 3 * (i / 3);
                const double Gi = pick9(G, i), Fi = pick9(F, i);
                double Pi = hmu * Fi + h2 * Gi;
                const double ur = r == 0 ? u[0] : (r == 1 ? u[1] : u[2]);
                const double mc = c == 0 ? mv[0] : (c == 1 ? mv[1] : mv[2]);
                if (grp >= 0) Pi += mp.w * (1.0 - rr) * ur * mc;
                W.P[s][i] = Pi;
                if (!a.want_hess) continue;
                // G[r*3+cp] and G[rp*3+c] for the nine columns (rp, cp)
                double Gr[3], Gc[3];
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    Gr[k] = pick9(G, r * 3 + k);
                    Gc[k] = pick9(G, k * 3 + c);
                }
                double cf = 1.0 - rr;
                if (PROJ && cf < 0.0) cf = 0.0;
#pragma unroll
                for (int j = 0; j < 9; j++) {
                    const int rp = j / 3, cp = j - 3 * (j / 3);
                    double val = h1 * Gi * G[j] - h2 * Gr[cp] * Gc[rp];
                    if (SNH) val += h4 * Fi * F[j];
                    if (i == j) val += hmu;
                    if (!qok) val = 0.0;
                    if (grp >= 0) {
                        const double M = (1.0 - cf) * ur * u[rp] * il2 + (r == rp ? cf : 0.0);
                        val += mp.w * mc * mv[cp] * M;
                    }
                    W.A[s][i * 9 + j] = (HT)val;
                }
            }
            if (a.want_hess && PROJ && qok) {
                HT Fh[9];
#pragma unroll
                for (int k = 0; k < 9; k++) Fh[k] = (HT)F[k];
                NhModes<HT> pm;
                if (SNH) snh_modes<HT>(Fh, (HT)J, (HT)IC, (HT)m.x, (HT)m.y, (HT)alpha, pm);
                else nh_modes<HT>(Fh, (HT)J, (HT)logJ, (HT)m.x, (HT)m.y, pm);
                if (pm.any) {
                    const HT r2 = HT(0.70710678118654752440);
                    HT Q[9];
                    auto add_mode = [&](HT lam_m) {
#pragma unroll
                        for (int ii = 0; ii < 3; ii++) {
                            const int i = part + 4 * ii;
                            if (i >= 9) break;
                            const HT Qi = pick9(Q, i);
#pragma unroll
                            for (int j = 0; j < 9; j++) W.A[s][i * 9 + j] += -lam_m * Qi * Q[j];
                        }
                    };
#pragma unroll
                    for (int mm = 0; mm < 3; mm++) {
                        const int I = mm == 2 ? 1 : 0, JJ = mm == 0 ? 1 : 2;
#pragma unroll
                        for (int sg = 0; sg < 2; sg++) {
                            const HT lam_m = sg == 0 ? pm.lt[mm] : pm.lf[mm];
                            if (!(lam_m < HT(0))) continue;
                            const HT sign = sg == 0 ? HT(-1) : HT(1);
#pragma unroll
                            for (int r = 0; r < 3; r++)
#pragma unroll
                                for (int c = 0; c < 3; c++)
                                    Q[r * 3 + c] = (pm.U[r * 3 + I] * pm.V[c * 3 + JJ] +
                                                    sign * pm.U[r * 3 + JJ] * pm.V[c * 3 + I]) * r2;
                            add_mode(lam_m);
                        }
                    }
#pragma unroll
                    for (int mm = 0; mm < 3; mm++) {
                        if (!(pm.ls[mm] < HT(0))) continue;
#pragma unroll
                        for (int r = 0; r < 3; r++)
#pragma unroll
                            for (int c = 0; c < 3; c++) {
                                HT acc = HT(0);
#pragma unroll
                                for (int k = 0; k < 3; k++)
                                    acc += pm.U[r * 3 + k] * pm.Y[k * 3 + mm] * pm.V[c * 3 + k];
                                Q[r * 3 + c] = acc;
                            }
                        add_mode(pm.ls[mm]);
                    }
                }
            }
        }
        __syncwarp();
        const double wV = W.wV;
        // gradient rows: g_v = sum_s wV P_s d_sv
        if (lane < 24) {
            const int v = lane / 3, r = lane - 3 * (lane / 3);
            double acc = 0.0;
            for (int s2 = 0; s2 < 8; s2++)
                acc += wV * (W.P[s2][r * 3 + 0] * W.d[s2][v][0] + W.P[s2][r * 3 + 1] * W.d[s2][v][1] +
                             W.P[s2][r * 3 + 2] * W.d[s2][v][2]);
            a.hex_gtile[(size_t)e * 24 + lane] = acc;
        }
        if (a.want_hess) {
            HT acc[4][3];
#pragma unroll
            for (int u = 0; u < 4; u++)
#pragma unroll
                for (int l = 0; l < 3; l++) acc[u][l] = HT(0);
            for (int s2 = 0; s2 < 8; s2++) {
                HT* Tb = W.T[s2 & 1];
                const HT* A = W.A[s2];
                // T_sw[k,i][l] = sum_j A_s[(k,i),(l,j)] d_sw[j], index w*27 + (k*3+i)*3 + l
#pragma unroll
                for (int t2 = lane; t2 < 216; t2 += 32) {
                    const int w = t2 / 27, rem = t2 - 27 * (t2 / 27);
                    const int ki = rem / 3, l = rem - 3 * (rem / 3);
                    const HT* Ar = A + ki * 9 + l * 3;
                    Tb[t2] = Ar[0] * hex_d(W, s2, w, 0) + Ar[1] * hex_d(W, s2, w, 1) + Ar[2] * hex_d(W, s2, w, 2);
                }
                __syncwarp();
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int t = lane + 32 * u;
                    if (t >= 108) break;
                    const int k = t - 3 * (t / 3);
                    const HT dv0 = hex_d(W, s2, bv[u], 0), dv1 = hex_d(W, s2, bv[u], 1), dv2 = hex_d(W, s2, bv[u], 2);
                    const HT* Tr = Tb + bw[u] * 27 + k * 9;
#pragma unroll
                    for (int l = 0; l < 3; l++) acc[u][l] += dv0 * Tr[l] + dv1 * Tr[3 + l] + dv2 * Tr[6 + l];
                }
            }
            HT* tile = reinterpret_cast<HT*>(a.hex_tile) + (size_t)e * 36 * 9;
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int t = lane + 32 * u;
                if (t >= 108) break;
                const int b = t / 3, k = t - 3 * (t / 3);
#pragma unroll
                for (int l = 0; l < 3; l++) tile[b * 9 + k * 3 + l] = (HT)wV * acc[u][l];
            }
        }
        __syncwarp();
    }
    if (!ok) atomicOr(a.status, kFlagInverted);
}

template <typename HT>
__global__ void __launch_bounds__(256) k_hex_gather(AsmArgs<HT> a) {
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    const HT* tiles = reinterpret_cast<const HT*>(a.hex_tile);
    for (int row = blockIdx.x * wpb + (threadIdx.x >> 5); row < a.N; row += gridDim.x * wpb) {
        const int p0 = __ldg(a.pair_ptr + row);
        const unsigned mrow = a.node_mask[row];
        if (lane < 3) {
            double g = 0.0;
            for (int p = p0; p < __ldg(a.pair_ptr + row + 1); p++) {
                const int ev = __ldg(a.pair_ev + p);
                g += a.hex_gtile[(size_t)(ev >> 3) * 24 + (ev & 7) * 3 + lane];
            }
            if (a.apply_mask && ((mrow >> lane) & 1u)) g = 0.0;
            a.g_int[3 * (size_t)row + lane] = g;
        }
        if (!a.want_hess) continue;
        const int b0 = __ldg(a.row_ptr + row), nb = __ldg(a.row_ptr + row + 1) - b0;
        const double md = a.inertia_coef * a.mass[row];
        for (int k = lane; k < nb; k += 32) {
            const int bg = b0 + k;
            HT acc[9];
#pragma unroll
            for (int t = 0; t < 9; t++) acc[t] = HT(0);
            for (int it = __ldg(a.slot_item_ptr + bg); it < __ldg(a.slot_item_ptr + bg + 1); ++it) {
                const int item = __ldg(a.slot_items + it);
                const int kp = item >> 3, w = item & 7;
                const int ev = __ldg(a.pair_ev + p0 + kp);
                const int e = ev >> 3, v = ev & 7;
                const HT* T = tiles + ((size_t)e * 36 + (v <= w ? hex_upper(v, w) : hex_upper(w, v))) * 9;
                if (v <= w) {
#pragma unroll
                    for (int t = 0; t < 9; t++) acc[t] += T[t];
                } else {
#pragma unroll
                    for (int r = 0; r < 3; r++)
#pragma unroll
                        for (int c = 0; c < 3; c++) acc[r * 3 + c] += T[c * 3 + r];
                }
            }
            const int j = __ldg(a.col + bg);
            const unsigned mcol = a.node_mask[j];
#pragma unroll
            for (int rc = 0; rc < 9; rc++) {
                const int r = rc / 3, c = rc - 3 * (rc / 3);
                const bool rmask = (mrow >> r) & 1u;
                double val = (double)acc[rc] * a.hscale;
                if (a.apply_mask && (rmask || ((mcol >> c) & 1u))) val = 0.0;
                if (j == row && r == c) {
                    val += md;
                    if (a.neumann_override && rmask) val = 1.0;
                }
                a.H[hval(bg, rc, a.nnzb)] = (HT)val;
            }
        }
    }
}

// Pass 2 with a thread per CSR block (the row from hex_blk_row), so that the
// lanes of a warp write consecutive blocks, then a thread per gradient entry;
// each block and each entry sums its items in slot order, as k_hex_gather.
template <typename HT>
__global__ void __launch_bounds__(256) k_hex_gather_blocks(AsmArgs<HT> a, long long nblk) {
    const HT* tiles = reinterpret_cast<const HT*>(a.hex_tile);
    const long long total = nblk + 3LL * a.N;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        if (t >= nblk) {
            // gradient entry u of row u / 3
            const long long u = t - nblk;
            const int row = (int)(u / 3), lane = (int)(u - 3 * (u / 3));
            double g = 0.0;
            for (int p = __ldg(a.pair_ptr + row); p < __ldg(a.pair_ptr + row + 1); p++) {
                const int ev = __ldg(a.pair_ev + p);
                g += a.hex_gtile[(size_t)(ev >> 3) * 24 + (ev & 7) * 3 + lane];
            }
            if (a.apply_mask && ((a.node_mask[row] >> lane) & 1u)) g = 0.0;
            a.g_int[3 * (size_t)row + lane] = g;
            continue;
        }
        const int bg = (int)t;
        const int row = __ldg(a.hex_blk_row + bg);
        const int p0 = __ldg(a.pair_ptr + row);
        const unsigned mrow = a.node_mask[row];
        HT acc[9];
#pragma unroll
        for (int k = 0; k < 9; k++) acc[k] = HT(0);
        for (int it = __ldg(a.slot_item_ptr + bg); it < __ldg(a.slot_item_ptr + bg + 1); ++it) {
            const int item = __ldg(a.slot_items + it);
            const int kp = item >> 3, w = item & 7;
            const int ev = __ldg(a.pair_ev + p0 + kp);
            const int e = ev >> 3, v = ev & 7;
            const HT* T = tiles + ((size_t)e * 36 + (v <= w ? hex_upper(v, w) : hex_upper(w, v))) * 9;
            if (v <= w) {
#pragma unroll
                for (int k = 0; k < 9; k++) acc[k] += T[k];
            } else {
#pragma unroll
                for (int r = 0; r < 3; r++)
#pragma unroll
                    for (int c = 0; c < 3; c++) acc[r * 3 + c] += T[c * 3 + r];
            }
        }
        const int j = __ldg(a.col + bg);
        const unsigned mcol = a.node_mask[j];
        const double md = a.inertia_coef * a.mass[row];
#pragma unroll
        for (int rc = 0; rc < 9; rc++) {
            const int r = rc / 3, c = rc - 3 * (rc / 3);
            const bool rmask = (mrow >> r) & 1u;
            double val = (double)acc[rc] * a.hscale;
            if (a.apply_mask && (rmask || ((mcol >> c) & 1u))) val = 0.0;
            if (j == row && r == c) {
                val += md;
                if (a.neumann_override && rmask) val = 1.0;
            }
            a.H[hval(bg, rc, a.nnzb)] = (HT)val;
        }
    }
}

template <typename HT>
static void launch_hex_tiles(const AsmArgs<HT>& a, cudaStream_t st) {
    const bool snh = a.material == 2, proj = a.project != 0;
    const long long hb = cap_grid(((long long)a.E + kHexWarps - 1) / kHexWarps);
    auto k = snh ? (proj ? k_hex_tiles<HT, true, true> : k_hex_tiles<HT, true, false>)
                 : (proj ? k_hex_tiles<HT, false, true> : k_hex_tiles<HT, false, false>);
    if (a.E > 0) k<<<(int)hb, 32 * kHexWarps, 0, st>>>(a, a.E);
    if (a.hex_blk_row) {
        const long long nblk = a.want_hess ? a.nnzb : 0;
        const long long total = nblk + 3LL * a.N;
        const long long gb = cap_grid((total + 255) / 256);
        k_hex_gather_blocks<HT><<<(int)gb, 256, 0, st>>>(a, nblk);
    } else {
        const long long gb = cap_grid(((long long)a.N + 7) / 8);
        k_hex_gather<HT><<<(int)gb, 256, 0, st>>>(a);
    }
    counted(2);
}

template <typename HT>
void launch_assemble(const AsmArgs<HT>& a, int max_pairs, cudaStream_t st) {
    if (a.N == 0) return;
    const int nv = a.nv;
    size_t per_warp = (size_t)a.stage_per_warp * sizeof(HT);
    int wpb = 8;
    while (wpb > 1 && per_warp * wpb > 200 * 1024) wpb >>= 1;
    size_t smem = per_warp * wpb;
    int threads = wpb * 32;
    long long rows_per_block = wpb;
    long long blocks = (a.N + rows_per_block - 1) / rows_per_block;
    if (blocks > (long long)sm_count() * 64) blocks = (long long)sm_count() * 64;
    blocks = cap_grid(blocks);
    const bool snh = a.material == 2;
    if (nv == 4 && a.ch.nchunks > 0 && !a.project && !a.mus.group && (a.material == 0 || snh)) {
        if (snh) launch_assemble_chunk<HT, true>(a, st);
        else launch_assemble_chunk<HT, false>(a, st);
        return;
    }
    if (nv == 8 && a.hex_tile && (a.material == 0 || snh)) {
        launch_hex_tiles<HT>(a, st);
        return;
    }
    if (nv == 4) {
        // tets: projection selects the kernel variant (the exact Hessian keeps
        // the projection's registers out of the common case)
        static std::atomic<int> limit[4][kMaxDevices];
        const int variant = (snh ? 2 : 0) + (a.project ? 1 : 0);
        auto k = snh ? (a.project ? k_assemble<HT, 4, true, true> : k_assemble<HT, 4, true, false>)
                     : (a.project ? k_assemble<HT, 4, false, true> : k_assemble<HT, 4, false, false>);
        set_smem_limit(k, smem, limit[variant]);
        k<<<(int)blocks, threads, smem, st>>>(a);
        counted();
    } else {
        static std::atomic<int> limit[2][kMaxDevices];
        auto k = snh ? k_assemble<HT, 8, true, false> : k_assemble<HT, 8, false, false>;
        set_smem_limit(k, smem, limit[snh ? 1 : 0]);
        k<<<(int)blocks, threads, smem, st>>>(a);
        counted();
    }
    (void)max_pairs;
}

// Element-level parity hook: thread per (element, local vertex).
template <typename HT, int NV>
__global__ void k_elem_rows(int E, const double* X, const double* q, const int* conn, const double2* mat,
                            const double* tsh, MuscleArgs mus, int material, int project, double* psi, double* grad,
                            double* hess, int* status) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)E * NV) return;
    int e = (int)(t / NV), v = (int)(t - (long long)e * NV);
    double g[3] = {0.0, 0.0, 0.0};
    HT blk[NV * 9];
    bool ok = material == 2
                  ? elem_row<HT, NV, true, true>(X, q, conn, mat, tsh, mus, e, v, material, project != 0, g, blk)
                  : elem_row<HT, NV, true, false>(X, q, conn, mat, tsh, mus, e, v, material, project != 0, g, blk);
    if (!ok) atomicOr(status, kFlagInverted);
    const int n = 3 * NV;
    if (grad)
        for (int r = 0; r < 3; r++) grad[(size_t)e * n + 3 * v + r] = g[r];
    if (hess)
        for (int w = 0; w < NV; w++)
            for (int k = 0; k < 3; k++)
                for (int l = 0; l < 3; l++)
                    hess[(size_t)e * n * n + (size_t)(3 * v + k) * n + 3 * w + l] = (double)blk[w * 9 + k * 3 + l];
    if (psi && v == 0) psi[e] = elem_energy<NV>(X, q, conn, mat, mus, e, material);
}

template <typename HT>
void launch_elem_rows(int E, int nv, const double* X, const double* q, const int* conn, const double2* mat,
                      const double* tsh, const MuscleArgs& mus, int material, int project, double* psi, double* grad, double* hess, int* status,
                      cudaStream_t st) {
    long long n = (long long)E * nv;
    if (n == 0) return;
    int threads = 128;
    int blocks = (int)((n + threads - 1) / threads);
    if (nv == 4)
        k_elem_rows<HT, 4><<<blocks, threads, 0, st>>>(E, X, q, conn, mat, tsh, mus, material, project, psi, grad,
                                                       hess, status);
    else
        k_elem_rows<HT, 8><<<blocks, threads, 0, st>>>(E, X, q, conn, mat, tsh, mus, material, project, psi, grad,
                                                       hess, status);
    counted();
}

// ---------------------------------------------------------------------------
// element energies (all elements, unmasked: energy.cpp:212-227)
// ---------------------------------------------------------------------------
template <int NV>
__global__ void __launch_bounds__(kRedThreads) k_elem_energy(int E, const double* __restrict__ Xg,
                                                             const double* __restrict__ qg,
                                                             const int* __restrict__ conn,
                                                             const double2* __restrict__ mat, MuscleArgs mus,
                                                             int material, double* partials, DevScalars* sc) {
    double acc[1] = {0.0};
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x)
        acc[0] += elem_energy<NV>(Xg, qg, conn, mat, mus, e, material);
    double tot[1];
    if (reduce_grid<1>(acc, partials, &sc->counters[0], tot) && threadIdx.x == 0) sc->e_elem = tot[0];
}

void launch_elem_energy(int E, int nv, const double* X, const double* q, const int* conn, const double2* mat,
                        const MuscleArgs& mus, int material, double* partials, DevScalars* sc, cudaStream_t st) {
    int blocks = red_grid(E);
    if (nv == 4)
        k_elem_energy<4><<<blocks, kRedThreads, 0, st>>>(E, X, q, conn, mat, mus, material, partials, sc);
    else
        k_elem_energy<8><<<blocks, kRedThreads, 0, st>>>(E, X, q, conn, mat, mus, material, partials, sc);
    counted();
}

// ---------------------------------------------------------------------------
// pressure force (pressureForce.cpp:14-56) and its Jacobian (:59-186),
// row-owner over surface nodes
// ---------------------------------------------------------------------------
__device__ __forceinline__ void face_area(const int* f, int fnv, const double* q, double* area) {
    const double* x0 = q + 3 * (size_t)f[0];
    const double* x1 = q + 3 * (size_t)f[1];
    const double* x2 = q + 3 * (size_t)f[2];
    if (fnv == 3) {
        double v1[3] = {x1[0] - x0[0], x1[1] - x0[1], x1[2] - x0[2]};
        double v2[3] = {x2[0] - x0[0], x2[1] - x0[1], x2[2] - x0[2]};
        area[0] = 0.5 * (v1[1] * v2[2] - v1[2] * v2[1]);
        area[1] = 0.5 * (v1[2] * v2[0] - v1[0] * v2[2]);
        area[2] = 0.5 * (v1[0] * v2[1] - v1[1] * v2[0]);
    } else {
        const double* x3 = q + 3 * (size_t)f[3];
        double v1[3] = {x1[0] - x0[0], x1[1] - x0[1], x1[2] - x0[2]};
        double v2[3] = {x3[0] - x0[0], x3[1] - x0[1], x3[2] - x0[2]};
        double v3[3] = {x3[0] - x2[0], x3[1] - x2[1], x3[2] - x2[2]};
        double v4[3] = {x1[0] - x2[0], x1[1] - x2[1], x1[2] - x2[2]};
        area[0] = 0.5 * (v1[1] * v2[2] - v1[2] * v2[1]) + 0.5 * (v3[1] * v4[2] - v3[2] * v4[1]);
        area[1] = 0.5 * (v1[2] * v2[0] - v1[0] * v2[2]) + 0.5 * (v3[2] * v4[0] - v3[0] * v4[2]);
        area[2] = 0.5 * (v1[0] * v2[1] - v1[1] * v2[0]) + 0.5 * (v3[0] * v4[1] - v3[1] * v4[0]);
    }
}

__global__ void k_pressure_force(PressureArgs p) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= p.nsurf) return;
    int node = p.surf_nodes[s];
    double f[3] = {0.0, 0.0, 0.0};
    for (int t = p.sface_ptr[s]; t < p.sface_ptr[s + 1]; t++) {
        int fl = p.sface_fl[t];
        int face = fl >> 2;
        const int* fv = p.faces + (size_t)face * p.fnv;
        double area[3];
        face_area(fv, p.fnv, p.q, area);
        double pr = p.pressure[p.face_group[face]];
        for (int k = 0; k < 3; k++) f[k] += -pr * area[k] / p.fnv;
    }
    for (int k = 0; k < 3; k++) p.f_ext[3 * (size_t)node + k] += f[k];
}

void launch_pressure_force(const PressureArgs& p, cudaStream_t st) {
    if (p.nsurf == 0) return;
    k_pressure_force<<<(p.nsurf + 127) / 128, 128, 0, st>>>(p);
    counted();
}

// skew(b - a) as in pressureForce.cpp:76-90
__device__ __forceinline__ void skew_ba(const double* a, const double* b, double* M) {
    double d0 = b[0] - a[0], d1 = b[1] - a[1], d2 = b[2] - a[2];
    M[0] = 0;   M[1] = -d2; M[2] = d1;
    M[3] = d2;  M[4] = 0;   M[5] = -d0;
    M[6] = -d1; M[7] = d0;  M[8] = 0;
}

__device__ void face_hess(const int* f, int fnv, const double* q, double (*h)[9]) {
    const double* x0 = q + 3 * (size_t)f[0];
    const double* x1 = q + 3 * (size_t)f[1];
    const double* x2 = q + 3 * (size_t)f[2];
    if (fnv == 3) {
        skew_ba(x1, x2, h[0]);
        skew_ba(x2, x0, h[1]);
        skew_ba(x0, x1, h[2]);
    } else {
        const double* x3 = q + 3 * (size_t)f[3];
        double t1[9], t3[9];
        skew_ba(x1, x3, h[0]);
        skew_ba(x3, x0, h[1]);
        skew_ba(x0, x1, h[3]);
        skew_ba(x3, x1, h[2]);
        skew_ba(x2, x3, t1);
        skew_ba(x1, x2, t3);
        for (int k = 0; k < 9; k++) { h[1][k] += t1[k]; h[3][k] += t3[k]; }
    }
}

// The reference's LDL^T reads the lower triangle of its input, so the
// non-symmetric follower-load Jacobian enters as P(max(a,b), min(a,b)).
template <typename HT>
__global__ void k_pressure_jac(PressureArgs p, const int* row_ptr, const int* col, const uint8_t* node_mask,
                               double cscale, HT* H, long long nnzb) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= p.nsurf) return;
    int i = p.surf_nodes[s];
    int b0 = row_ptr[i], b1 = row_ptr[i + 1];
    unsigned mi = node_mask[i];
    for (int t = p.sface_ptr[s]; t < p.sface_ptr[s + 1]; t++) {
        int fl = p.sface_fl[t];
        int face = fl >> 2, ki = fl & 3;
        const int* fv = p.faces + (size_t)face * p.fnv;
        double h[4][9];
        face_hess(fv, p.fnv, p.q, h);
        double coef = cscale * p.pressure[p.face_group[face]] / 6.0;
        for (int kj = 0; kj < p.fnv; kj++) {
            int j = fv[kj];
            int slot = -1;
            for (int b = b0; b < b1; b++)
                if (col[b] == j) { slot = b; break; }
            if (slot < 0) continue;
            unsigned mj = node_mask[j];
            for (int l = 0; l < 3; l++) {
                if ((mi >> l) & 1u) continue;
                for (int m = 0; m < 3; m++) {
                    if ((mj >> m) & 1u) continue;
                    long long a = 3LL * i + l, b = 3LL * j + m;
                    double val = 0.0;
                    if (a > b) val = h[kj][l * 3 + m];
                    else if (a < b) val = h[ki][m * 3 + l];
                    if (val != 0.0) H[hval(slot, l * 3 + m, nnzb)] += (HT)(coef * val);
                }
            }
        }
    }
}

template <typename HT>
void launch_pressure_jac(const PressureArgs& p, const int* row_ptr, const int* col, const uint8_t* node_mask,
                         double cscale, HT* H, long long nnzb, cudaStream_t st) {
    if (p.nsurf == 0) return;
    k_pressure_jac<HT><<<(p.nsurf + 127) / 128, 128, 0, st>>>(p, row_ptr, col, node_mask, cscale, H, nnzb);
    counted();
}

// Adjoint correction of the follower load, y = (T^T - S) lam on the surface
// rows (y is zero elsewhere and must be cleared by the caller):
//   T: the exact derivative of the residual's pressure term,
//      d g_j / d x_k = p / (2 fnv) * 2 dA/dx_k for every vertex j of the face
//      (face_hess gives 2 dA/dx_k; p/6 for triangles, p/8 for quads);
//   S: what k_pressure_jac adds to the Newton matrix, s_scale times the
//      reference's coefficient p/6 for both face types (0: none), lower
//      triangle mirrored, held DOFs skipped.
// The Newton matrix H = K + S is symmetric; the adjoint needs (K + T)^T =
// H + (T^T - S).
__global__ void k_pressure_adj_corr(PressureArgs p, const uint8_t* node_mask, double s_scale, const double* lam,
                                    double* y) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= p.nsurf) return;
    int i = p.surf_nodes[s];
    unsigned mi = node_mask[i];
    double acc[3] = {0.0, 0.0, 0.0};
    for (int t = p.sface_ptr[s]; t < p.sface_ptr[s + 1]; t++) {
        int fl = p.sface_fl[t];
        int face = fl >> 2, ki = fl & 3;
        const int* fv = p.faces + (size_t)face * p.fnv;
        double h[4][9];
        face_hess(fv, p.fnv, p.q, h);
        const double pr = p.pressure[p.face_group[face]];
        const double c_true = pr / (2.0 * p.fnv), c_ref = s_scale * pr / 6.0;
        for (int kj = 0; kj < p.fnv; kj++) {
            int j = fv[kj];
            unsigned mj = node_mask[j];
            for (int l = 0; l < 3; l++) {
                for (int m = 0; m < 3; m++) {
                    const double lb = lam[3 * (size_t)j + m];
                    // (T^T lam)_a: T[b][a] = c_true h[ki](m, l), a = 3i+l, b = 3j+m
                    double v = c_true * h[ki][m * 3 + l];
                    if (s_scale != 0.0 && !((mi >> l) & 1u) && !((mj >> m) & 1u)) {
                        const long long a = 3LL * i + l, b = 3LL * j + m;
                        if (a > b) v -= c_ref * h[kj][l * 3 + m];
                        else if (a < b) v -= c_ref * h[ki][m * 3 + l];
                    }
                    acc[l] += v * lb;
                }
            }
        }
    }
    for (int l = 0; l < 3; l++) y[3 * (size_t)i + l] = acc[l];
}

void launch_pressure_adj_corr(const PressureArgs& p, const uint8_t* node_mask, double s_scale, const double* lam,
                              double* y, cudaStream_t st) {
    if (p.nsurf == 0) return;
    k_pressure_adj_corr<<<(p.nsurf + 127) / 128, 128, 0, st>>>(p, node_mask, s_scale, lam, y);
    counted();
}

// ---------------------------------------------------------------------------
// gradient finalisation: external forces, integrator, Neumann rows
// (energy.cpp:282-306, integrator.cpp:45-84)
// ---------------------------------------------------------------------------
struct GradArgs {
    int n;
    const double *g_int, *f_ext, *q, *qPrev, *vPrev, *gPrev, *mass, *mval;
    double* gPrevTmp;
    const uint8_t* mask;
    double dt, alpha, grav0, grav1, grav2;
    int scheme, neumann_override, has_ext;
    double* g;
};

__global__ void __launch_bounds__(kRedThreads) k_finalize_grad(GradArgs a, double* partials, DevScalars* sc) {
    double acc[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        int node = i / 3, comp = i - 3 * node;
        double m = a.mass[node];
        double gr = comp == 0 ? a.grav0 : (comp == 1 ? a.grav1 : a.grav2);
        double gi = a.g_int[i] - (a.has_ext ? a.f_ext[i] : 0.0);
        double out;
        if (a.dt == 0.0) {
            out = -m * gr + gi;
        } else {
            a.gPrevTmp[i] = gi;
            double v = a.scheme == 0 ? (a.q[i] - a.qPrev[i]) / a.dt : 2.0 * (a.q[i] - a.qPrev[i]) / a.dt - a.vPrev[i];
            double inert = m * ((v - a.vPrev[i]) / a.dt) + (-m * gr) + a.alpha * m * v;
            out = a.scheme == 0 ? inert + gi : inert + 0.5 * (gi + a.gPrev[i]);
        }
        if (a.neumann_override && ((a.mask[node] >> comp) & 1u)) out = -(a.qPrev[i] + a.dt * a.mval[i] - a.q[i]);
        a.g[i] = out;
        acc[0] += out * out;
    }
    double tot[1];
    if (reduce_grid<1>(acc, partials, &sc->counters[1], tot) && threadIdx.x == 0) sc->gnorm2 = tot[0];
}

void launch_finalize_grad(int N, const double* g_int, const double* f_ext, const double* q, const double* qPrev,
                          const double* vPrev, const double* gPrev, double* gPrevTmp, const double* mass,
                          const uint8_t* mask, const double* mval, double dt, int scheme, double alpha,
                          const double* grav, int neumann_override, int has_ext, double* g, double* partials,
                          DevScalars* sc, cudaStream_t st) {
    GradArgs a;
    a.n = 3 * N; a.g_int = g_int; a.f_ext = f_ext; a.q = q; a.qPrev = qPrev; a.vPrev = vPrev; a.gPrev = gPrev;
    a.gPrevTmp = gPrevTmp; a.mass = mass; a.mask = mask; a.mval = mval; a.dt = dt; a.scheme = scheme;
    a.alpha = alpha; a.grav0 = grav[0]; a.grav1 = grav[1]; a.grav2 = grav[2];
    a.neumann_override = neumann_override; a.has_ext = has_ext; a.g = g;
    k_finalize_grad<<<red_grid(a.n, 4), kRedThreads, 0, st>>>(a, partials, sc);
    counted();
}

// per-DOF energy terms (integrator.cpp:3-42, energy.cpp:229-244)
struct DofEnergyArgs {
    int n;
    const double *q, *qPrev, *vPrev, *mass, *f_ext;
    int has_ext, scheme;
    double dt, alpha, grav0, grav1, grav2;
};

__global__ void __launch_bounds__(kRedThreads) k_dof_energy(DofEnergyArgs a, double* partials, DevScalars* sc) {
    double acc[1] = {0.0};
    double kc, dc;
    if (a.scheme == 0) { kc = 0.5 * a.dt * a.dt; dc = 0.5 * a.alpha * a.dt; }
    else { kc = 0.25 * a.dt * a.dt; dc = 0.25 * a.alpha * a.dt; }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        int node = i / 3, comp = i - 3 * node;
        double m = a.mass[node];
        double gr = comp == 0 ? a.grav0 : (comp == 1 ? a.grav1 : a.grav2);
        double e = -m * a.q[i] * gr;
        if (a.has_ext) e += a.f_ext[i] * (a.q[i] - a.qPrev[i]);
        if (a.dt != 0.0) {
            double v = a.scheme == 0 ? (a.q[i] - a.qPrev[i]) / a.dt : 2.0 * (a.q[i] - a.qPrev[i]) / a.dt - a.vPrev[i];
            double ac = (v - a.vPrev[i]) / a.dt;
            e += kc * m * ac * ac + dc * m * v * v;
        }
        acc[0] += e;
    }
    double tot[1];
    if (reduce_grid<1>(acc, partials, &sc->counters[2], tot) && threadIdx.x == 0) sc->e_dof = tot[0];
}

void launch_dof_energy(int N, const double* q, const double* qPrev, const double* vPrev, const double* mass,
                       const double* f_ext, int has_ext, double dt, int scheme, double alpha, const double* grav,
                       double* partials, DevScalars* sc, cudaStream_t st) {
    DofEnergyArgs a;
    a.n = 3 * N; a.q = q; a.qPrev = qPrev; a.vPrev = vPrev; a.mass = mass; a.f_ext = f_ext; a.has_ext = has_ext;
    a.scheme = scheme; a.dt = dt; a.alpha = alpha; a.grav0 = grav[0]; a.grav1 = grav[1]; a.grav2 = grav[2];
    k_dof_energy<<<red_grid(a.n, 4), kRedThreads, 0, st>>>(a, partials, sc);
    counted();
}

// ---------------------------------------------------------------------------
// block-Jacobi preconditioner: inverse of each 3x3 diagonal block
// ---------------------------------------------------------------------------
template <typename HT, typename VT>
__global__ void k_block_jacobi(int N, const int* row_ptr, const int* diag_slot, const HT* H, long long nnzb,
                               VT* Minv) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const size_t d = (size_t)diag_slot[i];
    double a[9], c[9];
    for (int k = 0; k < 9; k++) a[k] = (double)H[hval(d, k, nnzb)];
    // symmetric part: the lower triangle defines the operator
    a[1] = a[3]; a[2] = a[6]; a[5] = a[7];
    cof3(a, c);
    double det = a[0] * c[0] + a[1] * c[1] + a[2] * c[2];
    VT* o = Minv + (size_t)i * 9;
    if (det != 0.0 && det == det) {
        double id = 1.0 / det;
        for (int r = 0; r < 3; r++)
            for (int cc = 0; cc < 3; cc++) o[r * 3 + cc] = (VT)(c[cc * 3 + r] * id);
    } else {
        for (int k = 0; k < 9; k++) o[k] = (VT)((k % 4 == 0) ? 1.0 : 0.0);
    }
}

template <typename HT, typename VT>
void launch_block_jacobi(int N, const int* row_ptr, const int* diag_slot, const HT* H, long long nnzb, VT* Minv,
                         cudaStream_t st) {
    if (N == 0) return;
    k_block_jacobi<HT, VT><<<(N + 255) / 256, 256, 0, st>>>(N, row_ptr, diag_slot, H, nnzb, Minv);
    counted();
}

// ---------------------------------------------------------------------------
// PCG (block-Jacobi preconditioned CG), FP64 dots
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// Constraint projection for the SQP subproblems: per node a flag byte (bits
// 0-2: DOF held by a Neumann equality, bit 3: contact normal held) and the
// contact normal in pn[i].xyz.  Projects a 3-vector onto the free subspace.
// ---------------------------------------------------------------------------
template <typename VT>
__device__ __forceinline__ void project3(const uint8_t* __restrict__ pflag, const double4* __restrict__ pn, int i,
                                         VT (&y)[3]) {
    if (!pflag) return;
    const unsigned f = __ldg(pflag + i);
    if (!f) return;
    if (f & 1u) y[0] = VT(0);
    if (f & 2u) y[1] = VT(0);
    if (f & 4u) y[2] = VT(0);
    if (f & 8u) {
        const double4 n = pn[i];
        const VT d = (VT)n.x * y[0] + (VT)n.y * y[1] + (VT)n.z * y[2];
        y[0] -= d * (VT)n.x;
        y[1] -= d * (VT)n.y;
        y[2] -= d * (VT)n.z;
    }
}

template <typename VT>
__global__ void __launch_bounds__(kRedThreads) k_pcg_init(int N, const double* g, const VT* Minv, VT* x, VT* r,
                                                           VT* z, VT* p0, double eta2, double abs_tol2, int maxit,
                                                           const uint8_t* pflag, const double4* pn,
                                                           double* partials, DevScalars* sc) {
    double acc[2] = {0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        VT rr[3];
        for (int k = 0; k < 3; k++) {
            rr[k] = (VT)(-g[3 * (size_t)i + k]);
            x[3 * (size_t)i + k] = VT(0);
            p0[4 * (size_t)i + k] = VT(0);
        }
        p0[4 * (size_t)i + 3] = VT(0);
        project3<VT>(pflag, pn, i, rr);
        for (int k = 0; k < 3; k++) r[3 * (size_t)i + k] = rr[k];
        const VT* M = Minv + (size_t)i * 9;
        VT zz[3];
        for (int k = 0; k < 3; k++) zz[k] = M[k * 3 + 0] * rr[0] + M[k * 3 + 1] * rr[1] + M[k * 3 + 2] * rr[2];
        project3<VT>(pflag, pn, i, zz);
        for (int k = 0; k < 3; k++) {
            z[3 * (size_t)i + k] = zz[k];
            acc[0] += (double)rr[k] * (double)zz[k];
            acc[1] += (double)rr[k] * (double)rr[k];
        }
    }
    double tot[2];
    if (reduce_grid<2>(acc, partials, &sc->counters[3], tot) && threadIdx.x == 0) {
        sc->rz = tot[0];
        sc->rr = tot[1];
        sc->bnorm2 = tot[1];
        double t2 = eta2 * tot[1];
        sc->tol2 = t2 > abs_tol2 ? t2 : abs_tol2;
        sc->beta = 0.0;
        sc->it = 0;
        sc->maxit = maxit;
        sc->breakdown = 0;
        sc->counters[4] = 0u;  // SpMV / update reduction sites start clean
        sc->counters[5] = 0u;
        sc->done = (tot[1] <= sc->tol2 || maxit <= 0) ? 1 : 0;
    }
}

template <typename HT, typename VT>
void launch_pcg_init(int N, const double* g, const VT* Minv, VT* x, VT* r, VT* z, VT* p0, double eta2,
                     double abs_tol2, int maxit, const uint8_t* pflag, const double4* pn, double* partials,
                     DevScalars* sc, cudaStream_t st) {
    k_pcg_init<VT><<<red_grid(N, 2), kRedThreads, 0, st>>>(N, g, Minv, x, r, z, p0, eta2, abs_tol2, maxit, pflag,
                                                           pn, partials, sc);
    counted();
}

// The search direction p is stored padded, four values per node (the fourth
// zero), so that a gather of p at a column is one 16-byte load (two for doubles).
template <typename VT>
__device__ __forceinline__ void ld_p4(const VT* __restrict__ p4, size_t i, VT& a, VT& b, VT& c) {
    if constexpr (sizeof(VT) == 4) {
        const float4 t = __ldg(reinterpret_cast<const float4*>(p4) + i);
        a = t.x; b = t.y; c = t.z;
    } else {
        const double2* d = reinterpret_cast<const double2*>(p4) + 2 * i;
        const double2 t0 = __ldg(d), t1 = __ldg(d + 1);
        a = t0.x; b = t0.y; c = t1.x;
    }
}

// p_new = z + beta p_old (padded layout), before the SpMV gathers it.
template <typename VT>
__global__ void __launch_bounds__(kRedThreads) k_form_p(int N, const VT* __restrict__ z, const VT* __restrict__ p_old,
                                                         VT* __restrict__ p_new, const DevScalars* sc) {
    if (*(volatile const int*)&sc->done) return;
    const VT beta = (VT)sc->beta;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        VT a, b, c;
        ld_p4<VT>(p_old, i, a, b, c);
        const size_t k = 3 * (size_t)i;
        a = z[k] + beta * a;
        b = z[k + 1] + beta * b;
        c = z[k + 2] + beta * c;
        if constexpr (sizeof(VT) == 4) {
            reinterpret_cast<float4*>(p_new)[i] = make_float4(a, b, c, 0.0f);
        } else {
            double2* d = reinterpret_cast<double2*>(p_new) + 2 * i;
            d[0] = make_double2(a, b);
            d[1] = make_double2(c, 0.0);
        }
    }
}
template <typename VT>
void launch_form_p(int N, const VT* z, const VT* p_old, VT* p_new, const DevScalars* sc, cudaStream_t st) {
    k_form_p<VT><<<red_grid(N, 2), kRedThreads, 0, st>>>(N, z, p_old, p_new, sc);
    counted();
}

// Nine vector loads of G consecutive 3x3 blocks (9 G values; G * sizeof(HT)
// bytes each): the group of blocks gi starts at 9 G sizeof(HT) gi bytes, a
// multiple of the vector size.
template <typename HT, int G>
__device__ __forceinline__ void load_group(const HT* __restrict__ H, int gi, HT (&hv)[9 * G]) {
    constexpr int VB = G * (int)sizeof(HT);
    if constexpr (VB == 4 || VB == 8 && sizeof(HT) == 8) {
        const HT* src = H + (size_t)gi * 9;
#pragma unroll
        for (int k = 0; k < 9; k++) hv[k] = __ldg(src + k);
    } else if constexpr (VB == 8) {
        const float2* src = reinterpret_cast<const float2*>(H) + (size_t)gi * 9;
#pragma unroll
        for (int k = 0; k < 9; k++) {
            const float2 t = __ldg(src + k);
            hv[2 * k] = t.x; hv[2 * k + 1] = t.y;
        }
    } else if constexpr (sizeof(HT) == 4) {
        const float4* src = reinterpret_cast<const float4*>(H) + (size_t)gi * 9;
#pragma unroll
        for (int k = 0; k < 9; k++) {
            const float4 t = __ldg(src + k);
            hv[4 * k] = t.x; hv[4 * k + 1] = t.y; hv[4 * k + 2] = t.z; hv[4 * k + 3] = t.w;
        }
    } else {
        const double2* src = reinterpret_cast<const double2*>(H) + (size_t)gi * 9;
#pragma unroll
        for (int k = 0; k < 9; k++) {
            const double2 t = __ldg(src + k);
            hv[2 * k] = t.x; hv[2 * k + 1] = t.y;
        }
    }
}

// q = A p with the dot p.q (p formed by k_form_p, padded layout).
// A group of LPR lanes owns one block-row; its lanes take the row's groups of
// G consecutive blocks (the first and last group may hold blocks of the
// neighbouring rows, which the lane skips): nine vector loads of the group's
// values, its G column indices in one load, and one 16-byte gather of p per
// block (two for doubles); the group of lanes is reduced with shuffles.  The
// launcher uses G = 2 (nine 8-byte loads per two FP32 blocks, nine 16-byte
// loads per two FP64 blocks): against one block per lane (nine 4-byte loads)
// 77.5 -> 64.4 us FP32 and 150 -> 123 us FP64; G = 4 (16-byte FP32 loads)
// needs 36 value registers a lane and measured 87-99 us.
// MODE 1 is the MINRES SpMV (minres section below): p4 holds the unnormalised
// z_j, the dot gives delta_j = z_j.A z_j / gamma_j^2 (no curvature test), and
// the lanes that store row i of q also apply the previous iteration's pending
// solution update to row i (MinresUpd).
template <typename VT>
struct MinresUpd {
    const VT* zprev = nullptr;  // z_{j-1}, padded
    const VT* wread = nullptr;  // w_{j-1}
    VT* wrw = nullptr;          // w_{j-2} in, w_j out
    VT* x = nullptr;
};

template <typename VT>
__device__ __forceinline__ void minres_row_update(const MinresUpd<VT>& u, size_t row, int d, VT ig, VT a1i, VT a2,
                                                  VT a3, VT ceta) {
    const size_t k = 3 * row + d;
    const VT wn = (u.zprev[4 * row + d] * ig - a3 * u.wrw[k] - a2 * u.wread[k]) * a1i;
    u.wrw[k] = wn;
    u.x[k] += ceta * wn;
}

template <typename HT, typename VT, int LPR, int G, int MODE = 0>
__global__ void __launch_bounds__(kRedThreads, sizeof(HT) == 4 ? 8 : 4) k_pcg_spmv(
    int N, const int* __restrict__ row_ptr, const int* __restrict__ col, const HT* __restrict__ H, long long nnzb,
    const VT* __restrict__ p4, VT* __restrict__ qv, double* partials, DevScalars* sc, MinresUpd<VT> mu) {
    (void)nnzb;
    if (*(volatile int*)&sc->done) return;
    // (named apart from the row sums a0..a2 below)
    bool pend = false;
    VT u_ig = VT(0), u_a1i = VT(0), u_a2 = VT(0), u_a3 = VT(0), u_ceta = VT(0);
    if constexpr (MODE == 1) {
        pend = *(volatile int*)&sc->mr_pending != 0;
        if (pend) {
            u_ig = (VT)sc->mr_ig; u_a1i = (VT)(1.0 / sc->mr_a1); u_a2 = (VT)sc->mr_a2; u_a3 = (VT)sc->mr_a3;
            u_ceta = (VT)sc->mr_ceta;
        }
    }
    const int lane = threadIdx.x & 31;
    const int sub = lane / LPR, sl = lane % LPR;
    constexpr int RPW = 32 / LPR;
    const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    double acc[1] = {0.0};
    for (int base = gwarp * RPW; base < N; base += nwarps * RPW) {
        const int row = base + sub;
        VT a0 = VT(0), a1 = VT(0), a2 = VT(0);
        if (row < N) {
            const int b0 = __ldg(row_ptr + row), b1 = __ldg(row_ptr + row + 1);
            const int g0 = b0 / G, g1 = (b1 - 1) / G;
            for (int gi = g0 + sl; gi <= g1; gi += LPR) {
                HT hv[9 * G];
                load_group<HT, G>(H, gi, hv);
                auto blk = [&](const int u, const int j) {
                    const int b = gi * G + u;
                    if (G > 1 && (b < b0 || b >= b1)) return;
                    VT p0, p1, p2;
                    ld_p4<VT>(p4, (size_t)j, p0, p1, p2);
                    a0 += (VT)hv[9 * u] * p0 + (VT)hv[9 * u + 1] * p1 + (VT)hv[9 * u + 2] * p2;
                    a1 += (VT)hv[9 * u + 3] * p0 + (VT)hv[9 * u + 4] * p1 + (VT)hv[9 * u + 5] * p2;
                    a2 += (VT)hv[9 * u + 6] * p0 + (VT)hv[9 * u + 7] * p1 + (VT)hv[9 * u + 8] * p2;
                };
                if constexpr (G == 4) {
                    const int4 c4 = __ldg(reinterpret_cast<const int4*>(col) + gi);
                    blk(0, c4.x);
                    blk(1, c4.y);
                    blk(2, c4.z);
                    blk(3, c4.w);
                } else if constexpr (G == 2) {
                    const int2 c2 = __ldg(reinterpret_cast<const int2*>(col) + gi);
                    blk(0, c2.x);
                    blk(1, c2.y);
                } else {
                    blk(0, __ldg(col + gi));
                }
            }
        }
#pragma unroll
        for (int o = LPR / 2; o > 0; o >>= 1) {
            a0 += __shfl_xor_sync(0xffffffffu, a0, o);
            a1 += __shfl_xor_sync(0xffffffffu, a1, o);
            a2 += __shfl_xor_sync(0xffffffffu, a2, o);
        }
        if (row < N && sl < 3) {
            const VT qi = sl == 0 ? a0 : (sl == 1 ? a1 : a2);
            qv[3 * (size_t)row + sl] = qi;
            acc[0] += (double)p4[4 * (size_t)row + sl] * (double)qi;
            if constexpr (MODE == 1)
                if (pend) minres_row_update<VT>(mu, (size_t)row, sl, u_ig, u_a1i, u_a2, u_a3, u_ceta);
        }
    }
    double tot[1];
    if (reduce_grid<1>(acc, partials, &sc->counters[4], tot) && threadIdx.x == 0) {
        if constexpr (MODE == 1) {
            sc->pq = tot[0];
            sc->mr_delta = tot[0] / (sc->mr_g * sc->mr_g);
            return;
        }
        sc->pq = tot[0];
        if (!(tot[0] > 0.0)) {
            sc->breakdown = 1;
            sc->done = 1;
            sc->alpha = 0.0;
        } else {
            sc->alpha = sc->rz / tot[0];
        }
    }
}

template <typename HT, typename VT, int G, int MODE = 0>
static void launch_spmv_g(int N, int max_row_blocks, const int* row_ptr, const int* col, const HT* H,
                          long long nnzb, const VT* p4, VT* qv, double* partials, DevScalars* sc, cudaStream_t st,
                          MinresUpd<VT> mu = MinresUpd<VT>()) {
    // groups a row of max_row_blocks blocks can span, rounded up to a power of two
    const int groups = G == 1 ? max_row_blocks : (max_row_blocks + 2 * G - 2) / G;
    const int lpr = groups <= 2 ? 2 : (groups <= 4 ? 4 : (groups <= 8 ? 8 : (groups <= 16 ? 16 : 32)));
    const int rows_per_block = (kRedThreads / 32) * (32 / lpr);
    long long blocks = (N + rows_per_block - 1) / rows_per_block;
    if (blocks > kRedBlocks) blocks = kRedBlocks;
    if (blocks < 1) blocks = 1;
    blocks = cap_grid(blocks);
    switch (lpr) {
        case 2: k_pcg_spmv<HT, VT, 2, G, MODE><<<(int)blocks, kRedThreads, 0, st>>>(N, row_ptr, col, H, nnzb, p4, qv, partials, sc, mu); break;
        case 4: k_pcg_spmv<HT, VT, 4, G, MODE><<<(int)blocks, kRedThreads, 0, st>>>(N, row_ptr, col, H, nnzb, p4, qv, partials, sc, mu); break;
        case 8: k_pcg_spmv<HT, VT, 8, G, MODE><<<(int)blocks, kRedThreads, 0, st>>>(N, row_ptr, col, H, nnzb, p4, qv, partials, sc, mu); break;
        case 16: k_pcg_spmv<HT, VT, 16, G, MODE><<<(int)blocks, kRedThreads, 0, st>>>(N, row_ptr, col, H, nnzb, p4, qv, partials, sc, mu); break;
        default: k_pcg_spmv<HT, VT, 32, G, MODE><<<(int)blocks, kRedThreads, 0, st>>>(N, row_ptr, col, H, nnzb, p4, qv, partials, sc, mu); break;
    }
    counted();
}

template <typename HT, typename VT>
void launch_pcg_spmv(int N, int max_row_blocks, const int* row_ptr, const int* col, const HT* H, long long nnzb,
                     const VT* p4, VT* qv, double* partials, DevScalars* sc, cudaStream_t st) {
    launch_spmv_g<HT, VT, 2>(N, max_row_blocks, row_ptr, col, H, nnzb, p4, qv, partials, sc, st);
}

template <typename VT>
__global__ void __launch_bounds__(kRedThreads) k_pcg_update(int N, const VT* __restrict__ p, const VT* __restrict__ qv,
                                                             const VT* __restrict__ Minv, VT* __restrict__ x,
                                                             VT* __restrict__ r, VT* __restrict__ z,
                                                             const uint8_t* __restrict__ pflag,
                                                             const double4* __restrict__ pn, double* partials,
                                                             DevScalars* sc) {
    if (*(volatile int*)&sc->done) return;
    const VT alpha = (VT)sc->alpha;
    double acc[2] = {0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        VT rr[3], qq[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const size_t ii = 3 * (size_t)i + k;
            x[ii] += alpha * p[4 * (size_t)i + k];
            qq[k] = qv[ii];
        }
        project3<VT>(pflag, pn, i, qq);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const size_t ii = 3 * (size_t)i + k;
            rr[k] = r[ii] - alpha * qq[k];
            r[ii] = rr[k];
        }
        const VT* M = Minv + (size_t)i * 9;
        VT zz[3];
#pragma unroll
        for (int k = 0; k < 3; k++) zz[k] = M[k * 3 + 0] * rr[0] + M[k * 3 + 1] * rr[1] + M[k * 3 + 2] * rr[2];
        project3<VT>(pflag, pn, i, zz);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            z[3 * (size_t)i + k] = zz[k];
            acc[0] += (double)rr[k] * (double)zz[k];
            acc[1] += (double)rr[k] * (double)rr[k];
        }
    }
    double tot[2];
    if (reduce_grid<2>(acc, partials, &sc->counters[5], tot) && threadIdx.x == 0) {
        sc->beta = tot[0] / sc->rz;
        sc->rz = tot[0];
        sc->rr = tot[1];
        sc->it += 1;
        if (tot[1] <= sc->tol2 || sc->it >= sc->maxit || !(tot[1] == tot[1])) sc->done = 1;
    }
}

template <typename VT>
void launch_pcg_update(int N, const VT* p, const VT* qv, const VT* Minv, VT* x, VT* r, VT* z, const uint8_t* pflag,
                       const double4* pn, double* partials, DevScalars* sc, cudaStream_t st) {
    k_pcg_update<VT><<<red_grid(N, 2), kRedThreads, 0, st>>>(N, p, qv, Minv, x, r, z, pflag, pn, partials, sc);
    counted();
}

// ---------------------------------------------------------------------------
// Newton update q = q0 + alpha dx, ||alpha dx||^2; g.dx; update_state
// ---------------------------------------------------------------------------
template <typename VT>
__global__ void __launch_bounds__(kRedThreads) k_newton_update(int n, const VT* dx, double alpha, double* q,
                                                                const double* q0, double* partials, DevScalars* sc,
                                                                int counter) {
    double acc[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double d = alpha * (double)dx[i];
        q[i] = q0[i] + d;
        acc[0] += d * d;
    }
    double tot[1];
    if (reduce_grid<1>(acc, partials, &sc->counters[counter], tot) && threadIdx.x == 0) sc->dxnorm2 = tot[0];
}

template <typename VT>
void launch_newton_update(int n, const VT* dx, double alpha, double* q, const double* q0, double* partials,
                          DevScalars* sc, int counter, cudaStream_t st) {
    k_newton_update<VT><<<red_grid(n, 4), kRedThreads, 0, st>>>(n, dx, alpha, q, q0, partials, sc, counter);
    counted();
}

template <typename VT>
__global__ void __launch_bounds__(kRedThreads) k_dot_gdx(int n, const double* g, const VT* dx, double* partials,
                                                          DevScalars* sc) {
    double acc[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) acc[0] += g[i] * (double)dx[i];
    double tot[1];
    if (reduce_grid<1>(acc, partials, &sc->counters[7], tot) && threadIdx.x == 0) sc->gdx = tot[0];
}

template <typename VT>
void launch_dot_gdx(int n, const double* g, const VT* dx, double* partials, DevScalars* sc, cudaStream_t st) {
    k_dot_gdx<VT><<<red_grid(n, 4), kRedThreads, 0, st>>>(n, g, dx, partials, sc);
    counted();
}

__global__ void k_update_state(int n, const double* q, double* qPrev, double* vPrev, double* gPrev,
                               const double* gPrevTmp, double dt, int scheme) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v = scheme == 0 ? (q[i] - qPrev[i]) / dt : 2.0 * (q[i] - qPrev[i]) / dt - vPrev[i];
    vPrev[i] = v;
    qPrev[i] = q[i];
    gPrev[i] = gPrevTmp[i];
}

void launch_update_state(int n, const double* q, double* qPrev, double* vPrev, double* gPrev,
                         const double* gPrevTmp, double dt, int scheme, cudaStream_t st) {
    if (n == 0) return;
    k_update_state<<<(n + 255) / 256, 256, 0, st>>>(n, q, qPrev, vPrev, gPrev, gPrevTmp, dt, scheme);
    counted();
}

// Newton predictor q += dt v_prev
// CFL time step inputs (cpp/src/solver.cpp:300-331): the shortest edge of any
// element at q, over every vertex pair (Element::compute_minimal_edge_length,
// cpp/headers/geometries/element.h:131-142), and max |vPrev|.  Minimum and
// maximum do not depend on the order of evaluation, so the result is the
// reference loop's exactly.  sc->minedge, sc->vmax.
__global__ void __launch_bounds__(kRedThreads) k_cfl(int E, int nv, const double* __restrict__ q,
                                                     const int* __restrict__ conn, int n,
                                                     const double* __restrict__ vPrev, double* partials,
                                                     DevScalars* sc) {
    __shared__ double sh[32][2];
    __shared__ bool am_last;
    double lmin = INFINITY, vmax = 0.0;
    const int stride = gridDim.x * blockDim.x;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += stride) {
        double x[8][3];
        for (int w = 0; w < nv; w++) {
            const int v = __ldg(conn + (size_t)e * nv + w);
#pragma unroll
            for (int r = 0; r < 3; r++) x[w][r] = q[3 * (size_t)v + r];
        }
        for (int i = 0; i < nv; i++)
            for (int j = i + 1; j < nv; j++) {
                const double d0 = x[i][0] - x[j][0], d1 = x[i][1] - x[j][1], d2 = x[i][2] - x[j][2];
                lmin = fmin(lmin, sqrt(d0 * d0 + d1 * d1 + d2 * d2));
            }
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) vmax = fmax(vmax, fabs(vPrev[i]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lmin = fmin(lmin, __shfl_xor_sync(0xffffffffu, lmin, o));
        vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
    if (l == 0) { sh[w][0] = lmin; sh[w][1] = vmax; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < nw; k++) { lmin = fmin(lmin, sh[k][0]); vmax = fmax(vmax, sh[k][1]); }
        partials[2 * blockIdx.x] = lmin;
        partials[2 * blockIdx.x + 1] = vmax;
        __threadfence();
        am_last = (atomicAdd(&sc->counters[10], 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!am_last || threadIdx.x != 0) return;
    __threadfence();
    const volatile double* vp = partials;
    double a = INFINITY, b = 0.0;
    for (int k = 0; k < (int)gridDim.x; k++) { a = fmin(a, vp[2 * k]); b = fmax(b, vp[2 * k + 1]); }
    sc->minedge = a;
    sc->vmax = b;
    sc->counters[10] = 0u;
}

void launch_cfl(int E, int nv, const double* q, const int* conn, int n, const double* vPrev, double* partials,
                DevScalars* sc, cudaStream_t st) {
    k_cfl<<<red_grid(E > n ? E : n), kRedThreads, 0, st>>>(E, nv, q, conn, n, vPrev, partials, sc);
    counted();
}

// dst[3i + k] = src[3 idx[i] + k]: DOF vectors between the caller's node
// numbering and the handle's (idx is the permutation in one direction or the other)
__global__ void k_gather_dofs(int N, const double* __restrict__ src, const int* __restrict__ idx,
                              double* __restrict__ dst) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 3 * N; t += gridDim.x * blockDim.x) {
        const int i = t / 3, k = t - 3 * i;
        dst[t] = src[3 * (size_t)__ldg(idx + i) + k];
    }
}

void launch_gather_dofs(int N, const double* src, const int* idx, double* dst, cudaStream_t st) {
    if (N == 0) return;
    k_gather_dofs<<<red_grid(3LL * N), kRedThreads, 0, st>>>(N, src, idx, dst);
    counted();
}

__global__ void k_predict(int n, double* q, const double* vPrev, double dt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) q[i] += dt * vPrev[i];
}

void launch_predict(int n, double* q, const double* vPrev, double dt, cudaStream_t st) {
    if (n == 0) return;
    k_predict<<<(n + 255) / 256, 256, 0, st>>>(n, q, vPrev, dt);
    counted();
}

// y = H x (tests / diagnostics)
template <typename HT>
__global__ void k_spmv_plain(int N, const int* row_ptr, const int* col, const HT* H, long long nnzb, const double* x,
                             double* y) {
    int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    int lane = threadIdx.x & 31;
    if (row >= N) return;
    int b0 = row_ptr[row], nval = (row_ptr[row + 1] - b0) * 9;
    double a[3] = {0, 0, 0};
    // t runs over (block of the row, entry of the block)
    for (int t = lane; t < nval; t += 32) {
        int blk = t / 9, rc = t - blk * 9, r = rc / 3, c = rc - r * 3;
        double pr = (double)H[hval((size_t)b0 + blk, rc, nnzb)] * x[3 * (size_t)col[b0 + blk] + c];
        a[0] += r == 0 ? pr : 0.0; a[1] += r == 1 ? pr : 0.0; a[2] += r == 2 ? pr : 0.0;
    }
    warp_sum<3>(a);
    if (lane < 3) y[3 * (size_t)row + lane] = a[lane];
}

template <typename HT>
void launch_spmv_plain(int N, const int* row_ptr, const int* col, const HT* H, long long nnzb, const double* x,
                       double* y, cudaStream_t st) {
    if (N == 0) return;
    k_spmv_plain<HT><<<(N + 7) / 8, 256, 0, st>>>(N, row_ptr, col, H, nnzb, x, y);
    counted();
}

// ---------------------------------------------------------------------------
// SQP subproblem helpers (minimize_SQP)
// ---------------------------------------------------------------------------
// Particular solution of the working constraints: Neumann DOFs move to their
// prescribed position, dx_i = -(q_i - qPrev_i - dt val_i) (neumannBC.cpp:4-21),
// contact nodes move by b along their normal (pn.w = b); zero elsewhere.
__global__ void k_qp_x0(int N, const uint8_t* __restrict__ pflag, const double4* __restrict__ pn,
                        const double* __restrict__ q, const double* __restrict__ qPrev,
                        const double* __restrict__ mval, double dt, double* __restrict__ x0) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const unsigned f = pflag[i];
    double x[3] = {0.0, 0.0, 0.0};
    if (f & 8u) {
        const double4 n = pn[i];
        x[0] = n.w * n.x; x[1] = n.w * n.y; x[2] = n.w * n.z;
    }
#pragma unroll
    for (int k = 0; k < 3; k++)
        if ((f >> k) & 1u) {
            const size_t ii = 3 * (size_t)i + k;
            x[k] = -(q[ii] - qPrev[ii] - dt * mval[ii]);
        }
#pragma unroll
    for (int k = 0; k < 3; k++) x0[3 * (size_t)i + k] = x[k];
}

// Warm start for a re-solve after the working set changed: the previous step
// dx with the constraints of the new working set imposed again (Neumann DOFs
// at their target, held contact nodes moved to their bound along the normal,
// tangential motion kept).
__global__ void k_qp_warm(int N, const uint8_t* __restrict__ pflag, const double4* __restrict__ pn,
                          const double* __restrict__ q, const double* __restrict__ qPrev,
                          const double* __restrict__ mval, double dt, const double* __restrict__ dx_prev,
                          double* __restrict__ x0) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const unsigned f = pflag[i];
    double x[3];
#pragma unroll
    for (int k = 0; k < 3; k++) x[k] = dx_prev[3 * (size_t)i + k];
    if (f & 8u) {
        const double4 n = pn[i];
        const double d = n.w - (n.x * x[0] + n.y * x[1] + n.z * x[2]);
        x[0] += d * n.x; x[1] += d * n.y; x[2] += d * n.z;
    }
#pragma unroll
    for (int k = 0; k < 3; k++)
        if ((f >> k) & 1u) {
            const size_t ii = 3 * (size_t)i + k;
            x[k] = -(q[ii] - qPrev[ii] - dt * mval[ii]);
        }
#pragma unroll
    for (int k = 0; k < 3; k++) x0[3 * (size_t)i + k] = x[k];
}

void launch_qp_warm(int N, const uint8_t* pflag, const double4* pn, const double* q, const double* qPrev,
                    const double* mval, double dt, const double* dx_prev, double* x0, cudaStream_t st) {
    k_qp_warm<<<(N + 255) / 256, 256, 0, st>>>(N, pflag, pn, q, qPrev, mval, dt, dx_prev, x0);
    counted();
}

// out = a + b (b of the PCG vector type)
template <typename VT>
__global__ void k_add_vec(int n, const double* __restrict__ a, const VT* __restrict__ b, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = a[i] + (double)b[i];
}

// Per contact constraint c at node v with normal n and bound b:
// slack = n.dx_v - b (>= 0 when satisfied), mu = n.(H dx + g)_v (the multiplier
// when the constraint is held).  cnb[c] = (n, b).
__global__ void k_qp_check(int m, const int* __restrict__ cnode, const double4* __restrict__ cnb,
                           const double* __restrict__ dx, const double* __restrict__ y, const double* __restrict__ g,
                           double* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m) return;
    const int v = cnode[c];
    const double4 n = cnb[c];
    const size_t b = 3 * (size_t)v;
    out[c] = n.x * dx[b] + n.y * dx[b + 1] + n.z * dx[b + 2] - n.w;
    out[(size_t)m + c] = n.x * (y[b] + g[b]) + n.y * (y[b + 1] + g[b + 1]) + n.z * (y[b + 2] + g[b + 2]);
}

// out[3c + k] = q[3 node_c + k]
__global__ void k_gather_nodes(int m, const int* __restrict__ node, const double* __restrict__ q,
                               double* __restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * m) return;
    const int c = t / 3, k = t - 3 * c;
    out[t] = q[3 * (size_t)node[c] + k];
}

// Max-distance rows a_p = (-n_p at node i_p, +n_p at node j_p): y += s_p a_p for
// every listed pair, coef[p] = (n_p, s_p).  Pairs may share nodes, so one
// thread walks them in order (a handful of pairs; deterministic).
__global__ void k_pair_axpy(int np, const int2* __restrict__ ij, const double4* __restrict__ coef,
                            double* __restrict__ y) {
    if (blockIdx.x || threadIdx.x) return;
    for (int p = 0; p < np; p++) {
        const int2 e = ij[p];
        const double4 c = coef[p];
        const size_t a = 3 * (size_t)e.x, b = 3 * (size_t)e.y;
        y[a] -= c.w * c.x; y[a + 1] -= c.w * c.y; y[a + 2] -= c.w * c.z;
        y[b] += c.w * c.x; y[b + 1] += c.w * c.y; y[b + 2] += c.w * c.z;
    }
}

// y += alpha x
__global__ void k_axpy(int n, double alpha, const double* __restrict__ x, double* __restrict__ y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] += alpha * x[i];
}

void launch_pair_axpy(int np, const int2* ij, const double4* coef, double* y, cudaStream_t st) {
    if (np == 0) return;
    k_pair_axpy<<<1, 1, 0, st>>>(np, ij, coef, y);
    counted();
}
void launch_axpy(int n, double alpha, const double* x, double* y, cudaStream_t st) {
    k_axpy<<<(n + 255) / 256, 256, 0, st>>>(n, alpha, x, y);
    counted();
}

void launch_qp_x0(int N, const uint8_t* pflag, const double4* pn, const double* q, const double* qPrev,
                  const double* mval, double dt, double* x0, cudaStream_t st) {
    k_qp_x0<<<(N + 255) / 256, 256, 0, st>>>(N, pflag, pn, q, qPrev, mval, dt, x0);
    counted();
}
template <typename VT>
void launch_add_vec(int n, const double* a, const VT* b, double* out, cudaStream_t st) {
    k_add_vec<VT><<<(n + 255) / 256, 256, 0, st>>>(n, a, b, out);
    counted();
}
void launch_qp_check(int m, const int* cnode, const double4* cnb, const double* dx, const double* y,
                     const double* g, double* out, cudaStream_t st) {
    if (m == 0) return;
    k_qp_check<<<(m + 127) / 128, 128, 0, st>>>(m, cnode, cnb, dx, y, g, out);
    counted();
}
void launch_gather_nodes(int m, const int* node, const double* q, double* out, cudaStream_t st) {
    if (m == 0) return;
    k_gather_nodes<<<(3 * m + 255) / 256, 256, 0, st>>>(m, node, q, out);
    counted();
}
template void launch_add_vec<double>(int, const double*, const double*, double*, cudaStream_t);
template void launch_add_vec<float>(int, const double*, const float*, double*, cudaStream_t);

// ---------------------------------------------------------------------------
// Two-level preconditioner
// ---------------------------------------------------------------------------
// Column m of P_i (3 values): translation e_m (m < 3) or rotation
// e_{m-3} x (X_i - c) s (m >= 3); rows of Neumann-held DOFs are zero.
__device__ __forceinline__ void coarse_col(const CoarseArgs& c, int i, int m, double (&u)[3]) {
    if (m < 3) {
        u[0] = m == 0; u[1] = m == 1; u[2] = m == 2;
    } else {
        const float4 o = c.off[i];
        const double dx = o.x, dy = o.y, dz = o.z;
        if (m == 3) { u[0] = 0.0; u[1] = -dz; u[2] = dy; }
        else if (m == 4) { u[0] = dz; u[1] = 0.0; u[2] = -dx; }
        else { u[0] = -dy; u[1] = dx; u[2] = 0.0; }
    }
    if (c.fixed) {
        const unsigned f = c.fixed[i];
        if (f & 1u) u[0] = 0.0;
        if (f & 2u) u[1] = 0.0;
        if (f & 4u) u[2] = 0.0;
    }
}

// P_i^T v (6 values) and P_i w (3 values) for one node, from its offset.
__device__ __forceinline__ void coarse_restrict_node(const CoarseArgs& c, int i, const double (&v)[3],
                                                     double (&y)[6]) {
    double w[3] = {v[0], v[1], v[2]};
    if (c.fixed) {
        const unsigned f = c.fixed[i];
        if (f & 1u) w[0] = 0.0;
        if (f & 2u) w[1] = 0.0;
        if (f & 4u) w[2] = 0.0;
    }
    const float4 o = c.off[i];
    const double dx = o.x, dy = o.y, dz = o.z;
    y[0] = w[0]; y[1] = w[1]; y[2] = w[2];
    y[3] = -dz * w[1] + dy * w[2];
    y[4] = dz * w[0] - dx * w[2];
    y[5] = -dy * w[0] + dx * w[1];
}

// Ac = P^T H P: one block per aggregate pair (a, b); thread (r, c) sums
// P_i[:, r]^T H_ij P_j[:, c] over the Hessian blocks (i in a, j in b) in the
// fixed order of the pair's item list.
template <typename HT>
__global__ void k_coarse_galerkin(int npairs, const int* __restrict__ cpair_ptr, const int2* __restrict__ items,
                                  const int2* __restrict__ ab, const int* __restrict__ col,
                                  const HT* __restrict__ H, long long nnzb, CoarseArgs c, double* __restrict__ Ac) {
    const int pr = blockIdx.x;
    const int t = threadIdx.x;
    if (pr >= npairs || t >= 36) return;
    const int r = t / 6, cc = t - 6 * (t / 6);
    const int2 pab = ab[pr];
    double acc = 0.0;
    for (int it = cpair_ptr[pr]; it < cpair_ptr[pr + 1]; it++) {
        const int2 bi = items[it];
        const int bg = bi.x, i = bi.y, j = __ldg(col + bg);
        double u[3], w[3];
        coarse_col(c, i, r, u);
        coarse_col(c, j, cc, w);
        const HT* hb = H + hval((size_t)bg, 0, (size_t)nnzb);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const double hw = (double)hb[k * 3] * w[0] + (double)hb[k * 3 + 1] * w[1] + (double)hb[k * 3 + 2] * w[2];
            acc += u[k] * hw;
        }
    }
    Ac[(size_t)(6 * pab.x + r) * c.nc + 6 * pab.y + cc] = acc;
}

void launch_coarse_galerkin_f(int npairs, const int* cpair_ptr, const int2* cpair_items, const int2* cpair_ab,
                              const int* col, const float* H, long long nnzb, const CoarseArgs& c, double* Ac,
                              cudaStream_t st) {
    if (npairs == 0) return;
    k_coarse_galerkin<float><<<npairs, 64, 0, st>>>(npairs, cpair_ptr, cpair_items, cpair_ab, col, H, nnzb, c, Ac);
    counted();
}
void launch_coarse_galerkin_d(int npairs, const int* cpair_ptr, const int2* cpair_items, const int2* cpair_ab,
                              const int* col, const double* H, long long nnzb, const CoarseArgs& c, double* Ac,
                              cudaStream_t st) {
    if (npairs == 0) return;
    k_coarse_galerkin<double><<<npairs, 64, 0, st>>>(npairs, cpair_ptr, cpair_items, cpair_ab, col, H, nnzb, c, Ac);
    counted();
}

// Coarse unknowns with (near-)zero diagonal (an aggregate held entirely by
// Neumann DOFs) become identity rows, so the inverse exists.
__global__ void k_coarse_fix(int nc, double* Ac) {
    __shared__ double smax[256];
    double m = 0.0;
    for (int k = threadIdx.x; k < nc; k += blockDim.x) m = fmax(m, fabs(Ac[(size_t)k * nc + k]));
    smax[threadIdx.x] = m;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) smax[threadIdx.x] = fmax(smax[threadIdx.x], smax[threadIdx.x + o]);
        __syncthreads();
    }
    const double tiny = 1e-12 * smax[0];
    for (int k = 0; k < nc; k++) {
        if (fabs(Ac[(size_t)k * nc + k]) > tiny) continue;
        for (int j = threadIdx.x; j < nc; j += blockDim.x) {
            Ac[(size_t)k * nc + j] = 0.0;
            Ac[(size_t)j * nc + k] = 0.0;
        }
        __syncthreads();
        if (threadIdx.x == 0) Ac[(size_t)k * nc + k] = 1.0;
        __syncthreads();
    }
}

// In-place Gauss-Jordan inversion of the SPD coarse matrix, one pivot per pair
// of launches: copy pivot row and column, then update every entry from the copies.
__global__ void k_gj_copy(int nc, const double* __restrict__ A, int k, double* __restrict__ rowk,
                          double* __restrict__ colk) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nc) return;
    rowk[j] = A[(size_t)k * nc + j];
    colk[j] = A[(size_t)j * nc + k];
}

__global__ void k_gj_update(int nc, double* __restrict__ A, int k, const double* __restrict__ rowk,
                            const double* __restrict__ colk) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)nc * nc) return;
    const int i = (int)(t / nc), j = (int)(t - (long long)i * nc);
    const double p = rowk[k];
    double v;
    if (i == k && j == k) v = 1.0 / p;
    else if (i == k) v = rowk[j] / p;
    else if (j == k) v = -colk[i] / p;
    else v = A[t] - colk[i] * rowk[j] / p;
    A[t] = v;
}

void launch_coarse_invert(int nc, double* Ac, double* rowk, double* colk, cudaStream_t st) {
    if (nc == 0) return;
    k_coarse_fix<<<1, 256, 0, st>>>(nc, Ac);
    counted();
    const long long n2 = (long long)nc * nc;
    const int bu = (int)((n2 + 255) / 256), bc = (nc + 255) / 256;
    for (int k = 0; k < nc; k++) {
        k_gj_copy<<<bc, 256, 0, st>>>(nc, Ac, k, rowk, colk);
        k_gj_update<<<bu, 256, 0, st>>>(nc, Ac, k, rowk, colk);
    }
    g_kernel_launches.fetch_add(2LL * nc);
}

// yc = P^T r: one block per aggregate, a fixed-order tree sum.  The fused
// variant first applies the CG update x += alpha p, r -= alpha P q to the
// aggregate's nodes (each node belongs to exactly one aggregate).
constexpr int kAggThreads = 256;  // threads per aggregate block

template <typename VT, bool UPDATE>
__global__ void __launch_bounds__(kAggThreads) k_coarse_restrict(CoarseArgs c, const VT* __restrict__ p,
                                                                 const VT* __restrict__ qv, VT* __restrict__ x,
                                                                 VT* __restrict__ r, const uint8_t* __restrict__ pflag,
                                                                 const double4* __restrict__ pn,
                                                                 double* __restrict__ yc, const DevScalars* sc) {
    if (UPDATE && *(volatile const int*)&sc->done) return;
    __shared__ double sh[32][6];
    const int a = blockIdx.x;
    const VT alpha = UPDATE ? (VT)sc->alpha : VT(0);
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int k = c.agg_ptr[a] + threadIdx.x; k < c.agg_ptr[a + 1]; k += blockDim.x) {
        const int i = c.agg_nodes[k];
        double ri[3];
        if (UPDATE) {
            VT qq[3], rr[3];
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const size_t ii = 3 * (size_t)i + d;
                x[ii] += alpha * p[4 * (size_t)i + d];
                qq[d] = qv[ii];
            }
            project3<VT>(pflag, pn, i, qq);
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const size_t ii = 3 * (size_t)i + d;
                rr[d] = r[ii] - alpha * qq[d];
                r[ii] = rr[d];
                ri[d] = (double)rr[d];
            }
        } else {
#pragma unroll
            for (int d = 0; d < 3; d++) ri[d] = (double)r[3 * (size_t)i + d];
        }
        double y[6];
        coarse_restrict_node(c, i, ri, y);
#pragma unroll
        for (int m = 0; m < 6; m++) acc[m] += y[m];
    }
    block_sum<6>(acc, sh);
    if (threadIdx.x == 0)
#pragma unroll
        for (int m = 0; m < 6; m++) yc[6 * a + m] = acc[m];
}
template <typename VT>
void launch_coarse_restrict(const CoarseArgs& c, const VT* r, double* yc, cudaStream_t st) {
    if (c.nagg == 0) return;
    k_coarse_restrict<VT, false><<<c.nagg, kAggThreads, 0, st>>>(c, nullptr, nullptr, nullptr, const_cast<VT*>(r),
                                                                  nullptr, nullptr, yc, nullptr);
    counted();
}
template <typename VT>
void launch_tl_update_restrict(const CoarseArgs& c, const VT* p, const VT* qv, VT* x, VT* r, const uint8_t* pflag,
                               const double4* pn, double* yc, DevScalars* sc, cudaStream_t st) {
    k_coarse_restrict<VT, true><<<c.nagg, kAggThreads, 0, st>>>(c, p, qv, x, r, pflag, pn, yc, sc);
    counted();
}

// The same update and restriction when every aggregate is a contiguous node
// range (the locality numbering makes it so): one node per thread in blocks of
// kRunThreads consecutive nodes, so the whole grid works on it.  A block's
// nodes fall into runs of one aggregate (cut at block ends); each run is
// summed in a fixed order by one warp into its partial slot, and the last
// block to finish sums each aggregate's consecutive runs into yc.
constexpr int kRunThreads = 256;

template <typename VT>
__global__ void __launch_bounds__(kRunThreads) k_tl_update_restrict_runs(CoarseArgs c, CoarseRuns ru,
                                                                        const VT* __restrict__ p,
                                                                        const VT* __restrict__ qv, VT* __restrict__ x,
                                                                        VT* __restrict__ r,
                                                                        const uint8_t* __restrict__ pflag,
                                                                        const double4* __restrict__ pn,
                                                                        const DevScalars* sc) {
    if (*(volatile const int*)&sc->done) return;
    __shared__ double ys[kRunThreads][6];
    const int i = blockIdx.x * kRunThreads + threadIdx.x;
    double y[6] = {0, 0, 0, 0, 0, 0};
    if (i < c.N) {
        const VT alpha = (VT)sc->alpha;
        VT qq[3], rr[3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const size_t ii = 3 * (size_t)i + d;
            x[ii] += alpha * p[4 * (size_t)i + d];
            qq[d] = qv[ii];
        }
        project3<VT>(pflag, pn, i, qq);
        double ri[3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const size_t ii = 3 * (size_t)i + d;
            rr[d] = r[ii] - alpha * qq[d];
            r[ii] = rr[d];
            ri[d] = (double)rr[d];
        }
        coarse_restrict_node(c, i, ri, y);
    }
#pragma unroll
    for (int m = 0; m < 6; m++) ys[threadIdx.x][m] = y[m];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int node0 = blockIdx.x * kRunThreads;
    for (int k = ru.block_run_ptr[blockIdx.x] + warp; k < ru.block_run_ptr[blockIdx.x + 1]; k += kRunThreads / 32) {
        const int s0 = ru.run_start[k] - node0, s1 = ru.run_start[k + 1] - node0;
        double acc[6] = {0, 0, 0, 0, 0, 0};
        for (int t = s0 + lane; t < s1; t += 32)
#pragma unroll
            for (int m = 0; m < 6; m++) acc[m] += ys[t][m];
        warp_sum<6>(acc);
        if (lane == 0)
#pragma unroll
            for (int m = 0; m < 6; m++) ru.partial[6 * (size_t)k + m] = acc[m];
    }
}

// yc[6a + m] = the sum of aggregate a's run partials, in run order.
__global__ void k_tl_restrict_finalize(int nagg, CoarseRuns ru, double* __restrict__ yc, const DevScalars* sc) {
    if (*(volatile const int*)&sc->done) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 6 * nagg) return;
    const int a = t / 6, m = t - 6 * (t / 6);
    const int k0 = __ldg(ru.agg_run_begin + a), k1 = __ldg(ru.agg_run_begin + a + 1);
    double acc = 0.0;
    for (int k = k0; k < k1; k++) acc += ru.partial[6 * (size_t)k + m];
    yc[t] = acc;
}

template <typename VT>
void launch_tl_update_restrict_runs(const CoarseArgs& c, const CoarseRuns& ru, const VT* p, const VT* qv, VT* x,
                                    VT* r, const uint8_t* pflag, const double4* pn, double* yc, DevScalars* sc,
                                    cudaStream_t st) {
    if (c.nagg >= 2 * sm_count()) {
        // enough aggregates to fill the GPU: one block per aggregate is faster
        // (3.0M-tet block, 500 aggregates: 12.7 us against 18.8 us in two launches)
        k_coarse_restrict<VT, true><<<c.nagg, kAggThreads, 0, st>>>(c, p, qv, x, r, pflag, pn, yc, sc);
        counted();
        return;
    }
    const int blocks = (c.N + kRunThreads - 1) / kRunThreads;
    k_tl_update_restrict_runs<VT><<<blocks, kRunThreads, 0, st>>>(c, ru, p, qv, x, r, pflag, pn, sc);
    k_tl_restrict_finalize<<<(6 * c.nagg + 255) / 256, 256, 0, st>>>(c.nagg, ru, yc, sc);
    counted(2);
}
template void launch_tl_update_restrict_runs<float>(const CoarseArgs&, const CoarseRuns&, const float*, const float*,
                                                    float*, float*, const uint8_t*, const double4*, double*,
                                                    DevScalars*, cudaStream_t);
template void launch_tl_update_restrict_runs<double>(const CoarseArgs&, const CoarseRuns&, const double*,
                                                     const double*, double*, double*, const uint8_t*, const double4*,
                                                     double*, DevScalars*, cudaStream_t);

// 16-byte loads of the coarse inverse: 4 floats or 2 doubles
template <typename VT>
__device__ __forceinline__ void load16(const VT* p, VT (&v)[16 / sizeof(VT)]) {
    if constexpr (sizeof(VT) == 4) {
        const float4 t = __ldg(reinterpret_cast<const float4*>(p));
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    } else {
        const double2 t = __ldg(reinterpret_cast<const double2*>(p));
        v[0] = t.x; v[1] = t.y;
    }
}

// z = Minv r + P zc, zc = Ainv yc, with the dots r.z and r.r.  One block per
// aggregate: it forms its own six coarse values (rows 6a..6a+5 of Ainv, leading
// dimension ld, zero padded, times yc) and prolongs them to its nodes, so the
// coarse matvec needs no launch of its own and Ainv is read once in all.  In
// FP32 each thread loads two nodes before using either (8 % faster than one at
// a time; four, at 108 registers, was slower); FP64 takes one (two spill).
// Held to 64 registers so that 4 blocks fit an SM and every aggregate block
// is resident at once.  (Storing Ainv in FP16 with a symmetric diagonal
// scaling halved its bytes but measured slower, 18.9 -> 21.8 us.)
// init = 1: first z of a solve (sets rz); init = 0: one CG iteration's end
// (beta, it, done as k_pcg_update).
template <typename VT>
__global__ void __launch_bounds__(kAggThreads, 4) k_tl_coarse_z(CoarseArgs c, int ld, const VT* __restrict__ Ainv,
                                                             const double* __restrict__ yc, const VT* __restrict__ r,
                                                             const VT* __restrict__ Minv, VT* __restrict__ z, int init,
                                                             const uint8_t* __restrict__ pflag,
                                                             const double4* __restrict__ pn, double* partials,
                                                             DevScalars* sc, int S) {
    if (!init && *(volatile int*)&sc->done) return;
    __shared__ double sh[32][6];
    constexpr int W = 16 / sizeof(VT);
    // S blocks per aggregate: each forms the aggregate's six coarse values and
    // takes every S-th slice of its nodes
    const int a = blockIdx.x / S, sub = blockIdx.x - S * (blockIdx.x / S);
    double zc[6] = {0, 0, 0, 0, 0, 0};
    const VT* A = Ainv + (size_t)(6 * a) * ld;
    for (int j = threadIdx.x * W; j < ld; j += blockDim.x * W) {
        double y[W];
#pragma unroll
        for (int w = 0; w < W; w++) y[w] = yc[j + w];
#pragma unroll
        for (int m = 0; m < 6; m++) {
            VT v[W];
            load16<VT>(A + (size_t)m * ld + j, v);
#pragma unroll
            for (int w = 0; w < W; w++) zc[m] += (double)v[w] * y[w];
        }
    }
    block_sum<6>(zc, sh);
    const VT t0 = (VT)zc[0], t1 = (VT)zc[1], t2 = (VT)zc[2];
    const VT w0 = (VT)zc[3], w1 = (VT)zc[4], w2 = (VT)zc[5];
    double acc[2] = {0.0, 0.0};
    constexpr int U = sizeof(VT) == 4 ? 2 : 1;  // nodes per thread in flight
    const int k0 = c.agg_ptr[a], k1 = c.agg_ptr[a + 1];
    for (int kb = k0 + sub * U * blockDim.x + threadIdx.x; kb < k1; kb += U * blockDim.x * S) {
        int id[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int k = kb + u * blockDim.x;
            id[u] = k < k1 ? __ldg(c.agg_nodes + k) : -1;
        }
        VT rv[U][3], Mv[U][9];
        float4 o[U];
        unsigned f[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            if (id[u] < 0) continue;
            const size_t b = 3 * (size_t)id[u];
#pragma unroll
            for (int d = 0; d < 3; d++) rv[u][d] = r[b + d];
#pragma unroll
            for (int e = 0; e < 9; e++) Mv[u][e] = __ldg(Minv + 9 * (size_t)id[u] + e);
            o[u] = __ldg(c.off + id[u]);
            f[u] = c.fixed ? (unsigned)__ldg(c.fixed + id[u]) : 0u;
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            if (id[u] < 0) continue;
            const int i = id[u];
            VT zz[3];
#pragma unroll
            for (int d = 0; d < 3; d++)
                zz[d] = Mv[u][d * 3 + 0] * rv[u][0] + Mv[u][d * 3 + 1] * rv[u][1] + Mv[u][d * 3 + 2] * rv[u][2];
            // P_i zc: translation + rotation x offset, held DOFs dropped
            const VT ox = (VT)o[u].x, oy = (VT)o[u].y, oz = (VT)o[u].z;
            VT add[3] = {t0 + w1 * oz - w2 * oy, t1 - w0 * oz + w2 * ox, t2 + w0 * oy - w1 * ox};
            if (f[u] & 1u) add[0] = VT(0);
            if (f[u] & 2u) add[1] = VT(0);
            if (f[u] & 4u) add[2] = VT(0);
#pragma unroll
            for (int d = 0; d < 3; d++) zz[d] += add[d];
            project3<VT>(pflag, pn, i, zz);
#pragma unroll
            for (int d = 0; d < 3; d++) {
                z[3 * (size_t)i + d] = zz[d];
                acc[0] += (double)rv[u][d] * (double)zz[d];
                acc[1] += (double)rv[u][d] * (double)rv[u][d];
            }
        }
    }
    double tot[2];
    if (reduce_grid<2>(acc, partials, &sc->counters[init ? 8 : 9], tot) && threadIdx.x == 0) {
        if (init) {
            sc->rz = tot[0];
        } else {
            sc->beta = tot[0] / sc->rz;
            sc->rz = tot[0];
            sc->rr = tot[1];
            sc->it += 1;
            if (tot[1] <= sc->tol2 || sc->it >= sc->maxit || !(tot[1] == tot[1])) sc->done = 1;
        }
    }
}
template <typename VT>
void launch_tl_coarse_z(const CoarseArgs& c, int ld, const VT* Ainv, const double* yc, const VT* r, const VT* Minv,
                        VT* z, int init, const uint8_t* pflag, const double4* pn, double* partials, DevScalars* sc,
                        cudaStream_t st) {
    if (c.nagg == 0) return;
    // few aggregates: several blocks per aggregate, about two blocks per SM in all
    const int want = 2 * sm_count();
    const int S = c.nagg >= want ? 1 : std::min(8, (want + c.nagg - 1) / c.nagg);
    k_tl_coarse_z<VT><<<c.nagg * S, kAggThreads, 0, st>>>(c, ld, Ainv, yc, r, Minv, z, init, pflag, pn, partials, sc,
                                                         S);
    counted();
}

// out (nc rows, leading dimension ld >= nc, padding zero) = in (nc x nc), symmetrised
template <typename VT>
__global__ void k_to_vt_pad(int nc, int ld, const double* __restrict__ in, VT* __restrict__ out) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)nc * ld) return;
    const int i = (int)(t / ld), j = (int)(t - (long long)i * ld);
    out[t] = j < nc ? (VT)(0.5 * (in[(size_t)i * nc + j] + in[(size_t)j * nc + i])) : VT(0);
}
template <typename VT>
void launch_to_vt_pad(int nc, int ld, const double* in, VT* out, cudaStream_t st) {
    if (nc == 0) return;
    const long long n = (long long)nc * ld;
    k_to_vt_pad<VT><<<(int)((n + 255) / 256), 256, 0, st>>>(nc, ld, in, out);
    counted();
}

template void launch_to_vt_pad<float>(int, int, const double*, float*, cudaStream_t);
template void launch_to_vt_pad<double>(int, int, const double*, double*, cudaStream_t);
template void launch_tl_update_restrict<float>(const CoarseArgs&, const float*, const float*, float*, float*,
                                               const uint8_t*, const double4*, double*, DevScalars*, cudaStream_t);
template void launch_tl_update_restrict<double>(const CoarseArgs&, const double*, const double*, double*, double*,
                                                const uint8_t*, const double4*, double*, DevScalars*, cudaStream_t);
template void launch_coarse_restrict<float>(const CoarseArgs&, const float*, double*, cudaStream_t);
template void launch_coarse_restrict<double>(const CoarseArgs&, const double*, double*, cudaStream_t);
template void launch_tl_coarse_z<float>(const CoarseArgs&, int, const float*, const double*, const float*,
                                        const float*, float*, int, const uint8_t*, const double4*, double*,
                                        DevScalars*, cudaStream_t);
template void launch_tl_coarse_z<double>(const CoarseArgs&, int, const double*, const double*, const double*,
                                         const double*, double*, int, const uint8_t*, const double4*, double*,
                                         DevScalars*, cudaStream_t);

// ---------------------------------------------------------------------------
// explicit instantiations
// ---------------------------------------------------------------------------
template void launch_assemble<double>(const AsmArgs<double>&, int, cudaStream_t);
template void launch_assemble<float>(const AsmArgs<float>&, int, cudaStream_t);
template void launch_elem_rows<double>(int, int, const double*, const double*, const int*, const double2*,
                                       const double*, const MuscleArgs&, int, int,
                                       double*, double*, double*, int*, cudaStream_t);
template void launch_elem_rows<float>(int, int, const double*, const double*, const int*, const double2*,
                                      const double*, const MuscleArgs&, int, int,
                                      double*, double*, double*, int*, cudaStream_t);
template void launch_pressure_jac<double>(const PressureArgs&, const int*, const int*, const uint8_t*, double, double*,
                                          long long, cudaStream_t);
template void launch_pressure_jac<float>(const PressureArgs&, const int*, const int*, const uint8_t*, double, float*,
                                         long long, cudaStream_t);
template void launch_block_jacobi<double, double>(int, const int*, const int*, const double*, long long, double*,
                                                  cudaStream_t);
template void launch_block_jacobi<float, float>(int, const int*, const int*, const float*, long long, float*,
                                                cudaStream_t);
template void launch_pcg_init<double, double>(int, const double*, const double*, double*, double*, double*, double*,
                                              double, double, int, const uint8_t*, const double4*, double*,
                                              DevScalars*, cudaStream_t);
template void launch_pcg_init<float, float>(int, const double*, const float*, float*, float*, float*, float*, double,
                                            double, int, const uint8_t*, const double4*, double*, DevScalars*,
                                            cudaStream_t);
template void launch_pcg_spmv<double, double>(int, int, const int*, const int*, const double*, long long,
                                              const double*, double*, double*, DevScalars*, cudaStream_t);
template void launch_pcg_spmv<float, float>(int, int, const int*, const int*, const float*, long long, const float*,
                                            float*, double*, DevScalars*, cudaStream_t);
template void launch_form_p<double>(int, const double*, const double*, double*, const DevScalars*, cudaStream_t);
template void launch_form_p<float>(int, const float*, const float*, float*, const DevScalars*, cudaStream_t);
template void launch_pcg_update<double>(int, const double*, const double*, const double*, double*, double*, double*,
                                        const uint8_t*, const double4*, double*, DevScalars*, cudaStream_t);
template void launch_pcg_update<float>(int, const float*, const float*, const float*, float*, float*, float*,
                                       const uint8_t*, const double4*, double*, DevScalars*, cudaStream_t);
template void launch_newton_update<double>(int, const double*, double, double*, const double*, double*, DevScalars*,
                                           int, cudaStream_t);
template void launch_newton_update<float>(int, const float*, double, double*, const double*, double*, DevScalars*, int,
                                          cudaStream_t);
template void launch_dot_gdx<double>(int, const double*, const double*, double*, DevScalars*, cudaStream_t);
template void launch_dot_gdx<float>(int, const double*, const float*, double*, DevScalars*, cudaStream_t);
template void launch_spmv_plain<double>(int, const int*, const int*, const double*, long long, const double*,
                                        double*, cudaStream_t);
template void launch_spmv_plain<float>(int, const int*, const int*, const float*, long long, const double*, double*,
                                       cudaStream_t);

// ---------------------------------------------------------------------------
// MINRES for the symmetric indefinite Newton systems of the exact Hessian
// (Paige & Saunders 1975, preconditioned form as in Elman, Silvester &
// Wathen, "Finite Elements and Fast Iterative Solvers", 2nd ed., Alg. 4.1).
// The reference factors such systems with LDL^T (cpp/src/solver.cpp:65-84);
// CG cannot take them.  The preconditioner must be SPD: block Jacobi on
// |D_ii| (each diagonal block with its eigenvalues replaced by their absolute
// values), plus the two-level coarse correction built from the SPD-projected
// Hessian.  Iteration j (1-based): the SpMV q = A z_j on the unnormalised
// z_j (MODE 1 of k_pcg_spmv, which also applies iteration j-1's pending
// solution update row by row), then the Lanczos step
//   v_{j+1} = q / g_j - (delta_j / g_j) v_j - (g_j / g_{j-1}) v_{j-1}
// fused with z_{j+1} = M^-1 v_{j+1} and the dot g_{j+1}^2 = v_{j+1}.z_{j+1},
// whose last block advances the Givens QR (minres_advance).  Buffers
// alternate by parity: Z[j & 1] (padded), V[j & 1], W[j & 1]; the Lanczos
// step writes v_{j+1} and z_{j+1} over v_{j-1} and z_{j-1}, the update writes
// w_{j+1} over w_{j-1}.  After the last iteration the host applies its
// pending update with k_minres_finish.
// ---------------------------------------------------------------------------
template <typename HT, typename VT>
__global__ void k_block_jacobi_abs(int N, const int* diag_slot, const HT* H, long long nnzb, VT* Minv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const size_t d = (size_t)diag_slot[i];
    double a[9], w[3], Y[9];
#pragma unroll
    for (int k = 0; k < 9; k++) a[k] = (double)H[hval(d, k, nnzb)];
    // symmetric part: the lower triangle defines the operator
    a[1] = a[3]; a[2] = a[6]; a[5] = a[7];
    sym3_eig(a, w, Y);
    double amax = 0.0;
#pragma unroll
    for (int k = 0; k < 3; k++) amax = fmax(amax, fabs(w[k]));
    double iw[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const double aw = fabs(w[k]);
        iw[k] = (aw > 1e-12 * amax && aw == aw) ? 1.0 / aw : (amax > 0.0 ? 1.0 / amax : 1.0);
    }
    VT* o = Minv + (size_t)i * 9;
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++)
            o[r * 3 + c] = (VT)(Y[r * 3 + 0] * iw[0] * Y[c * 3 + 0] + Y[r * 3 + 1] * iw[1] * Y[c * 3 + 1] +
                                Y[r * 3 + 2] * iw[2] * Y[c * 3 + 2]);
}

template <typename HT, typename VT>
void launch_block_jacobi_abs(int N, const int* diag_slot, const HT* H, long long nnzb, VT* Minv, cudaStream_t st) {
    if (N == 0) return;
    k_block_jacobi_abs<HT, VT><<<(N + 127) / 128, 128, 0, st>>>(N, diag_slot, H, nnzb, Minv);
    counted();
}

// First Lanczos vector: v_1 = b = -g (gamma_1 = ||b||_{M^-1} = eta_0).
__device__ void minres_start(DevScalars* sc, double vz, double vv, double eta2, double abs_tol2, int maxit) {
    sc->it = 0;
    sc->maxit = maxit;
    sc->breakdown = 0;
    sc->mr_bad = (vz >= 0.0) ? 0 : 1;
    const double g = vz > 0.0 ? sqrt(vz) : 0.0;
    sc->mr_g = g;
    sc->mr_gprev = 1.0;
    sc->mr_delta = 0.0;
    sc->mr_c = sc->mr_cprev = 1.0;
    sc->mr_s = sc->mr_sprev = 0.0;
    sc->mr_eta = g;
    sc->mr_pending = 0;
    sc->bnorm2 = vz;
    sc->rr = vz;
    // the absolute target is a 2-norm; scaled to the M^-1 norm by their ratio at b
    const double t1 = eta2 * vz, t2 = vv > 0.0 ? abs_tol2 * vz / vv : 0.0;
    sc->tol2 = t1 > t2 ? t1 : t2;
    sc->counters[4] = 0u;
    sc->counters[12] = 0u;
    sc->done = (vz <= sc->tol2 || maxit <= 0 || g == 0.0 || sc->mr_bad) ? 1 : 0;
}

// Givens step of iteration j from g_{j+1}^2 = vz: leaves the solution update
// w_{j+1} = (z_j / g_j - a3 w_{j-1} - a2 w_j) / a1, x += c_{j+1} eta_j w_{j+1}
// pending, and |eta_{j+1}| = ||r_j||_{M^-1}.
__device__ void minres_advance(DevScalars* sc, double vz) {
    const double g = sc->mr_g, d = sc->mr_delta;
    if (!(vz >= 0.0)) sc->mr_bad = 1;
    const double gn = vz > 0.0 ? sqrt(vz) : 0.0;
    const double a0 = sc->mr_c * d - sc->mr_cprev * sc->mr_s * g;
    const double a1 = sqrt(a0 * a0 + gn * gn);
    const double a2 = sc->mr_s * d + sc->mr_cprev * sc->mr_c * g;
    const double a3 = sc->mr_sprev * g;
    sc->it += 1;
    if (!(a1 > 0.0) || !(d == d)) {
        sc->breakdown = 1;
        sc->mr_pending = 0;
        sc->done = 1;
        return;
    }
    const double cn = a0 / a1, sn = gn / a1;
    sc->mr_a1 = a1;
    sc->mr_a2 = a2;
    sc->mr_a3 = a3;
    sc->mr_ceta = cn * sc->mr_eta;
    sc->mr_ig = 1.0 / g;
    sc->mr_pending = 1;
    sc->mr_eta = -sn * sc->mr_eta;
    sc->mr_cprev = sc->mr_c;
    sc->mr_c = cn;
    sc->mr_sprev = sc->mr_s;
    sc->mr_s = sn;
    sc->mr_gprev = g;
    sc->mr_g = gn;
    sc->rr = sc->mr_eta * sc->mr_eta;
    if (sc->rr <= sc->tol2 || sc->it >= sc->maxit || gn == 0.0 || sc->mr_bad) sc->done = 1;
}

template <typename VT>
__device__ __forceinline__ void st_pad(VT* z4, size_t i, const VT (&z)[3]) {
    if constexpr (sizeof(VT) == 4) {
        reinterpret_cast<float4*>(z4)[i] = make_float4(z[0], z[1], z[2], 0.0f);
    } else {
        double2* d = reinterpret_cast<double2*>(z4) + 2 * i;
        d[0] = make_double2(z[0], z[1]);
        d[1] = make_double2(z[2], 0.0);
    }
}

// v_1 = -g into V[1], v_0 = 0, w_0 = w_1 = 0, x = 0; with the block-Jacobi
// preconditioner also z_1 = M^-1 v_1 into Z[1] and the start of the recurrence.
template <typename VT, bool WITHZ>
__global__ void __launch_bounds__(kRedThreads) k_minres_init(int N, const double* __restrict__ g, MinresBufs<VT> b,
                                                              double eta2, double abs_tol2, int maxit,
                                                              double* partials, DevScalars* sc) {
    double acc[2] = {0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        VT v[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const size_t ii = 3 * (size_t)i + k;
            v[k] = (VT)(-g[ii]);
            b.V[1][ii] = v[k];
            b.V[0][ii] = VT(0);
            b.W[0][ii] = VT(0);
            b.W[1][ii] = VT(0);
            b.x[ii] = VT(0);
        }
        if (WITHZ) {
            const VT* M = b.Minv + (size_t)i * 9;
            VT z[3];
#pragma unroll
            for (int k = 0; k < 3; k++) z[k] = M[k * 3 + 0] * v[0] + M[k * 3 + 1] * v[1] + M[k * 3 + 2] * v[2];
            st_pad<VT>(b.Z[1], (size_t)i, z);
#pragma unroll
            for (int k = 0; k < 3; k++) {
                acc[0] += (double)v[k] * (double)z[k];
                acc[1] += (double)v[k] * (double)v[k];
            }
        }
    }
    if (!WITHZ) return;
    double tot[2];
    if (reduce_grid<2>(acc, partials, &sc->counters[11], tot) && threadIdx.x == 0)
        minres_start(sc, tot[0], tot[1], eta2, abs_tol2, maxit);
}

template <typename VT>
void launch_minres_init(int N, const double* g, const MinresBufs<VT>& b, bool with_z, double eta2, double abs_tol2,
                        int maxit, double* partials, DevScalars* sc, cudaStream_t st) {
    if (with_z)
        k_minres_init<VT, true><<<red_grid(N, 2), kRedThreads, 0, st>>>(N, g, b, eta2, abs_tol2, maxit, partials, sc);
    else
        k_minres_init<VT, false><<<red_grid(N, 2), kRedThreads, 0, st>>>(N, g, b, eta2, abs_tol2, maxit, partials, sc);
    counted();
}

// Iteration j's SpMV (par = j & 1).
template <typename HT, typename VT>
void launch_minres_spmv(int N, int max_row_blocks, const int* row_ptr, const int* col, const HT* H, long long nnzb,
                        const MinresBufs<VT>& b, int par, double* partials, DevScalars* sc, cudaStream_t st) {
    MinresUpd<VT> u;
    u.zprev = b.Z[par ^ 1];
    u.wread = b.W[par ^ 1];
    u.wrw = b.W[par];
    u.x = b.x;
    launch_spmv_g<HT, VT, 2, 1>(N, max_row_blocks, row_ptr, col, H, nnzb, b.Z[par], b.q, partials, sc, st, u);
}

// The Lanczos vector of iteration j (par = j & 1) at node i, written over v_{j-1}.
template <typename VT>
__device__ __forceinline__ void minres_lanczos_node(const MinresBufs<VT>& b, int par, size_t i, VT ig, VT dg, VT gg,
                                                    VT (&v)[3]) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const size_t ii = 3 * i + k;
        v[k] = b.q[ii] * ig - dg * b.V[par][ii] - gg * b.V[par ^ 1][ii];
        b.V[par ^ 1][ii] = v[k];
    }
}

// Block-Jacobi variant: Lanczos step, z_{j+1} = M^-1 v_{j+1}, the Givens step.
template <typename VT>
__global__ void __launch_bounds__(kRedThreads) k_minres_lanczos(int N, MinresBufs<VT> b, int par, double* partials,
                                                                 DevScalars* sc) {
    if (*(volatile int*)&sc->done) return;
    const double g = sc->mr_g;
    const VT ig = (VT)(1.0 / g), dg = (VT)(sc->mr_delta / g), gg = (VT)(g / sc->mr_gprev);
    double acc[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        VT v[3];
        minres_lanczos_node<VT>(b, par, (size_t)i, ig, dg, gg, v);
        const VT* M = b.Minv + (size_t)i * 9;
        VT z[3];
#pragma unroll
        for (int k = 0; k < 3; k++) z[k] = M[k * 3 + 0] * v[0] + M[k * 3 + 1] * v[1] + M[k * 3 + 2] * v[2];
        st_pad<VT>(b.Z[par ^ 1], (size_t)i, z);
#pragma unroll
        for (int k = 0; k < 3; k++) acc[0] += (double)v[k] * (double)z[k];
    }
    double tot[1];
    if (reduce_grid<1>(acc, partials, &sc->counters[12], tot) && threadIdx.x == 0) minres_advance(sc, tot[0]);
}

template <typename VT>
void launch_minres_lanczos(int N, const MinresBufs<VT>& b, int par, double* partials, DevScalars* sc,
                           cudaStream_t st) {
    k_minres_lanczos<VT><<<red_grid(N, 2), kRedThreads, 0, st>>>(N, b, par, partials, sc);
    counted();
}

// Two-level variant, first half: the Lanczos step on each aggregate's nodes
// and yc = P^T v_{j+1} (one block per aggregate, fixed-order sums).
template <typename VT>
__global__ void __launch_bounds__(kAggThreads) k_minres_lanczos_restrict(CoarseArgs c, MinresBufs<VT> b, int par,
                                                                          double* __restrict__ yc,
                                                                          const DevScalars* sc) {
    if (*(volatile const int*)&sc->done) return;
    __shared__ double sh[32][6];
    const int a = blockIdx.x;
    const double g = sc->mr_g;
    const VT ig = (VT)(1.0 / g), dg = (VT)(sc->mr_delta / g), gg = (VT)(g / sc->mr_gprev);
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int k = c.agg_ptr[a] + threadIdx.x; k < c.agg_ptr[a + 1]; k += blockDim.x) {
        const int i = c.agg_nodes[k];
        VT v[3];
        minres_lanczos_node<VT>(b, par, (size_t)i, ig, dg, gg, v);
        const double vd[3] = {(double)v[0], (double)v[1], (double)v[2]};
        double y[6];
        coarse_restrict_node(c, i, vd, y);
#pragma unroll
        for (int m = 0; m < 6; m++) acc[m] += y[m];
    }
    block_sum<6>(acc, sh);
    if (threadIdx.x == 0)
#pragma unroll
        for (int m = 0; m < 6; m++) yc[6 * a + m] = acc[m];
}

template <typename VT>
void launch_minres_lanczos_restrict(const CoarseArgs& c, const MinresBufs<VT>& b, int par, double* yc,
                                    const DevScalars* sc, cudaStream_t st) {
    k_minres_lanczos_restrict<VT><<<c.nagg, kAggThreads, 0, st>>>(c, b, par, yc, sc);
    counted();
}

// Two-level variant, second half: z = M^-1 v + P Ainv yc for the Lanczos
// vector in V[vpar] into Z[vpar], with v.z (and v.v); init = 1 starts the
// recurrence (vpar = 1), init = 0 takes the Givens step.  The coarse rows are
// formed as in k_tl_coarse_z.
template <typename VT>
__global__ void __launch_bounds__(kAggThreads, 4) k_minres_coarse_z(CoarseArgs c, int ld, const VT* __restrict__ Ainv,
                                                                 const double* __restrict__ yc, MinresBufs<VT> b,
                                                                 int vpar, int init, double eta2, double abs_tol2,
                                                                 int maxit, double* partials, DevScalars* sc) {
    if (!init && *(volatile int*)&sc->done) return;
    __shared__ double sh[32][6];
    constexpr int W = 16 / sizeof(VT);
    const int a = blockIdx.x;
    double zc[6] = {0, 0, 0, 0, 0, 0};
    const VT* A = Ainv + (size_t)(6 * a) * ld;
    for (int j = threadIdx.x * W; j < ld; j += blockDim.x * W) {
        double y[W];
#pragma unroll
        for (int w = 0; w < W; w++) y[w] = yc[j + w];
#pragma unroll
        for (int m = 0; m < 6; m++) {
            VT v[W];
            load16<VT>(A + (size_t)m * ld + j, v);
#pragma unroll
            for (int w = 0; w < W; w++) zc[m] += (double)v[w] * y[w];
        }
    }
    block_sum<6>(zc, sh);
    const VT t0 = (VT)zc[0], t1 = (VT)zc[1], t2 = (VT)zc[2];
    const VT w0 = (VT)zc[3], w1 = (VT)zc[4], w2 = (VT)zc[5];
    const VT* vin = b.V[vpar];
    double acc[2] = {0.0, 0.0};
    for (int k = c.agg_ptr[a] + threadIdx.x; k < c.agg_ptr[a + 1]; k += blockDim.x) {
        const int i = __ldg(c.agg_nodes + k);
        const size_t bi = 3 * (size_t)i;
        const VT v[3] = {vin[bi], vin[bi + 1], vin[bi + 2]};
        const VT* M = b.Minv + 9 * (size_t)i;
        VT z[3];
#pragma unroll
        for (int d = 0; d < 3; d++) z[d] = M[d * 3 + 0] * v[0] + M[d * 3 + 1] * v[1] + M[d * 3 + 2] * v[2];
        const float4 o = __ldg(c.off + i);
        const unsigned f = c.fixed ? (unsigned)__ldg(c.fixed + i) : 0u;
        const VT ox = (VT)o.x, oy = (VT)o.y, oz = (VT)o.z;
        VT add[3] = {t0 + w1 * oz - w2 * oy, t1 - w0 * oz + w2 * ox, t2 + w0 * oy - w1 * ox};
        if (f & 1u) add[0] = VT(0);
        if (f & 2u) add[1] = VT(0);
        if (f & 4u) add[2] = VT(0);
#pragma unroll
        for (int d = 0; d < 3; d++) z[d] += add[d];
        st_pad<VT>(b.Z[vpar], (size_t)i, z);
#pragma unroll
        for (int d = 0; d < 3; d++) {
            acc[0] += (double)v[d] * (double)z[d];
            acc[1] += (double)v[d] * (double)v[d];
        }
    }
    double tot[2];
    if (reduce_grid<2>(acc, partials, &sc->counters[init ? 11 : 12], tot) && threadIdx.x == 0) {
        if (init) minres_start(sc, tot[0], tot[1], eta2, abs_tol2, maxit);
        else minres_advance(sc, tot[0]);
    }
}

template <typename VT>
void launch_minres_coarse_z(const CoarseArgs& c, int ld, const VT* Ainv, const double* yc, const MinresBufs<VT>& b,
                            int vpar, int init, double eta2, double abs_tol2, int maxit, double* partials,
                            DevScalars* sc, cudaStream_t st) {
    k_minres_coarse_z<VT><<<c.nagg, kAggThreads, 0, st>>>(c, ld, Ainv, yc, b, vpar, init, eta2, abs_tol2, maxit,
                                                           partials, sc);
    counted();
}

// The last iteration's pending solution update (par = (J + 1) & 1 for the
// last iteration J, as the SpMV of iteration J + 1 would have applied it).
template <typename VT>
__global__ void __launch_bounds__(kRedThreads) k_minres_finish(int N, MinresBufs<VT> b, int par, const DevScalars* sc) {
    if (!sc->mr_pending) return;
    MinresUpd<VT> u;
    u.zprev = b.Z[par ^ 1];
    u.wread = b.W[par ^ 1];
    u.wrw = b.W[par];
    u.x = b.x;
    const VT ig = (VT)sc->mr_ig, a1i = (VT)(1.0 / sc->mr_a1), a2 = (VT)sc->mr_a2, a3 = (VT)sc->mr_a3;
    const VT ceta = (VT)sc->mr_ceta;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
#pragma unroll
        for (int d = 0; d < 3; d++) minres_row_update<VT>(u, (size_t)i, d, ig, a1i, a2, a3, ceta);
}

template <typename VT>
void launch_minres_finish(int N, const MinresBufs<VT>& b, int par, const DevScalars* sc, cudaStream_t st) {
    k_minres_finish<VT><<<red_grid(N, 2), kRedThreads, 0, st>>>(N, b, par, sc);
    counted();
}

#define SORS_MINRES_INST(HT, VT)                                                                                   \
    template void launch_block_jacobi_abs<HT, VT>(int, const int*, const HT*, long long, VT*, cudaStream_t);     \
    template void launch_minres_spmv<HT, VT>(int, int, const int*, const int*, const HT*, long long,              \
                                             const MinresBufs<VT>&, int, double*, DevScalars*, cudaStream_t);
SORS_MINRES_INST(double, double)
SORS_MINRES_INST(float, float)
#undef SORS_MINRES_INST
#define SORS_MINRES_INST_V(VT)                                                                                      \
    template void launch_minres_init<VT>(int, const double*, const MinresBufs<VT>&, bool, double, double, int,     \
                                         double*, DevScalars*, cudaStream_t);                                      \
    template void launch_minres_lanczos<VT>(int, const MinresBufs<VT>&, int, double*, DevScalars*, cudaStream_t);  \
    template void launch_minres_lanczos_restrict<VT>(const CoarseArgs&, const MinresBufs<VT>&, int, double*,       \
                                                     const DevScalars*, cudaStream_t);                             \
    template void launch_minres_coarse_z<VT>(const CoarseArgs&, int, const VT*, const double*,                     \
                                             const MinresBufs<VT>&, int, int, double, double, int, double*,         \
                                             DevScalars*, cudaStream_t);                                            \
    template void launch_minres_finish<VT>(int, const MinresBufs<VT>&, int, const DevScalars*, cudaStream_t);
SORS_MINRES_INST_V(double)
SORS_MINRES_INST_V(float)
#undef SORS_MINRES_INST_V

}  // namespace sors
