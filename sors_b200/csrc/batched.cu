// batched.cu -- member-segmented PCG for handles that hold several meshes.
//
// A handle built from several independent meshes (a union: concatenated node
// ranges, no element couples two ranges) has a block-diagonal Hessian.  One
// conjugate-gradient run on the whole system would share its step lengths
// across the meshes and converge at the pace of the hardest; these kernels
// run one preconditioned CG per member instead, in the same launches: every
// thread block works on nodes of a single member, each member's dot products
// are summed in a fixed order from its own blocks' partial sums (the last of
// its blocks to finish does it), and each member carries its own step
// lengths, iteration count and convergence flag.  A member that has
// converged costs one flag read per block from then on.
#include <cuda_runtime.h>
#include <stdint.h>

#include "sors_internal.h"

namespace sors {

namespace {

constexpr int kBT = kBatchThreads;  // one node per thread

template <typename VT>
__device__ __forceinline__ void bproject3(const uint8_t* __restrict__ pflag, const double4* __restrict__ pn, int i,
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

// Block sum of NS values (lanes, then warps: fixed order); thread 0 gets them.
template <int NS>
__device__ __forceinline__ void bblock_sum(double (&v)[NS], double (*sh)[NS]) {
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int s = 0; s < NS; s++) v[s] += __shfl_xor_sync(0xffffffffu, v[s], o);
    if (l == 0)
#pragma unroll
        for (int s = 0; s < NS; s++) sh[w][s] = v[s];
    __syncthreads();
    if (threadIdx.x == 0)
        for (int k = 1; k < (int)(blockDim.x >> 5); k++)
#pragma unroll
            for (int s = 0; s < NS; s++) v[s] += sh[k][s];
}

// Writes this block's partial sums; returns true in thread 0 of the member's
// last block to finish, with the member's totals (its blocks in order) in tot.
template <int NS>
__device__ bool member_reduce(const BatchArgs& b, int m, double (&v)[NS], int site, double (&tot)[NS]) {
    __shared__ double sh[kBT / 32][NS];
    bblock_sum<NS>(v, sh);
    if (threadIdx.x != 0) return false;
#pragma unroll
    for (int s = 0; s < NS; s++) b.partials[(size_t)blockIdx.x * 2 + s] = v[s];
    __threadfence();
    MemberScalars& ms = b.ms[m];
    const int b0 = b.mem_blk0[m], nb = b.mem_blk0[m + 1] - b0;
    if (atomicAdd(&ms.counter[site], 1u) != (unsigned)(nb - 1)) return false;
    __threadfence();
    const volatile double* vp = b.partials;
#pragma unroll
    for (int s = 0; s < NS; s++) tot[s] = 0.0;
    for (int k = b0; k < b0 + nb; k++)
#pragma unroll
        for (int s = 0; s < NS; s++) tot[s] += vp[(size_t)k * 2 + s];
    ms.counter[site] = 0u;
    return true;
}

__device__ __forceinline__ void block_nodes(const BatchArgs& b, int& m, int& i) {
    m = __ldg(b.blk_mem + blockIdx.x);
    const int first = __ldg(b.mem_node0 + m) + (blockIdx.x - __ldg(b.mem_blk0 + m)) * kBT;
    i = first + (int)threadIdx.x;
    if (i >= __ldg(b.mem_node0 + m + 1)) i = -1;
}

template <typename VT>
__global__ void __launch_bounds__(kBT) k_bpcg_init(BatchArgs b, const double* __restrict__ g,
                                                   const VT* __restrict__ Minv, VT* x, VT* r, VT* z, VT* p0,
                                                   double eta2, double abs_tol2, int tol_mode, int maxit,
                                                   const uint8_t* __restrict__ pflag, const double4* __restrict__ pn) {
    int m, i;
    block_nodes(b, m, i);
    double acc[2] = {0.0, 0.0};
    if (i >= 0) {
        VT rr[3];
        for (int k = 0; k < 3; k++) {
            rr[k] = (VT)(-g[3 * (size_t)i + k]);
            x[3 * (size_t)i + k] = VT(0);
            p0[4 * (size_t)i + k] = VT(0);
        }
        p0[4 * (size_t)i + 3] = VT(0);
        bproject3<VT>(pflag, pn, i, rr);
        for (int k = 0; k < 3; k++) r[3 * (size_t)i + k] = rr[k];
        const VT* M = Minv + (size_t)i * 9;
        VT zz[3];
        for (int k = 0; k < 3; k++) zz[k] = M[k * 3 + 0] * rr[0] + M[k * 3 + 1] * rr[1] + M[k * 3 + 2] * rr[2];
        bproject3<VT>(pflag, pn, i, zz);
        for (int k = 0; k < 3; k++) {
            z[3 * (size_t)i + k] = zz[k];
            acc[0] += (double)rr[k] * (double)zz[k];
            acc[1] += (double)rr[k] * (double)rr[k];
        }
    }
    double tot[2];
    if (member_reduce<2>(b, m, acc, 0, tot)) {
        MemberScalars& ms = b.ms[m];
        ms.rz = tot[0];
        ms.rr = tot[1];
        ms.bnorm2 = tot[1];
        // tol_mode 0: relative eta or absolute tolerance, whichever is looser;
        // 1: relative, and remember eta^2 ||b||^2 as this member's absolute
        // target; 2: the remembered absolute target
        double t2 = eta2 * tot[1];
        if (tol_mode == 0) t2 = t2 > abs_tol2 ? t2 : abs_tol2;
        if (tol_mode == 1) ms.abs2 = t2;
        if (tol_mode == 2) t2 = ms.abs2;
        ms.tol2 = t2;
        ms.beta = 0.0;
        ms.alpha = 0.0;
        ms.it = 0;
        ms.maxit = maxit;
        ms.breakdown = 0;
        ms.done = (tot[1] <= t2 || maxit <= 0) ? 1 : 0;
    }
}

template <typename VT>
__global__ void __launch_bounds__(kBT) k_bform_p(BatchArgs b, const VT* __restrict__ z,
                                                 const VT* __restrict__ p_old, VT* __restrict__ p_new) {
    int m, i;
    block_nodes(b, m, i);
    const MemberScalars& ms = b.ms[m];
    if (*(volatile const int*)&ms.done || i < 0) return;
    const VT beta = (VT)ms.beta;
#pragma unroll
    for (int k = 0; k < 3; k++) p_new[4 * (size_t)i + k] = z[3 * (size_t)i + k] + beta * p_old[4 * (size_t)i + k];
    p_new[4 * (size_t)i + 3] = VT(0);
}

// q = H p for the block's rows (one row per thread) and the member's p . q
template <typename HT, typename VT>
__global__ void __launch_bounds__(kBT) k_bspmv(BatchArgs b, const int* __restrict__ row_ptr,
                                               const int* __restrict__ col, const HT* __restrict__ H,
                                               const VT* __restrict__ p, VT* __restrict__ qv) {
    int m, i;
    block_nodes(b, m, i);
    MemberScalars& ms = b.ms[m];
    if (*(volatile int*)&ms.done) return;
    double acc[1] = {0.0};
    if (i >= 0) {
        VT q0 = VT(0), q1 = VT(0), q2 = VT(0);
        for (int bk = __ldg(row_ptr + i); bk < __ldg(row_ptr + i + 1); bk++) {
            const int j = __ldg(col + bk);
            const VT a = p[4 * (size_t)j], c = p[4 * (size_t)j + 1], d = p[4 * (size_t)j + 2];
            const HT* B = H + 9 * (size_t)bk;
            q0 += (VT)B[0] * a + (VT)B[1] * c + (VT)B[2] * d;
            q1 += (VT)B[3] * a + (VT)B[4] * c + (VT)B[5] * d;
            q2 += (VT)B[6] * a + (VT)B[7] * c + (VT)B[8] * d;
        }
        qv[3 * (size_t)i] = q0;
        qv[3 * (size_t)i + 1] = q1;
        qv[3 * (size_t)i + 2] = q2;
        acc[0] = (double)p[4 * (size_t)i] * (double)q0 + (double)p[4 * (size_t)i + 1] * (double)q1 +
                 (double)p[4 * (size_t)i + 2] * (double)q2;
    }
    double tot[1];
    if (member_reduce<1>(b, m, acc, 1, tot)) {
        ms.pq = tot[0];
        if (!(tot[0] > 0.0)) {
            ms.breakdown = 1;
            ms.done = 1;
            ms.alpha = 0.0;
        } else {
            ms.alpha = ms.rz / tot[0];
        }
    }
}

// q = A p for a block's nodes with LPR lanes per row, in passes of kBT / LPR
// rows: each lane takes groups of two consecutive blocks of the row (nine
// 8-byte FP32 / 16-byte FP64 loads for 18 values, both columns in one load,
// one 16-byte gather of p per block), the row's lanes are summed with
// shuffles, and the member's p.q is reduced as in k_bspmv.
template <typename HT, typename VT, int LPR>
__global__ void __launch_bounds__(kBT) k_bspmv_g(BatchArgs b, const int* __restrict__ row_ptr,
                                                 const int* __restrict__ col, const HT* __restrict__ H,
                                                 const VT* __restrict__ p, VT* __restrict__ qv) {
    const int m = __ldg(b.blk_mem + blockIdx.x);
    const int first = __ldg(b.mem_node0 + m) + (blockIdx.x - __ldg(b.mem_blk0 + m)) * kBT;
    const int last = min(first + kBT, __ldg(b.mem_node0 + m + 1));
    MemberScalars& ms = b.ms[m];
    if (*(volatile int*)&ms.done) return;
    constexpr int RPP = kBT / LPR;
    const int sub = threadIdx.x / LPR, sl = threadIdx.x % LPR;
    double acc[1] = {0.0};
    for (int r0 = first; r0 < last; r0 += RPP) {
        const int row = r0 + sub;
        VT a0 = VT(0), a1 = VT(0), a2 = VT(0);
        if (row < last) {
            const int b0 = __ldg(row_ptr + row), b1 = __ldg(row_ptr + row + 1);
            for (int gi = b0 / 2 + sl; gi <= (b1 - 1) / 2; gi += LPR) {
                HT hv[18];
                if constexpr (sizeof(HT) == 4) {
                    const float2* src = reinterpret_cast<const float2*>(H) + 9 * (size_t)gi;
#pragma unroll
                    for (int k = 0; k < 9; k++) {
                        const float2 t = __ldg(src + k);
                        hv[2 * k] = t.x;
                        hv[2 * k + 1] = t.y;
                    }
                } else {
                    const double2* src = reinterpret_cast<const double2*>(H) + 9 * (size_t)gi;
#pragma unroll
                    for (int k = 0; k < 9; k++) {
                        const double2 t = __ldg(src + k);
                        hv[2 * k] = t.x;
                        hv[2 * k + 1] = t.y;
                    }
                }
                const int2 c2 = __ldg(reinterpret_cast<const int2*>(col) + gi);
#pragma unroll
                for (int u = 0; u < 2; u++) {
                    const int bk = 2 * gi + u;
                    if (bk < b0 || bk >= b1) continue;
                    const int j = u == 0 ? c2.x : c2.y;
                    const VT x0 = p[4 * (size_t)j], x1 = p[4 * (size_t)j + 1], x2 = p[4 * (size_t)j + 2];
                    a0 += (VT)hv[9 * u] * x0 + (VT)hv[9 * u + 1] * x1 + (VT)hv[9 * u + 2] * x2;
                    a1 += (VT)hv[9 * u + 3] * x0 + (VT)hv[9 * u + 4] * x1 + (VT)hv[9 * u + 5] * x2;
                    a2 += (VT)hv[9 * u + 6] * x0 + (VT)hv[9 * u + 7] * x1 + (VT)hv[9 * u + 8] * x2;
                }
            }
        }
#pragma unroll
        for (int o = LPR / 2; o > 0; o >>= 1) {
            a0 += __shfl_xor_sync(0xffffffffu, a0, o);
            a1 += __shfl_xor_sync(0xffffffffu, a1, o);
            a2 += __shfl_xor_sync(0xffffffffu, a2, o);
        }
        if (row < last && sl < 3) {
            const VT qi = sl == 0 ? a0 : (sl == 1 ? a1 : a2);
            qv[3 * (size_t)row + sl] = qi;
            acc[0] += (double)p[4 * (size_t)row + sl] * (double)qi;
        }
    }
    double tot[1];
    if (member_reduce<1>(b, m, acc, 1, tot)) {
        ms.pq = tot[0];
        if (!(tot[0] > 0.0)) {
            ms.breakdown = 1;
            ms.done = 1;
            ms.alpha = 0.0;
        } else {
            ms.alpha = ms.rz / tot[0];
        }
    }
}

template <typename VT>
__global__ void __launch_bounds__(kBT) k_bupdate(BatchArgs b, const VT* __restrict__ p, const VT* __restrict__ qv,
                                                 const VT* __restrict__ Minv, VT* __restrict__ x, VT* __restrict__ r,
                                                 VT* __restrict__ z, const uint8_t* __restrict__ pflag,
                                                 const double4* __restrict__ pn) {
    int m, i;
    block_nodes(b, m, i);
    MemberScalars& ms = b.ms[m];
    if (*(volatile int*)&ms.done) return;
    const VT alpha = (VT)ms.alpha;
    double acc[2] = {0.0, 0.0};
    if (i >= 0) {
        VT rr[3], qq[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            x[3 * (size_t)i + k] += alpha * p[4 * (size_t)i + k];
            qq[k] = qv[3 * (size_t)i + k];
        }
        bproject3<VT>(pflag, pn, i, qq);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            rr[k] = r[3 * (size_t)i + k] - alpha * qq[k];
            r[3 * (size_t)i + k] = rr[k];
        }
        const VT* M = Minv + (size_t)i * 9;
        VT zz[3];
#pragma unroll
        for (int k = 0; k < 3; k++) zz[k] = M[k * 3 + 0] * rr[0] + M[k * 3 + 1] * rr[1] + M[k * 3 + 2] * rr[2];
        bproject3<VT>(pflag, pn, i, zz);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            z[3 * (size_t)i + k] = zz[k];
            acc[0] += (double)rr[k] * (double)zz[k];
            acc[1] += (double)rr[k] * (double)rr[k];
        }
    }
    double tot[2];
    if (member_reduce<2>(b, m, acc, 2, tot)) {
        ms.beta = tot[0] / ms.rz;
        ms.rz = tot[0];
        ms.rr = tot[1];
        ms.it += 1;
        if (tot[1] <= ms.tol2 || ms.it >= ms.maxit || !(tot[1] == tot[1])) ms.done = 1;
    }
}

}  // namespace

template <typename VT>
void launch_bpcg_init(const BatchArgs& b, const double* g, const VT* Minv, VT* x, VT* r, VT* z, VT* p0, double eta2,
                      double abs_tol2, int tol_mode, int maxit, const uint8_t* pflag, const double4* pn,
                      cudaStream_t st) {
    k_bpcg_init<VT><<<b.nblocks, kBT, 0, st>>>(b, g, Minv, x, r, z, p0, eta2, abs_tol2, tol_mode, maxit, pflag, pn);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

template <typename HT, typename VT>
void launch_bpcg_iter(const BatchArgs& b, const int* row_ptr, const int* col, const HT* H, const VT* Minv,
                      const VT* z_in, const VT* p_old, VT* p_new, VT* qv, VT* x, VT* r, VT* z,
                      const uint8_t* pflag, const double4* pn, cudaStream_t st) {
    k_bform_p<VT><<<b.nblocks, kBT, 0, st>>>(b, z_in, p_old, p_new);
    const int groups = (b.max_row_blocks + 2) / 2;
    if (groups <= 4)
        k_bspmv_g<HT, VT, 4><<<b.nblocks, kBT, 0, st>>>(b, row_ptr, col, H, p_new, qv);
    else if (groups <= 8)
        k_bspmv_g<HT, VT, 8><<<b.nblocks, kBT, 0, st>>>(b, row_ptr, col, H, p_new, qv);
    else
        k_bspmv_g<HT, VT, 16><<<b.nblocks, kBT, 0, st>>>(b, row_ptr, col, H, p_new, qv);
    k_bupdate<VT><<<b.nblocks, kBT, 0, st>>>(b, p_new, qv, Minv, x, r, z, pflag, pn);
    g_kernel_launches.fetch_add(3, std::memory_order_relaxed);
}

template void launch_bpcg_init<float>(const BatchArgs&, const double*, const float*, float*, float*, float*, float*,
                                      double, double, int, int, const uint8_t*, const double4*, cudaStream_t);
template void launch_bpcg_init<double>(const BatchArgs&, const double*, const double*, double*, double*, double*,
                                       double*, double, double, int, int, const uint8_t*, const double4*,
                                       cudaStream_t);
template void launch_bpcg_iter<float, float>(const BatchArgs&, const int*, const int*, const float*, const float*,
                                             const float*, const float*, float*, float*, float*, float*, float*,
                                             const uint8_t*, const double4*, cudaStream_t);
template void launch_bpcg_iter<double, double>(const BatchArgs&, const int*, const int*, const double*,
                                               const double*, const double*, const double*, double*, double*,
                                               double*, double*, double*, const uint8_t*, const double4*,
                                               cudaStream_t);

}  // namespace sors
