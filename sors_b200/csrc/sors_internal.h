// sors_internal.h -- device data layout and kernel launchers of libsors_b200.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <string>
#include <vector>

#include "../../include/sors_b200.h"

namespace sors {

// kernels launched by this library (diagnostic counter)
extern std::atomic<long long> g_kernel_launches;

// status bits raised by kernels
enum : int { kFlagInverted = 1, kFlagPcgBreakdown = 2, kFlagNaN = 4, kFlagTimeout = 8 };

// Reduction scratch: per-block partial sums + a completion counter per site.
constexpr int kRedBlocks = 1184;      // 148 SMs x 8
constexpr int kRedThreads = 256;
constexpr int kMaxScalars = 4;
constexpr int kMaxDevices = 64;  // per-device caches of launch attributes

struct DevScalars {
    // Newton / energy reductions
    double gnorm2;       // ||gradient||^2
    double dxnorm2;      // ||dx||^2
    double e_elem;       // sum of element energies
    double e_dof;        // per-DOF energy terms
    double gdx;          // gradient . dx
    double minedge;      // CFL
    double vmax;         // CFL
    // PCG
    double rz, pq, alpha, beta, rr, tol2, bnorm2;
    int it, done, maxit, breakdown;
    // MINRES (Lanczos vectors with Givens QR, minres.cu): gamma_{j-1},
    // gamma_j, delta_j, c_{j-1}, c_j, s_{j-1}, s_j and eta (the preconditioned
    // residual norm, signed); the solution update the last iteration left
    // pending (alpha1, alpha2, alpha3, c_{j+1} eta_j, 1 / gamma_j)
    double mr_gprev, mr_g, mr_delta, mr_cprev, mr_c, mr_sprev, mr_s, mr_eta;
    double mr_a1, mr_a2, mr_a3, mr_ceta, mr_ig;
    int mr_pending, mr_bad;
    int status;          // kFlag* bits
    unsigned counters[16];
};

// SoftCon fibre terms (cpp/src/energies/softconMuscle.cpp): per element a
// muscle group (-1 = none) and (m_x, m_y, m_z, stiffness); activation per group.
// group == nullptr means no element has a fibre term.
struct MuscleArgs {
    const int* group = nullptr;
    const double4* param = nullptr;
    const double* act = nullptr;
};

// Hessian value storage: nnzb 3x3 blocks in CSR order, each block's 9 values
// contiguous and row-major.  (Splitting entries 0-7 from entry 8 for 16-byte
// vector loads was measured slower in the SpMV.)  The PCG SpMV also reads
// this layout directly, two blocks (18 values) at a time in nine vector loads;
// the allocation carries 160 bytes of padding for its last group.
__host__ __device__ __forceinline__ size_t hval(size_t b, int rc, size_t nnzb) {
    (void)nnzb;
    return 9 * b + (size_t)rc;
}

// Element-owner tet assembly over node chunks (kernels.cu k_assemble_chunk).
// At mesh load the nodes are cut into chunks of nearby nodes (Morton order of
// the undeformed positions); a chunk lists the elements incident to any of its
// nodes, each once, and for each of those elements the chunk-local pair slot
// of every vertex the chunk owns.  The Hessian items (one per element block
// that sums into a CSR block) follow slot_item_ptr's order, re-encoded as
// (chunk-local element << 4 | v << 2 | w).
struct ChunkArgs {
    int nchunks = 0;
    const int* ch_ptr = nullptr;        // nchunks+1: positions in ch_rows
    const int* ch_rows = nullptr;       // node ids, chunk by chunk
    const int* ch_eptr = nullptr;       // nchunks+1: positions in ch_elems
    const int* ch_elems = nullptr;      // element ids, chunk by chunk
    const ushort4* ch_eslot = nullptr;  // chunk-local pair slot of local vertex v (0xffff: not owned)
    const uint16_t* items = nullptr;    // one per slot item, same order as slot_items
    int rows_max = 0, elems_max = 0, pairs_max = 0;
    int region_bytes = 0;       // gradient pairs
    int smem_bytes = 0;         // dynamic shared memory of one chunk block
    void* gen = nullptr;        // two-pass variant: generator records (HT, padded), E of them
    double* gradg = nullptr;    // two-pass variant: V P d_v of every element vertex, 12 per element
};

// Chunk limits and shared-memory size of the chunked assembly for a Hessian
// type size (4 or 8 bytes) and material (0 Neo-Hookean, 2 stable Neo-Hookean).
struct ChunkLimits {
    int rows, elems, pairs;
};
ChunkLimits chunk_limits(int hsize, int material);
size_t chunk_region_bytes(int hsize, int material, int max_pairs);
size_t chunk_smem_bytes(int hsize, int material, int max_pairs);

// Row-owner assembly arguments (tet or hex).
template <typename HT>
struct AsmArgs {
    int N, nv, E;
    const double* X;        // 3N undeformed
    const double* q;        // 3N current
    const int* conn;        // E*nv
    const double2* mat;     // (mu, lambda) per element
    const double* tshape;   // tets: d_0..d_2 and volume per element (10 doubles)
    MuscleArgs mus;
    const int* pair_ptr;    // N+1
    const int* pair_ev;     // e*8 + v
    const int* row_ptr;     // N+1 (blocks)
    const int* diag_slot;   // N: the diagonal block of each row
    const int* col;         // nnzb
    const int* slot_item_ptr;   // nnzb+1
    const uint16_t* slot_items; // k*nv + w
    const uint8_t* node_mask;   // 3 bits per node
    const double* mass;     // per node
    HT* H;                  // nnzb*9, blocks in CSR order (hval)
    long long nnzb;
    double* g_int;          // 3N (masked element gradient)
    int* status;
    int stage_per_warp;     // HT elements per warp of staging
    int material;           // 0 NH, 1 quartic test, 2 stable NH
    int project;
    int apply_mask;         // drop masked DOFs from element terms (not SQP)
    int neumann_override;   // diag = 1 on masked DOFs ("minimize_newton")
    int want_hess;
    double hscale;          // 0.5 for Crank-Nicolson with dt != 0
    double inertia_coef;    // diag m * coef
    ChunkArgs ch;           // element-owner tet assembly (used when ch.nchunks > 0)
    void* hex_tile = nullptr;      // hexes: 36 upper 3x3 blocks (HT) per element, written by k_hex_tiles
    double* hex_gtile = nullptr;   // hexes: 8 gradient rows per element
    const int* hex_blk_row = nullptr;  // hexes: the row of each CSR block (k_hex_gather_blocks)
};

struct PressureArgs {
    int nsurf;                  // surface nodes with faces
    const int* surf_nodes;      // node id per surface row
    const int* sface_ptr;       // nsurf+1
    const int* sface_fl;        // face*4 + local vertex index
    const int* faces;           // F * fnv
    const int* face_group;
    int fnv;
    const double* pressure;     // per group
    const double* q;
    double* f_ext;              // 3N (written for surface nodes)
};

// Member-segmented PCG (batched.cu): a handle holding several independent
// meshes runs one preconditioned CG per member in the same launches.  Thread
// blocks of kBatchThreads nodes never straddle members.
constexpr int kBatchThreads = 256;
struct MemberScalars {
    double rz, rr, pq, alpha, beta, tol2, bnorm2, abs2;
    int it, done, breakdown, maxit;
    unsigned counter[4];
};
struct BatchArgs {
    int nmem = 0, nblocks = 0;
    int max_row_blocks = 0;           // longest block row (the SpMV's lanes per row)
    const int* mem_node0 = nullptr;   // nmem + 1: first node of each member
    const int* mem_blk0 = nullptr;    // nmem + 1: first thread block of each member
    const int* blk_mem = nullptr;     // nblocks: member of each thread block
    MemberScalars* ms = nullptr;      // nmem
    double* partials = nullptr;       // 2 per thread block
};
template <typename VT>
void launch_bpcg_init(const BatchArgs& b, const double* g, const VT* Minv, VT* x, VT* r, VT* z, VT* p0, double eta2,
                      double abs_tol2, int tol_mode, int maxit, const uint8_t* pflag, const double4* pn,
                      cudaStream_t st);
template <typename HT, typename VT>
void launch_bpcg_iter(const BatchArgs& b, const int* row_ptr, const int* col, const HT* H, const VT* Minv,
                      const VT* z_in, const VT* p_old, VT* p_new, VT* qv, VT* x, VT* r, VT* z,
                      const uint8_t* pflag, const double4* pn, cudaStream_t st);

// Caps the grid of every kernel launched from this thread (kernels.cu).
void set_grid_cap(int blocks);

// Two-level preconditioner (no reference counterpart): block Jacobi plus an
// exact correction on the coarse space spanned, per aggregate of nodes, by the
// three translations and three rotations about the aggregate's centre.
struct CoarseArgs {
    int N = 0, nagg = 0, nc = 0;       // nodes, aggregates, coarse unknowns (6 nagg)
    const int* aid = nullptr;          // aggregate of each node
    const double4* agg_c = nullptr;    // centre (x, y, z), 1 / length scale
    const int* agg_ptr = nullptr;      // nagg + 1
    const int* agg_nodes = nullptr;    // nodes of each aggregate, ascending
    const uint8_t* fixed = nullptr;    // Neumann bits per node (those rows of P are zero)
    const float4* off = nullptr;       // (X_i - centre) / length scale, per node
};
void launch_coarse_galerkin_f(int npairs, const int* cpair_ptr, const int2* cpair_items, const int2* cpair_ab,
                              const int* col, const float* H, long long nnzb, const CoarseArgs& c, double* Ac,
                              cudaStream_t st);
void launch_coarse_galerkin_d(int npairs, const int* cpair_ptr, const int2* cpair_items, const int2* cpair_ab,
                              const int* col, const double* H, long long nnzb, const CoarseArgs& c, double* Ac,
                              cudaStream_t st);
void launch_coarse_invert(int nc, double* Ac, double* rowk, double* colk, cudaStream_t st);
template <typename VT>
void launch_to_vt_pad(int nc, int ld, const double* in, VT* out, cudaStream_t st);
template <typename VT>
void launch_coarse_restrict(const CoarseArgs& c, const VT* r, double* yc, cudaStream_t st);
template <typename VT>
void launch_tl_update_restrict(const CoarseArgs& c, const VT* p, const VT* qv, VT* x, VT* r, const uint8_t* pflag,
                               const double4* pn, double* yc, DevScalars* sc, cudaStream_t st);
// Runs of the restriction over contiguous aggregates (k_tl_update_restrict_runs):
// node blocks of 256 cut into runs of one aggregate; run k covers nodes
// [run_start[k], run_start[k+1]); block b holds runs [block_run_ptr[b],
// block_run_ptr[b+1]); aggregate a's runs are [agg_run_begin[a], agg_run_begin[a+1]).
struct CoarseRuns {
    const int* run_start = nullptr;      // nruns + 1
    const int* block_run_ptr = nullptr;  // node blocks + 1
    const int* agg_run_begin = nullptr;  // nagg + 1 (aggregates in run order)
    double* partial = nullptr;           // 6 per run
    int nruns = 0;
};
template <typename VT>
void launch_tl_update_restrict_runs(const CoarseArgs& c, const CoarseRuns& ru, const VT* p, const VT* qv, VT* x,
                                    VT* r, const uint8_t* pflag, const double4* pn, double* yc, DevScalars* sc,
                                    cudaStream_t st);
template <typename VT>
void launch_tl_coarse_z(const CoarseArgs& c, int ld, const VT* Ainv, const double* yc, const VT* r, const VT* Minv,
                        VT* z, int init, const uint8_t* pflag, const double4* pn, double* partials, DevScalars* sc,
                        cudaStream_t st);

// MINRES work vectors (kernels.cu, minres section), by the parity of the
// iteration j: Z[j & 1] padded z_j (four values per node), V[j & 1] the
// Lanczos vector v_j, W[j & 1] the update direction w_j; x the solution, q
// the SpMV output, Minv the SPD block-Jacobi inverse.
template <typename VT>
struct MinresBufs {
    VT* Z[2] = {nullptr, nullptr};
    VT* V[2] = {nullptr, nullptr};
    VT* W[2] = {nullptr, nullptr};
    VT* x = nullptr;
    VT* q = nullptr;
    const VT* Minv = nullptr;
};
template <typename HT, typename VT>
void launch_block_jacobi_abs(int N, const int* diag_slot, const HT* H, long long nnzb, VT* Minv, cudaStream_t st);
template <typename VT>
void launch_minres_init(int N, const double* g, const MinresBufs<VT>& b, bool with_z, double eta2, double abs_tol2,
                        int maxit, double* partials, DevScalars* sc, cudaStream_t st);
template <typename HT, typename VT>
void launch_minres_spmv(int N, int max_row_blocks, const int* row_ptr, const int* col, const HT* H, long long nnzb,
                        const MinresBufs<VT>& b, int par, double* partials, DevScalars* sc, cudaStream_t st);
template <typename VT>
void launch_minres_lanczos(int N, const MinresBufs<VT>& b, int par, double* partials, DevScalars* sc,
                           cudaStream_t st);
template <typename VT>
void launch_minres_lanczos_restrict(const CoarseArgs& c, const MinresBufs<VT>& b, int par, double* yc,
                                    const DevScalars* sc, cudaStream_t st);
template <typename VT>
void launch_minres_coarse_z(const CoarseArgs& c, int ld, const VT* Ainv, const double* yc, const MinresBufs<VT>& b,
                            int vpar, int init, double eta2, double abs_tol2, int maxit, double* partials,
                            DevScalars* sc, cudaStream_t st);
template <typename VT>
void launch_minres_finish(int N, const MinresBufs<VT>& b, int par, const DevScalars* sc, cudaStream_t st);

// Sets the message returned by sors_last_error on this thread (capi.cu).
void set_last_error(const std::string& msg);

// Launchers (kernels.cu)
template <typename HT>
void launch_assemble(const AsmArgs<HT>& a, int max_pairs, cudaStream_t st);
template <typename HT>
void launch_elem_rows(int E, int nv, const double* X, const double* q, const int* conn, const double2* mat,
                      const double* tsh, const MuscleArgs& mus, int material, int project, double* psi, double* grad, double* hess, int* status,
                      cudaStream_t st);
void launch_elem_energy(int E, int nv, const double* X, const double* q, const int* conn, const double2* mat,
                        const MuscleArgs& mus, int material, double* partials, DevScalars* sc, cudaStream_t st);
void launch_pressure_force(const PressureArgs& p, cudaStream_t st);
void launch_pressure_adj_corr(const PressureArgs& p, const uint8_t* node_mask, double s_scale, const double* lam,
                              double* y, cudaStream_t st);
void launch_tet_shapes(int E, const double* X, const int* conn, double* out, cudaStream_t st);
void launch_adjoint_elem(int E, int nv, const double* X, const double* q, const int* conn, const double2* mat,
                         const MuscleArgs& mus, int material, const double* lam, double* out, cudaStream_t st);
template <typename HT>
void launch_pressure_jac(const PressureArgs& p, const int* row_ptr, const int* col, const uint8_t* node_mask,
                         double cscale, HT* H, long long nnzb, cudaStream_t st);
void launch_finalize_grad(int N, const double* g_int, const double* f_ext, const double* q, const double* qPrev,
                          const double* vPrev, const double* gPrev, double* gPrevTmp, const double* mass,
                          const uint8_t* mask, const double* mval, double dt, int scheme, double alpha,
                          const double* grav, int neumann_override, int has_ext, double* g, double* partials,
                          DevScalars* sc, cudaStream_t st);
void launch_dof_energy(int N, const double* q, const double* qPrev, const double* vPrev, const double* mass,
                       const double* f_ext, int has_ext, double dt, int scheme, double alpha, const double* grav,
                       double* partials, DevScalars* sc, cudaStream_t st);
template <typename HT, typename VT>
void launch_block_jacobi(int N, const int* row_ptr, const int* diag_slot, const HT* H, long long nnzb, VT* Minv,
                         cudaStream_t st);
template <typename HT, typename VT>
void launch_pcg_init(int N, const double* g, const VT* Minv, VT* x, VT* r, VT* z, VT* p0, double eta2,
                     double abs_tol2, int maxit, const uint8_t* pflag, const double4* pn, double* partials,
                     DevScalars* sc, cudaStream_t st);
template <typename HT, typename VT>
void launch_pcg_spmv(int N, int max_row_blocks, const int* row_ptr, const int* col, const HT* H, long long nnzb,
                     const VT* p4, VT* qv, double* partials, DevScalars* sc, cudaStream_t st);
template <typename VT>
void launch_form_p(int N, const VT* z, const VT* p_old, VT* p_new, const DevScalars* sc, cudaStream_t st);
template <typename VT>
void launch_pcg_update(int N, const VT* p, const VT* qv, const VT* Minv, VT* x, VT* r, VT* z, const uint8_t* pflag,
                       const double4* pn, double* partials, DevScalars* sc, cudaStream_t st);
void launch_qp_x0(int N, const uint8_t* pflag, const double4* pn, const double* q, const double* qPrev,
                  const double* mval, double dt, double* x0, cudaStream_t st);
void launch_qp_warm(int N, const uint8_t* pflag, const double4* pn, const double* q, const double* qPrev,
                    const double* mval, double dt, const double* dx_prev, double* x0, cudaStream_t st);
template <typename VT>
void launch_add_vec(int n, const double* a, const VT* b, double* out, cudaStream_t st);
void launch_qp_check(int m, const int* cnode, const double4* cnb, const double* dx, const double* y,
                     const double* g, double* out, cudaStream_t st);
void launch_gather_nodes(int m, const int* node, const double* q, double* out, cudaStream_t st);
void launch_pair_axpy(int np, const int2* ij, const double4* coef, double* y, cudaStream_t st);
void launch_axpy(int n, double alpha, const double* x, double* y, cudaStream_t st);
template <typename VT>
void launch_newton_update(int n, const VT* dx, double alpha, double* q, const double* q0, double* partials,
                          DevScalars* sc, int counter, cudaStream_t st);
template <typename VT>
void launch_dot_gdx(int n, const double* g, const VT* dx, double* partials, DevScalars* sc, cudaStream_t st);
void launch_update_state(int n, const double* q, double* qPrev, double* vPrev, double* gPrev,
                         const double* gPrevTmp, double dt, int scheme, cudaStream_t st);
void launch_predict(int n, double* q, const double* vPrev, double dt, cudaStream_t st);
void launch_gather_dofs(int N, const double* src, const int* idx, double* dst, cudaStream_t st);
void launch_cfl(int E, int nv, const double* q, const int* conn, int n, const double* vPrev, double* partials,
                DevScalars* sc, cudaStream_t st);
template <typename HT>
void launch_spmv_plain(int N, const int* row_ptr, const int* col, const HT* H, long long nnzb, const double* x,
                       double* y, cudaStream_t st);

}  // namespace sors
