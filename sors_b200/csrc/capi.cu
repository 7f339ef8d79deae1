// capi.cu -- C ABI, mesh-load set-up and the Newton / PCG driver.
//
// One handle = one mesh resident on one GPU with one CUDA stream.  Set-up
// builds, once, the 3x3-block CSR pattern of the Hessian, the node -> (element,
// local vertex) pair lists and the slot-item lists that map every pair block
// to its CSR slot.  A step then runs, per Newton iteration: the row-owner
// assembly (gradient rows + Hessian block-rows), the follower-load rows, the
// gradient finalisation (integrator + Neumann rows), the block-Jacobi
// inverses, PCG in CUDA-graph chunks, and the update.  One host
// synchronisation per Newton iteration and one per PCG chunk.
#include <cuda_runtime.h>
#include <math.h>
#include <tuple>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <cstdio>
#include <new>
#include <string>
#include <thread>
#include <limits>
#include <vector>

#include "../../include/sors_b200.h"
#include "sors_internal.h"

using namespace sors;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

#define CK(expr)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (expr);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            return fail(SORS_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e_) +     \
                                           " at " #expr);                                         \
    } while (0)

constexpr int kPcgChunk = 16;  // PCG iterations per captured graph (even)

// SORS_VERBOSE=1 prints one line per Newton iteration to stderr.
bool verbose() {
    static int v = -1;
    if (v < 0) {
        const char* e = getenv("SORS_VERBOSE");
        v = (e && *e && *e != '0') ? 1 : 0;
    }
    return v == 1;
}

}  // namespace

void sors::set_last_error(const std::string& msg) { g_last_error = msg; }

struct SorsHandle {
    SorsSettings s{};
    int N = 0, E = 0, nv = 0, ndof = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    int64_t nnzb = 0;
    int max_pairs = 0;
    int max_row_blocks = 0;
    size_t bytes = 0;
    std::vector<void*> allocs;

    // mesh + state
    double *X = nullptr, *q = nullptr, *q0 = nullptr, *qPrev = nullptr, *vPrev = nullptr, *gPrev = nullptr,
           *gPrevTmp = nullptr, *g = nullptr, *g_int = nullptr, *f_ext = nullptr, *mass = nullptr, *mval = nullptr,
           *vforce = nullptr, *q_save = nullptr;
    int* conn = nullptr;
    double2* mat = nullptr;
    double* tshape = nullptr;  // tets: shape gradients and volume per element
    int *row_ptr = nullptr, *col = nullptr, *diag_slot = nullptr, *pair_ptr = nullptr, *pair_ev = nullptr,
        *slot_item_ptr = nullptr;
    uint16_t* slot_items = nullptr;
    // node numbering: internal node i is the caller's node n2o[i] (identity
    // when renum is false); every entry point converts at the boundary
    bool renum = false;
    std::vector<int> n2o, o2n;
    // element order: internal element e is the caller's element e2o[e]
    bool renum_e = false;
    std::vector<int> e2o;
    int *n2o_d = nullptr, *o2n_d = nullptr;
    double* perm_tmp = nullptr;           // 3N staging for device-side conversions
    std::vector<int> caller_row_ptr, caller_col, caller_blk;  // sors_hessian_bsr in caller numbering
    // element-owner tet assembly: node chunks (build_tet_chunks)
    ChunkArgs chunks;
    long long chunk_elem_total = 0;  // sum over chunks of their element counts
    int asm_variant = 0;  // 0: chunked element-owner where it applies, 1: row-owner, 2: two-pass chunked
    void* hex_tile = nullptr;         // hexes: element tiles of the element-owner assembly
    double* hex_gtile = nullptr;
    int* hex_blk_row = nullptr;       // hexes: the row of each CSR block
    void* chunk_gen = nullptr;        // two-pass variant: element generator records
    double* chunk_gradg = nullptr;    // two-pass variant: element gradient rows
    uint8_t* node_mask = nullptr;
    std::vector<uint8_t> mask_h;
    std::vector<int> row_ptr_h, col_h;

    // linear system
    void* H = nullptr;
    void* Minv = nullptr;
    void *x = nullptr, *r = nullptr, *z = nullptr, *p0 = nullptr, *p1 = nullptr, *qv = nullptr;
    double* partials = nullptr;
    DevScalars* sc = nullptr;
    DevScalars* sc_host = nullptr;  // pinned
    int* status = nullptr;          // points into sc

    // follower load
    bool has_pressure = false, has_vforce = false, has_neumann = false;
    int n_faces = 0, fnv = 0, n_groups = 0, nsurf = 0;
    int *faces = nullptr, *face_group = nullptr, *surf_nodes = nullptr, *sface_ptr = nullptr, *sface_fl = nullptr;
    double* pressure_d = nullptr;

    // host copies used by the adjoint
    std::vector<double> youngs_h, poisson_h, mass_h;
    std::vector<int> mgroup_h;
    double *adj_l = nullptr, *adj_y = nullptr, *adj_e = nullptr;
    double *adj_q = nullptr, *adj_pg = nullptr;  // q_next of the last adjoint step; group pressures scratch
    bool adj_ready = false;                      // adj_l and adj_q hold the last adjoint step

    // SoftCon fibre terms
    int* mgroup = nullptr;
    double4* mparam = nullptr;
    double* mact = nullptr;
    int n_mgroups = 0;

    // contact (planeContact / diskContact) and the SQP subproblem
    struct Plane { double p[3], n[3]; };
    struct Disk { double c[3], n[3], r; };
    std::vector<Plane> planes;
    std::vector<int> plane_surf, plane_mask;
    std::vector<Disk> disks;
    // one DiskContact per group: its disks, candidate vertices, captured
    // footprint (global disk index per candidate, -1 none) and frozen flag
    struct DiskGroup {
        std::vector<int> disks, surf, mask;
        bool frozen = false;
    };
    std::vector<DiskGroup> disk_groups;
    uint8_t* pflag_d = nullptr;
    double4* pn_d = nullptr;
    std::vector<uint8_t> pflag_h;
    std::vector<double4> pn_h;
    int* cnode_d = nullptr;
    double4* cnb_d = nullptr;
    double *cout_d = nullptr, *cpos_d = nullptr;
    int c_cap = 0;
    double *qp_x0 = nullptr, *qp_y = nullptr, *qp_g2 = nullptr, *qp_dx = nullptr;
    int last_active = 0;
    std::vector<int> held_nodes;      // contacts held at the end of the last SQP step
    std::vector<double> held_normals;
    // maxDistance pairs |x_i - x_j| <= d (always active); in the SQP subproblem
    // the held pairs enter through a Schur complement on the node-projected
    // system: one projected solve w_k per held pair, cached in md_w
    std::vector<int> md_i, md_j;
    std::vector<double> md_d;
    std::vector<char> md_work;        // pair working set (persists over the Newton iterations)
    std::vector<int> held_pairs;      // pairs held at the end of the last SQP step
    std::vector<double> held_mu;      // and their multipliers
    std::vector<int> adj_pairs;       // held pairs and multipliers for the next adjoint steps
    std::vector<double> adj_mu;
    int* md_nodes_d = nullptr;        // i_0, j_0, i_1, j_1, ...
    double* md_pos_d = nullptr;       // gather buffer, 6 per pair
    int2* md_ij_d = nullptr;
    double4* md_coef_d = nullptr;
    int md_cap = 0;
    std::vector<double*> md_w;        // pool of n-vectors
    // two-level preconditioner (settings.two_level): node aggregates, the
    // Galerkin coarse matrix and its inverse (refreshed when PCG slows down)
    bool tl_ready = false, tl_active = false;
    bool tl_proj = false;             // the coarse operator came from the projected Hessian
    size_t l2_window_bytes = 0;       // coarse inverse marked persisting in L2 (keep_coarse_in_l2)
    double tl_ref_rate = 0.0;
    CoarseArgs cargs;
    CoarseRuns cruns;                 // nruns > 0: aggregates are contiguous node ranges
    int tl_npairs = 0;
    int *tl_pair_ptr = nullptr;
    int2 *tl_items = nullptr, *tl_ab = nullptr;
    double *tl_Ac = nullptr, *tl_yc = nullptr, *tl_rowk = nullptr, *tl_colk = nullptr;
    void* tl_Ainv = nullptr;
    int tl_ld = 0;                    // leading dimension of tl_Ainv (nc rounded up to 16 bytes)
    int tl_refreshes = 0;

    // projection used by the PCG kernels (null: none)
    const uint8_t* proj_flag = nullptr;
    const double4* proj_n = nullptr;
    int pcg_exec_mode = 0;  // bit 0 projected, bit 1 two-level, bit 2 member-segmented
    // several independent meshes in one handle (sors_set_members): one PCG per member
    BatchArgs batch;
    std::vector<int> mem_node0_h;
    std::vector<MemberScalars> ms_h;

    // PCG chunk graph
    cudaGraphExec_t pcg_exec = nullptr;
    long long pcg_graph_kernels = 0;  // kernel nodes of the captured chunk
    int64_t n_hess_evals = 0, n_grad_evals = 0;  // system evaluations with / without the Hessian
    bool graph_failed = false;

    double prev_gnorm = -1.0;
    // PCG directions with non-positive curvature met during the last step:
    // count and the most negative Rayleigh quotient p'Hp / p'p
    int step_indefinite = 0;
    double step_min_rq = INFINITY;
    // project_spd == 2: the exact Hessian first, the projected one for this
    // iteration after PCG met negative curvature
    bool proj_fallback = false;
    // >= 0: the projection of the next assemblies regardless of the settings
    // (the MINRES coarse operator is built from the projected Hessian)
    int force_project = -1;
    // MINRES (settings.linear_solver 1): the two update-direction buffers,
    // and whether the chunk graph runs MINRES iterations
    void* mr_w[2] = {nullptr, nullptr};
    bool mr_active = false;
};

namespace {

bool mixed(const SorsHandle* h) { return h->s.precision == 1; }

// (mu, lambda) of an element from Young's modulus and Poisson's ratio
// (neoHookean.cpp:10-11); stable Neo-Hookean reparameterises them as
// mu_s = 4/3 mu, lambda_s = lambda + 5/8 mu_s (stableNeoHookean.cpp:10-15).
double2 lame_params(double Ey, double nu, int material) {
    double2 m;
    m.y = (Ey * nu) / ((1 + nu) * (1 - 2 * nu));
    m.x = Ey / (2 * (1 + nu));
    if (material == 2) {
        m.x *= 4.0 / 3.0;
        m.y += 5.0 / 8.0 * m.x;
    }
    return m;
}
MuscleArgs muscles(const SorsHandle* h) {
    MuscleArgs m;
    if (h->mgroup) { m.group = h->mgroup; m.param = h->mparam; m.act = h->mact; }
    return m;
}
size_t hsize(const SorsHandle* h) { return mixed(h) ? sizeof(float) : sizeof(double); }

// Host<->device copies and fills go through the handle's stream: it is a
// non-blocking stream, so legacy-stream operations would not be ordered with
// its kernels.  They are complete when these return.
cudaError_t h2d(SorsHandle* h, void* dst, const void* src, size_t bytes) {
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, h->stream);
    return e == cudaSuccess ? cudaStreamSynchronize(h->stream) : e;
}
cudaError_t d2h(SorsHandle* h, void* dst, const void* src, size_t bytes) {
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, h->stream);
    return e == cudaSuccess ? cudaStreamSynchronize(h->stream) : e;
}
cudaError_t dzero(SorsHandle* h, void* dst, size_t bytes) {
    cudaError_t e = cudaMemsetAsync(dst, 0, bytes, h->stream);
    return e == cudaSuccess ? cudaStreamSynchronize(h->stream) : e;
}

int dalloc(SorsHandle* h, void** p, size_t bytes) {
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        return fail(SORS_ERR_OOM, std::string("device allocation of ") + std::to_string(bytes) +
                                      " bytes failed: " + cudaGetErrorString(e));
    }
    h->allocs.push_back(*p);
    h->bytes += bytes;
    return SORS_OK;
}

template <typename T>
int dalloc_t(SorsHandle* h, T** p, size_t count) {
    return dalloc(h, (void**)p, count * sizeof(T));
}

template <typename T>
int upload(SorsHandle* h, T** p, const T* src, size_t count) {
    int st = dalloc_t(h, p, count);
    if (st) return st;
    if (count) CK(h2d(h, *p, src, count * sizeof(T)));
    return SORS_OK;
}

double tet_vol_h(const double* a, const double* b, const double* c, const double* d) {
    double ab[3], ac[3], ad[3];
    for (int k = 0; k < 3; k++) { ab[k] = b[k] - a[k]; ac[k] = c[k] - a[k]; ad[k] = d[k] - a[k]; }
    double cx = ac[1] * ad[2] - ac[2] * ad[1], cy = ac[2] * ad[0] - ac[0] * ad[2], cz = ac[0] * ad[1] - ac[1] * ad[0];
    return fabs(ab[0] * cx + ab[1] * cy + ab[2] * cz) / 6.0;
}

// undeformed volume: tet (tetrahedron.cpp:137-149), hex 5-tet split (hexahedron.cpp:106-130)
double elem_volume(const double* X, const int* en, int nv) {
    if (nv == 4) return tet_vol_h(X + 3 * en[0], X + 3 * en[1], X + 3 * en[2], X + 3 * en[3]);
    static const int T5[5][4] = {{0, 1, 3, 4}, {1, 2, 3, 6}, {1, 4, 5, 6}, {3, 4, 6, 7}, {1, 3, 4, 6}};
    double v = 0;
    for (int t = 0; t < 5; t++)
        v += tet_vol_h(X + 3 * en[T5[t][0]], X + 3 * en[T5[t][1]], X + 3 * en[T5[t][2]], X + 3 * en[T5[t][3]]);
    return v;
}

template <typename F>
void parallel_for(int n, F&& f) {
    int nt = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    if (n < 4096 || nt == 1) {
        f(0, n);
        return;
    }
    std::vector<std::thread> ts;
    int chunk = (n + nt - 1) / nt;
    for (int t = 0; t < nt; t++) {
        int a = t * chunk, b = std::min(n, a + chunk);
        if (a >= b) break;
        ts.emplace_back([&f, a, b]() { f(a, b); });
    }
    for (auto& t : ts) t.join();
}

// Host copies of the pattern's pair lists and slot items (set-up only).
struct PatternHost {
    std::vector<int> pair_ptr, pair_ev, slot_cnt;
    std::vector<uint16_t> items;
};

// Builds pattern, pair lists and slot-item lists (host), then uploads.
int build_pattern(SorsHandle* h, const int32_t* conn, PatternHost* keep) {
    const int N = h->N, E = h->E, nv = h->nv;
    std::vector<int> pair_ptr(N + 1, 0);
    for (long long t = 0; t < (long long)E * nv; t++) pair_ptr[conn[t] + 1]++;
    for (int i = 0; i < N; i++) pair_ptr[i + 1] += pair_ptr[i];
    std::vector<int> pair_ev((size_t)E * nv);
    {
        std::vector<int> pos(pair_ptr.begin(), pair_ptr.end() - 1);
        for (int e = 0; e < E; e++)
            for (int v = 0; v < nv; v++) pair_ev[pos[conn[(size_t)e * nv + v]]++] = e * 8 + v;
    }
    int max_pairs = 0;
    for (int i = 0; i < N; i++) max_pairs = std::max(max_pairs, pair_ptr[i + 1] - pair_ptr[i]);
    if ((long long)max_pairs * nv > 65535)
        return fail(SORS_ERR_UNSUPPORTED, "a node has too many incident elements for the slot maps");
    h->max_pairs = max_pairs;

    // block pattern: row i = sorted unique nodes of incident elements
    std::vector<int> row_len(N, 0);
    std::vector<std::vector<int>> rows_tmp;  // filled per chunk
    std::vector<int> row_ptr(N + 1, 0);
    std::vector<int> cols_all;
    {
        std::vector<std::vector<int>> per(N);
        parallel_for(N, [&](int a, int b) {
            std::vector<int> buf;
            for (int i = a; i < b; i++) {
                buf.clear();
                for (int t = pair_ptr[i]; t < pair_ptr[i + 1]; t++) {
                    int e = pair_ev[t] >> 3;
                    for (int w = 0; w < nv; w++) buf.push_back(conn[(size_t)e * nv + w]);
                }
                if (buf.empty()) buf.push_back(i);  // isolated node keeps a diagonal block
                std::sort(buf.begin(), buf.end());
                buf.erase(std::unique(buf.begin(), buf.end()), buf.end());
                per[i] = buf;
            }
        });
        for (int i = 0; i < N; i++) row_ptr[i + 1] = row_ptr[i] + (int)per[i].size();
        if ((long long)row_ptr[N] > 0x7fffffffLL / 9)
            return fail(SORS_ERR_UNSUPPORTED, "Hessian pattern exceeds the 32-bit index range");
        cols_all.resize(row_ptr[N]);
        for (int i = 0; i < N; i++) std::copy(per[i].begin(), per[i].end(), cols_all.begin() + row_ptr[i]);
    }
    const int nnzb = row_ptr[N];
    h->nnzb = nnzb;
    for (int i = 0; i < N; i++) {
        int nb = row_ptr[i + 1] - row_ptr[i];
        if (nb > 255 * 9) return fail(SORS_ERR_UNSUPPORTED, "Hessian row too long");
        h->max_row_blocks = std::max(h->max_row_blocks, nb);
    }
    std::vector<int> diag(N);
    for (int i = 0; i < N; i++) {
        auto b = cols_all.begin() + row_ptr[i], e = cols_all.begin() + row_ptr[i + 1];
        diag[i] = (int)(std::lower_bound(b, e, i) - cols_all.begin());
    }
    // slot-item lists: items of slot b = (k*nv + w) for pairs k of row i whose vertex w is col[b]
    std::vector<int> slot_cnt(nnzb + 1, 0);
    std::vector<int> item_slot((size_t)E * nv * nv);
    parallel_for(N, [&](int a, int b) {
        for (int i = a; i < b; i++) {
            auto cb = cols_all.begin() + row_ptr[i], ce = cols_all.begin() + row_ptr[i + 1];
            for (int t = pair_ptr[i]; t < pair_ptr[i + 1]; t++) {
                int e = pair_ev[t] >> 3;
                for (int w = 0; w < nv; w++) {
                    int j = conn[(size_t)e * nv + w];
                    item_slot[(size_t)t * nv + w] = (int)(std::lower_bound(cb, ce, j) - cols_all.begin());
                }
            }
        }
    });
    for (size_t t = 0; t < item_slot.size() && t < (size_t)pair_ptr[N] * nv; t++) slot_cnt[item_slot[t] + 1]++;
    for (int b = 0; b < nnzb; b++) slot_cnt[b + 1] += slot_cnt[b];
    std::vector<uint16_t> items((size_t)pair_ptr[N] * nv);
    {
        std::vector<int> pos(slot_cnt.begin(), slot_cnt.end() - 1);
        for (int i = 0; i < N; i++)
            for (int t = pair_ptr[i]; t < pair_ptr[i + 1]; t++) {
                int k = t - pair_ptr[i];
                for (int w = 0; w < nv; w++) items[pos[item_slot[(size_t)t * nv + w]]++] = (uint16_t)(k * nv + w);
            }
    }
    int st;
    if ((st = upload(h, &h->pair_ptr, pair_ptr.data(), pair_ptr.size()))) return st;
    if ((st = upload(h, &h->pair_ev, pair_ev.data(), pair_ev.size()))) return st;
    if ((st = upload(h, &h->row_ptr, row_ptr.data(), row_ptr.size()))) return st;
    {
        // 4 ints of zero padding: the SpMV reads column indices 4 at a time
        // from 16-byte aligned groups, the last of which may run past nnzb
        std::vector<int> col_pad(cols_all.size() + 4, 0);
        std::copy(cols_all.begin(), cols_all.end(), col_pad.begin());
        if ((st = upload(h, &h->col, col_pad.data(), col_pad.size()))) return st;
    }
    if ((st = upload(h, &h->diag_slot, diag.data(), diag.size()))) return st;
    if ((st = upload(h, &h->slot_item_ptr, slot_cnt.data(), slot_cnt.size()))) return st;
    if ((st = upload(h, &h->slot_items, items.data(), items.size()))) return st;
    h->row_ptr_h = std::move(row_ptr);
    h->col_h = std::move(cols_all);
    if (keep) {
        keep->pair_ptr = std::move(pair_ptr);
        keep->pair_ev = std::move(pair_ev);
        keep->slot_cnt = std::move(slot_cnt);
        keep->items = std::move(items);
    }
    return SORS_OK;
}

// Node chunks of the element-owner tet assembly.  Nodes are taken in Morton
// order of their undeformed positions and cut greedily into chunks of at most
// chunk_limits(...) rows, incident elements and (element, vertex) pairs; each
// chunk lists its incident elements once, in first-seen order.  Meshes where
// a single node exceeds the limits keep the row-owner assembly only.
int build_tet_chunks(SorsHandle* h, const int32_t* conn, const double* X, const PatternHost& ph) {
    h->chunks = ChunkArgs{};
    if (h->nv != 4 || !(h->s.material == 0 || h->s.material == 2) || h->N == 0) return SORS_OK;
    const int N = h->N, E = h->E;
    const int hsz = mixed(h) ? 4 : 8;
    const ChunkLimits lim = chunk_limits(hsz, h->s.material);
    // two blocks per SM must fit (227 KB of shared memory per SM)
    if (chunk_smem_bytes(hsz, h->s.material, h->max_pairs) > 113 * 1024) return SORS_OK;
    for (int i = 0; i < N; i++) {
        const int np = ph.pair_ptr[i + 1] - ph.pair_ptr[i];
        if (np > lim.pairs || np > lim.elems) return SORS_OK;
    }
    // Morton order of the undeformed positions (21 bits per axis)
    double lo[3] = {X[0], X[1], X[2]}, hi[3] = {X[0], X[1], X[2]};
    for (int i = 0; i < N; i++)
        for (int k = 0; k < 3; k++) {
            lo[k] = std::min(lo[k], X[3 * (size_t)i + k]);
            hi[k] = std::max(hi[k], X[3 * (size_t)i + k]);
        }
    auto spread = [](uint64_t v) {
        v &= 0x1fffff;
        v = (v | v << 32) & 0x1f00000000ffffULL;
        v = (v | v << 16) & 0x1f0000ff0000ffULL;
        v = (v | v << 8) & 0x100f00f00f00f00fULL;
        v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
        v = (v | v << 2) & 0x1249249249249249ULL;
        return v;
    };
    std::vector<std::pair<uint64_t, int>> key(N);
    parallel_for(N, [&](int a, int b) {
        for (int i = a; i < b; i++) {
            uint64_t code = 0;
            for (int k = 0; k < 3; k++) {
                const double ext = hi[k] - lo[k];
                const double u = ext > 0 ? (X[3 * (size_t)i + k] - lo[k]) / ext : 0.0;
                const uint64_t c = (uint64_t)std::min(2097151.0, std::max(0.0, u * 2097151.0));
                code |= spread(c) << k;
            }
            key[i] = {code, i};
        }
    });
    std::sort(key.begin(), key.end());
    // greedy cut
    std::vector<int> ch_ptr{0}, ch_rows, ch_eptr{0}, ch_elems;
    ch_rows.reserve(N);
    ch_elems.reserve((size_t)E * 3 / 2);
    std::vector<int> mark(E, -1);
    int cur = 0, nr = 0, ne = 0, np = 0;
    for (int o = 0; o < N; o++) {
        const int i = key[o].second;
        const int p0 = ph.pair_ptr[i], p1 = ph.pair_ptr[i + 1];
        int fresh = 0;
        for (int t = p0; t < p1; t++) fresh += mark[ph.pair_ev[t] >> 3] != cur;
        if (nr > 0 && (nr + 1 > lim.rows || ne + fresh > lim.elems || np + (p1 - p0) > lim.pairs)) {
            cur++;
            ch_ptr.push_back((int)ch_rows.size());
            ch_eptr.push_back((int)ch_elems.size());
            nr = ne = np = 0;
        }
        ch_rows.push_back(i);
        nr++;
        np += p1 - p0;
        for (int t = p0; t < p1; t++) {
            const int e = ph.pair_ev[t] >> 3;
            if (mark[e] != cur) {
                mark[e] = cur;
                ch_elems.push_back(e);
                ne++;
            }
        }
    }
    ch_ptr.push_back((int)ch_rows.size());
    ch_eptr.push_back((int)ch_elems.size());
    const int nch = (int)ch_ptr.size() - 1;
    // per chunk: pair slots of owned vertices, and the (element, v) of every pair
    std::vector<uint16_t> eslot(ch_elems.size() * 4, 0xffff);
    std::vector<uint32_t> pair_sv(ph.pair_ev.size());
    parallel_for(nch, [&](int a, int b) {
        std::vector<std::pair<int, int>> loc;
        for (int c = a; c < b; c++) {
            loc.clear();
            for (int k = ch_eptr[c]; k < ch_eptr[c + 1]; k++) loc.push_back({ch_elems[k], k - ch_eptr[c]});
            std::sort(loc.begin(), loc.end());
            int slot = 0;
            for (int p = ch_ptr[c]; p < ch_ptr[c + 1]; p++) {
                const int r = ch_rows[p];
                for (int t = ph.pair_ptr[r]; t < ph.pair_ptr[r + 1]; t++, slot++) {
                    const int e = ph.pair_ev[t] >> 3, v = ph.pair_ev[t] & 7;
                    const int sidx = std::lower_bound(loc.begin(), loc.end(), std::make_pair(e, -1))->second;
                    eslot[(size_t)(ch_eptr[c] + sidx) * 4 + v] = (uint16_t)slot;
                    pair_sv[t] = (uint32_t)(sidx << 2 | v);
                }
            }
        }
    });
    // items in slot_items' order: (pair k of row r, vertex w) -> (element slot, v, w)
    std::vector<uint16_t> items(ph.items.size());
    const std::vector<int>& rp = h->row_ptr_h;
    parallel_for(N, [&](int a, int b) {
        for (int r = a; r < b; r++)
            for (int bk = rp[r]; bk < rp[r + 1]; bk++)
                for (int it = ph.slot_cnt[bk]; it < ph.slot_cnt[bk + 1]; it++) {
                    const int o = ph.items[it], k = o / 4, w = o % 4;
                    const uint32_t sv = pair_sv[ph.pair_ptr[r] + k];
                    items[it] = (uint16_t)(sv << 2 | (uint32_t)w);
                }
    });
    // every index the kernel derives from these tables stays inside its
    // shared-memory arrays: check them all here, before any upload
    std::vector<int> chunk_of_row(N, -1);
    for (int c = 0; c < nch; c++) {
        const int nrc = ch_ptr[c + 1] - ch_ptr[c], nec = ch_eptr[c + 1] - ch_eptr[c];
        if (nrc < 1 || nrc > lim.rows || nec < 0 || nec > lim.elems || nec > 4095)
            return fail(SORS_ERR_ARG, "internal: node chunk exceeds its limits");
        int npc = 0;
        for (int p = ch_ptr[c]; p < ch_ptr[c + 1]; p++) {
            const int r = ch_rows[p];
            if (r < 0 || r >= N || chunk_of_row[r] != -1) return fail(SORS_ERR_ARG, "internal: bad chunk row");
            chunk_of_row[r] = c;
            npc += ph.pair_ptr[r + 1] - ph.pair_ptr[r];
        }
        if (npc > lim.pairs) return fail(SORS_ERR_ARG, "internal: node chunk exceeds its pair limit");
        int owned = 0;
        for (size_t k = (size_t)ch_eptr[c] * 4; k < (size_t)ch_eptr[c + 1] * 4; k++) {
            if (eslot[k] == 0xffff) continue;
            if (eslot[k] >= npc) return fail(SORS_ERR_ARG, "internal: chunk pair slot out of range");
            owned++;
        }
        if (owned != npc) return fail(SORS_ERR_ARG, "internal: chunk pair slots incomplete");
    }
    for (int r = 0; r < N; r++) {
        if (chunk_of_row[r] < 0) return fail(SORS_ERR_ARG, "internal: node missing from the chunks");
        const int c = chunk_of_row[r], nec = ch_eptr[c + 1] - ch_eptr[c];
        for (int bk = rp[r]; bk < rp[r + 1]; bk++)
            for (int it = ph.slot_cnt[bk]; it < ph.slot_cnt[bk + 1]; it++)
                if ((int)(items[it] >> 4) >= nec) return fail(SORS_ERR_ARG, "internal: chunk item out of range");
    }
    if ((long long)nch > 0x7fffffffLL) return fail(SORS_ERR_ARG, "internal: too many node chunks");
    int st;
    ChunkArgs& c = h->chunks;
    int *d_ptr = nullptr, *d_rows = nullptr, *d_eptr = nullptr, *d_elems = nullptr;
    uint16_t *d_eslot = nullptr, *d_items = nullptr;
    if ((st = upload(h, &d_ptr, ch_ptr.data(), ch_ptr.size()))) return st;
    if ((st = upload(h, &d_rows, ch_rows.data(), ch_rows.size()))) return st;
    if ((st = upload(h, &d_eptr, ch_eptr.data(), ch_eptr.size()))) return st;
    if ((st = upload(h, &d_elems, ch_elems.data(), ch_elems.size()))) return st;
    if ((st = upload(h, &d_eslot, eslot.data(), eslot.size()))) return st;
    if ((st = upload(h, &d_items, items.data(), items.size()))) return st;
    c.ch_ptr = d_ptr; c.ch_rows = d_rows; c.ch_eptr = d_eptr; c.ch_elems = d_elems;
    c.ch_eslot = reinterpret_cast<const ushort4*>(d_eslot);
    c.items = d_items;
    c.rows_max = lim.rows; c.elems_max = lim.elems; c.pairs_max = lim.pairs;
    c.region_bytes = (int)chunk_region_bytes(hsz, h->s.material, h->max_pairs);
    c.smem_bytes = (int)chunk_smem_bytes(hsz, h->s.material, h->max_pairs);
    c.nchunks = nch;
    h->chunk_elem_total = (long long)ch_elems.size();
    return SORS_OK;
}

double inertia_coef(const SorsHandle* h, double dt) {
    if (dt == 0.0) return 0.0;
    double a = h->s.damping_alpha;
    if (h->s.time_stepping == 0) return 1.0 / (dt * dt) + a / dt;
    return 2.0 / (dt * dt) + 2.0 * a / dt;
}

int method(const SorsHandle* h) { return h->s.solver_method; }

// The Newton matrix's follower-load coefficient relative to the reference's
// p/6: 1, or with settings.pressure_jac_exact the exact derivative of the quad
// force -p A / 4 (p/8, 0.75 of p/6; triangles are exact at p/6).
double pressure_jac_scale(const SorsHandle* h) { return (h->s.pressure_jac_exact && h->fnv == 4) ? 0.75 : 1.0; }

PressureArgs pressure_args(SorsHandle* h) {
    PressureArgs p;
    p.nsurf = h->nsurf; p.surf_nodes = h->surf_nodes; p.sface_ptr = h->sface_ptr; p.sface_fl = h->sface_fl;
    p.faces = h->faces; p.face_group = h->face_group; p.fnv = h->fnv; p.pressure = h->pressure_d; p.q = h->q;
    p.f_ext = h->f_ext;
    return p;
}

// f_ext = vertexForce + pressure forces at h->q
int compute_external(SorsHandle* h) {
    if (!(h->has_vforce || h->has_pressure)) return SORS_OK;
    if (h->has_vforce)
        CK(cudaMemcpyAsync(h->f_ext, h->vforce, sizeof(double) * h->ndof, cudaMemcpyDeviceToDevice, h->stream));
    else
        CK(cudaMemsetAsync(h->f_ext, 0, sizeof(double) * h->ndof, h->stream));
    if (h->has_pressure) launch_pressure_force(pressure_args(h), h->stream);
    return SORS_OK;
}

// Gradient (and Hessian when want_hess) at h->q.  Leaves gnorm2 in sc.
// Assembly modes: the step's own (Neumann rows identity for "minimize_newton",
// unmasked otherwise), Neumann rows identity regardless of the method, or the
// unmasked system.
enum AsmMode { kAsmStep = 0, kAsmMaskedIdentity = 1, kAsmFull = 2 };

// Assembly arguments of the handle at h->q for one evaluation.
template <typename HT>
AsmArgs<HT> asm_args(SorsHandle* h, double dt, bool want_hess, AsmMode mode, int project) {
    AsmArgs<HT> a;
    a.N = h->N; a.nv = h->nv; a.E = h->E; a.X = h->X; a.q = h->q; a.conn = h->conn; a.mat = h->mat; a.mus = muscles(h);
    a.tshape = h->tshape;
    a.pair_ptr = h->pair_ptr; a.pair_ev = h->pair_ev; a.row_ptr = h->row_ptr; a.col = h->col;
    a.diag_slot = h->diag_slot;
    a.slot_item_ptr = h->slot_item_ptr; a.slot_items = h->slot_items; a.node_mask = h->node_mask; a.mass = h->mass;
    a.H = (HT*)h->H; a.nnzb = h->nnzb; a.g_int = h->g_int; a.status = h->status;
    a.stage_per_warp = h->max_pairs * h->nv * 9;
    a.material = h->s.material; a.project = project;
    a.apply_mask = mode == kAsmFull ? 0 : 1;
    a.neumann_override = mode == kAsmFull ? 0
                         : ((mode == kAsmMaskedIdentity || method(h) == 0) && h->has_neumann) ? 1 : 0;
    a.want_hess = want_hess ? 1 : 0;
    a.hscale = (h->s.time_stepping == 1 && dt != 0.0) ? 0.5 : 1.0;
    a.inertia_coef = inertia_coef(h, dt);
    if (h->asm_variant == 0 || h->asm_variant == 2) {
        a.ch = h->chunks;
        a.hex_tile = h->hex_tile;
        a.hex_gtile = h->hex_gtile;
        a.hex_blk_row = h->hex_blk_row;
    }
    if (h->asm_variant == 2) {
        a.ch.gen = h->chunk_gen;
        a.ch.gradg = h->chunk_gradg;
    }
    return a;
}

template <typename HT>
int eval_system(SorsHandle* h, double dt, bool want_hess, AsmMode mode = kAsmStep) {
    int st = compute_external(h);
    if (st) return st;
    (want_hess ? h->n_hess_evals : h->n_grad_evals)++;
    const int project = h->force_project >= 0 ? h->force_project
                        : (h->s.project_spd == 2 ? (h->proj_fallback ? 1 : 0) : h->s.project_spd);
    AsmArgs<HT> a = asm_args<HT>(h, dt, want_hess, mode, project);
    launch_assemble<HT>(a, h->max_pairs, h->stream);
    if (want_hess && h->has_pressure && method(h) == 0)
        launch_pressure_jac<HT>(pressure_args(h), h->row_ptr, h->col, h->node_mask, a.hscale * pressure_jac_scale(h),
                                (HT*)h->H, h->nnzb, h->stream);
    launch_finalize_grad(h->N, h->g_int, h->f_ext, h->q, h->qPrev, h->vPrev, h->gPrev, h->gPrevTmp, h->mass,
                         h->node_mask, h->mval, dt, h->s.time_stepping, h->s.damping_alpha, h->s.grav,
                         a.neumann_override, (h->has_vforce || h->has_pressure) ? 1 : 0, h->g, h->partials, h->sc,
                         h->stream);
    CK(cudaGetLastError());
    return SORS_OK;
}

int eval_energy(SorsHandle* h, double dt, double* out) {
    int st = compute_external(h);
    if (st) return st;
    launch_elem_energy(h->E, h->nv, h->X, h->q, h->conn, h->mat, muscles(h), h->s.material, h->partials, h->sc, h->stream);
    launch_dof_energy(h->N, h->q, h->qPrev, h->vPrev, h->mass, h->f_ext, (h->has_vforce || h->has_pressure) ? 1 : 0,
                      dt, h->s.time_stepping, h->s.damping_alpha, h->s.grav, h->partials, h->sc, h->stream);
    CK(cudaMemcpyAsync(h->sc_host, h->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    *out = h->sc_host->e_elem + h->sc_host->e_dof;
    return SORS_OK;
}

template <typename VT>
MinresBufs<VT> minres_bufs(SorsHandle* h) {
    MinresBufs<VT> b;
    b.Z[1] = (VT*)h->p0;
    b.Z[0] = (VT*)h->p1;
    b.V[1] = (VT*)h->r;
    b.V[0] = (VT*)h->z;
    b.W[0] = (VT*)h->mr_w[0];
    b.W[1] = (VT*)h->mr_w[1];
    b.x = (VT*)h->x;
    b.q = (VT*)h->qv;
    b.Minv = (const VT*)h->Minv;
    return b;
}

template <typename HT, typename VT>
void pcg_iter_pair(SorsHandle* h) {
    VT* z = (VT*)h->z;
    if (h->mr_active) {
        // two MINRES iterations, j odd then j even (a chunk starts at an odd j)
        const MinresBufs<VT> b = minres_bufs<VT>(h);
        for (int par = 1; par >= 0; par--) {
            launch_minres_spmv<HT, VT>(h->N, h->max_row_blocks, h->row_ptr, h->col, (const HT*)h->H, h->nnzb, b, par,
                                       h->partials, h->sc, h->stream);
            if (h->tl_active) {
                launch_minres_lanczos_restrict<VT>(h->cargs, b, par, h->tl_yc, h->sc, h->stream);
                launch_minres_coarse_z<VT>(h->cargs, h->tl_ld, (const VT*)h->tl_Ainv, h->tl_yc, b, par ^ 1, 0, 0.0,
                                           0.0, 0, h->partials, h->sc, h->stream);
            } else {
                launch_minres_lanczos<VT>(h->N, b, par, h->partials, h->sc, h->stream);
            }
        }
        return;
    }
    if (h->batch.nmem > 1) {
        for (int half = 0; half < 2; half++) {
            VT* pin = (VT*)(half ? h->p1 : h->p0);
            VT* pout = (VT*)(half ? h->p0 : h->p1);
            launch_bpcg_iter<HT, VT>(h->batch, h->row_ptr, h->col, (const HT*)h->H, (const VT*)h->Minv, z, pin, pout,
                                     (VT*)h->qv, (VT*)h->x, (VT*)h->r, z, h->proj_flag, h->proj_n, h->stream);
        }
        return;
    }
    if (h->tl_active) {
        for (int half = 0; half < 2; half++) {
            VT* pin = (VT*)(half ? h->p1 : h->p0);
            VT* pout = (VT*)(half ? h->p0 : h->p1);
            launch_form_p<VT>(h->N, z, pin, pout, h->sc, h->stream);
            launch_pcg_spmv<HT, VT>(h->N, h->max_row_blocks, h->row_ptr, h->col, (const HT*)h->H, h->nnzb, pout,
                                    (VT*)h->qv, h->partials, h->sc, h->stream);
            if (h->cruns.nruns > 0)
                launch_tl_update_restrict_runs<VT>(h->cargs, h->cruns, pout, (VT*)h->qv, (VT*)h->x, (VT*)h->r,
                                                   h->proj_flag, h->proj_n, h->tl_yc, h->sc, h->stream);
            else
                launch_tl_update_restrict<VT>(h->cargs, pout, (VT*)h->qv, (VT*)h->x, (VT*)h->r, h->proj_flag,
                                              h->proj_n, h->tl_yc, h->sc, h->stream);
            launch_tl_coarse_z<VT>(h->cargs, h->tl_ld, (const VT*)h->tl_Ainv, h->tl_yc, (VT*)h->r,
                                   (const VT*)h->Minv, z, 0, h->proj_flag, h->proj_n, h->partials, h->sc, h->stream);
        }
        return;
    }
    launch_form_p<VT>(h->N, z, (VT*)h->p0, (VT*)h->p1, h->sc, h->stream);
    launch_pcg_spmv<HT, VT>(h->N, h->max_row_blocks, h->row_ptr, h->col, (const HT*)h->H, h->nnzb, (VT*)h->p1,
                            (VT*)h->qv, h->partials, h->sc, h->stream);
    launch_pcg_update<VT>(h->N, (VT*)h->p1, (VT*)h->qv, (VT*)h->Minv, (VT*)h->x, (VT*)h->r, z, h->proj_flag,
                          h->proj_n, h->partials, h->sc, h->stream);
    launch_form_p<VT>(h->N, z, (VT*)h->p1, (VT*)h->p0, h->sc, h->stream);
    launch_pcg_spmv<HT, VT>(h->N, h->max_row_blocks, h->row_ptr, h->col, (const HT*)h->H, h->nnzb, (VT*)h->p0,
                            (VT*)h->qv, h->partials, h->sc, h->stream);
    launch_pcg_update<VT>(h->N, (VT*)h->p0, (VT*)h->qv, (VT*)h->Minv, (VT*)h->x, (VT*)h->r, z, h->proj_flag,
                          h->proj_n, h->partials, h->sc, h->stream);
}

template <typename HT, typename VT>
int pcg_chunk(SorsHandle* h) {
    const int mode = (h->proj_flag ? 1 : 0) + (h->tl_active ? 2 : 0) + (h->batch.nmem > 1 ? 4 : 0) +
                     (h->mr_active ? 8 : 0);
    if (h->pcg_exec && h->pcg_exec_mode != mode) {
        // the captured launches carry the projection pointers: capture again
        cudaGraphExecDestroy(h->pcg_exec);
        h->pcg_exec = nullptr;
    }
    if (!h->pcg_exec && !h->graph_failed) {
        h->pcg_exec_mode = mode;
        cudaGraph_t graph = nullptr;
        const long long launches_before = g_kernel_launches.load();
        cudaError_t e = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            for (int k = 0; k < kPcgChunk / 2; k++) pcg_iter_pair<HT, VT>(h);
            e = cudaStreamEndCapture(h->stream, &graph);
        }
        h->pcg_graph_kernels = g_kernel_launches.load() - launches_before;
        g_kernel_launches.store(launches_before);  // captured launches run when the graph runs
        if (e == cudaSuccess) e = cudaGraphInstantiate(&h->pcg_exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            h->graph_failed = true;
            h->pcg_exec = nullptr;
            cudaGetLastError();
        }
    }
    if (h->pcg_exec) {
        CK(cudaGraphLaunch(h->pcg_exec, h->stream));
        g_kernel_launches.fetch_add(h->pcg_graph_kernels);
    } else {
        for (int k = 0; k < kPcgChunk / 2; k++) pcg_iter_pair<HT, VT>(h);
        CK(cudaGetLastError());
    }
    return SORS_OK;
}

// Records the curvature of the PCG direction that broke down: iteration `it`
// multiplied p1 (it even) or p0 (it odd), padded to 4 values per node, and no
// kernel wrote either after the breakdown.
template <typename VT>
int record_curvature(SorsHandle* h) {
    const int it = h->sc_host->it;
    const VT* pb = (const VT*)((it & 1) ? h->p0 : h->p1);
    std::vector<VT> p((size_t)4 * h->N);
    CK(cudaMemcpyAsync(p.data(), pb, sizeof(VT) * p.size(), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    double pp = 0.0;
    for (int i = 0; i < h->N; i++)
        for (int k = 0; k < 3; k++) pp += (double)p[4 * (size_t)i + k] * (double)p[4 * (size_t)i + k];
    h->step_indefinite++;
    if (pp > 0.0) h->step_min_rq = std::min(h->step_min_rq, h->sc_host->pq / pp);
    return SORS_OK;
}

// Solves H dx = -g (dx in h->x), g = h->g unless given.  With h->proj_flag set
// the solve runs on the subspace the constraint projection leaves free.
// Returns PCG iterations in *iters.
// Member-segmented solve (sors_set_members): one PCG per member in the same
// launches.  Tolerances per member: eta relative to its own residual, or the
// absolute target of the call, or (a re-solve: eta 0, absolute target set)
// eta^2 ||b_k||^2 remembered from its last relative solve.  Summaries for the
// callers: the most iterations of any member, breakdown if any member broke
// down, squared norms summed over members.
template <typename HT, typename VT>
int pcg_solve_members(SorsHandle* h, double eta, double abs_tol, int* iters, const double* g) {
    const int tol_mode = (eta > 0.0 && abs_tol == 0.0) ? 1 : ((eta == 0.0 && abs_tol > 0.0) ? 2 : 0);
    launch_bpcg_init<VT>(h->batch, g ? g : h->g, (const VT*)h->Minv, (VT*)h->x, (VT*)h->r, (VT*)h->z, (VT*)h->p0,
                         eta * eta, abs_tol * abs_tol, tol_mode, h->s.pcg_max_iter, h->proj_flag, h->proj_n,
                         h->stream);
    CK(cudaGetLastError());
    const int nm = h->batch.nmem;
    const int maxchunks = (h->s.pcg_max_iter + kPcgChunk - 1) / kPcgChunk + 1;
    for (int c = 0; c < maxchunks; c++) {
        CK(cudaMemcpyAsync(h->ms_h.data(), h->batch.ms, sizeof(MemberScalars) * nm, cudaMemcpyDeviceToHost,
                           h->stream));
        CK(cudaStreamSynchronize(h->stream));
        bool all = true;
        for (int k = 0; k < nm && all; k++) all = h->ms_h[k].done != 0;
        if (all) break;
        int st = pcg_chunk<HT, VT>(h);
        if (st) return st;
    }
    CK(cudaMemcpyAsync(h->ms_h.data(), h->batch.ms, sizeof(MemberScalars) * nm, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    DevScalars& sh = *h->sc_host;
    sh.it = 0; sh.breakdown = 0; sh.done = 1; sh.bnorm2 = 0.0; sh.rr = 0.0; sh.rz = 0.0;
    bool first_iteration_breakdown = false;
    for (int k = 0; k < nm; k++) {
        const MemberScalars& m = h->ms_h[k];
        sh.it = std::max(sh.it, m.it);
        sh.bnorm2 += m.bnorm2;
        sh.rr += m.rr;
        if (!m.breakdown) continue;
        sh.breakdown = 1;
        first_iteration_breakdown |= m.it == 0;
        // this member's breaking direction: its nodes of p1 (it even) or p0 (it odd)
        const int n0 = h->mem_node0_h[k], n1 = h->mem_node0_h[k + 1];
        const VT* pb = (const VT*)((m.it & 1) ? h->p0 : h->p1) + 4 * (size_t)n0;
        std::vector<VT> pv((size_t)4 * (n1 - n0));
        CK(cudaMemcpyAsync(pv.data(), pb, sizeof(VT) * pv.size(), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        double pp = 0.0;
        for (size_t i = 0; i < pv.size(); i++)
            if ((i & 3) != 3) pp += (double)pv[i] * (double)pv[i];
        h->step_indefinite++;
        if (pp > 0.0) h->step_min_rq = std::min(h->step_min_rq, m.pq / pp);
    }
    *iters = sh.it;
    if (first_iteration_breakdown && !(h->s.project_spd == 2 && !h->proj_fallback))
        return fail(SORS_ERR_PCG_BREAKDOWN, "PCG breakdown: the Hessian is not positive definite");
    return SORS_OK;
}

// Keeps the coarse inverse in L2 between PCG iterations: an access-policy
// window on the handle's stream (captured into the PCG graphs) marks it
// persisting, within the context's persisting-L2 limit (a per-process
// setting that ends with the process).  The SpMV streams several times the
// L2 through between two coarse solves and would evict it otherwise.
void keep_coarse_in_l2(SorsHandle* h, size_t bytes) {
    if (h->l2_window_bytes == bytes) return;
    int dev = 0, maxp = 0, maxw = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&maxp, cudaDevAttrMaxPersistingL2CacheSize, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&maxw, cudaDevAttrMaxAccessPolicyWindowSize, dev) != cudaSuccess || maxp <= 0 ||
        maxw <= 0) {
        cudaGetLastError();
        return;
    }
    size_t limit = 0;
    cudaDeviceGetLimit(&limit, cudaLimitPersistingL2CacheSize);
    const size_t want = std::min((size_t)maxp, bytes);
    if (limit < want && cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    cudaStreamAttrValue v = {};
    v.accessPolicyWindow.base_ptr = h->tl_Ainv;
    v.accessPolicyWindow.num_bytes = std::min((size_t)maxw, bytes);
    v.accessPolicyWindow.hitRatio = (float)std::min(1.0, (double)std::max(limit, want) / (double)v.accessPolicyWindow.num_bytes);
    v.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    v.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    if (cudaStreamSetAttribute(h->stream, cudaStreamAttributeAccessPolicyWindow, &v) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    h->l2_window_bytes = bytes;
    // graphs captured before carry no window: capture again
    if (h->pcg_exec) {
        cudaGraphExecDestroy(h->pcg_exec);
        h->pcg_exec = nullptr;
    }
}

// The coarse operator P^T H P of the Hessian in h->H, inverted in place.
template <typename HT, typename VT>
int build_coarse(SorsHandle* h) {
    const int nc = h->cargs.nc;
    CK(cudaMemsetAsync(h->tl_Ac, 0, sizeof(double) * (size_t)nc * nc, h->stream));
    if (sizeof(HT) == 4)
        launch_coarse_galerkin_f(h->tl_npairs, h->tl_pair_ptr, h->tl_items, h->tl_ab, h->col, (const float*)h->H,
                                 h->nnzb, h->cargs, h->tl_Ac, h->stream);
    else
        launch_coarse_galerkin_d(h->tl_npairs, h->tl_pair_ptr, h->tl_items, h->tl_ab, h->col, (const double*)h->H,
                                 h->nnzb, h->cargs, h->tl_Ac, h->stream);
    launch_coarse_invert(nc, h->tl_Ac, h->tl_rowk, h->tl_colk, h->stream);
    launch_to_vt_pad<VT>(nc, h->tl_ld, h->tl_Ac, (VT*)h->tl_Ainv, h->stream);
    keep_coarse_in_l2(h, (size_t)nc * h->tl_ld * sizeof(VT));
    h->tl_ready = true;
    h->tl_refreshes++;
    return SORS_OK;
}

// Rebuilds the coarse operator when the iterations per decade of residual
// reduction of a solve of two decades or more doubled against the first such
// solve after the last rebuild.
void coarse_rate_check(SorsHandle* h, bool refreshed) {
    if (refreshed) h->tl_ref_rate = -1.0;
    const DevScalars& sh = *h->sc_host;
    if (h->tl_active && sh.it >= 8 && sh.rr > 0.0 && sh.bnorm2 >= 1e4 * sh.rr) {
        const double rate = sh.it / (0.5 * log10(sh.bnorm2 / sh.rr));
        if (h->tl_ref_rate <= 0.0) h->tl_ref_rate = rate;
        else if (rate > 2.0 * h->tl_ref_rate) h->tl_ready = false;
    }
}

template <typename HT, typename VT>
int pcg_solve(SorsHandle* h, double eta, double abs_tol, int* iters, const double* g = nullptr) {
    launch_block_jacobi<HT, VT>(h->N, h->row_ptr, h->diag_slot, (const HT*)h->H, h->nnzb, (VT*)h->Minv, h->stream);
    if (h->batch.nmem > 1) return pcg_solve_members<HT, VT>(h, eta, abs_tol, iters, g);
    // the two-level preconditioner: with a constraint projection (SQP, adjoint)
    // the correction is projected too, so the preconditioner stays SPD on the
    // free subspace (the coarse matrix itself is built without the projection)
    h->tl_active = h->s.two_level && h->cargs.nc > 0 && h->batch.nmem <= 1;
    bool refreshed = false;
    if (h->tl_active && !h->tl_ready) {
        int st = build_coarse<HT, VT>(h);
        if (st) return st;
        h->tl_proj = false;
        refreshed = true;
    }
    launch_pcg_init<HT, VT>(h->N, g ? g : h->g, (const VT*)h->Minv, (VT*)h->x, (VT*)h->r, (VT*)h->z, (VT*)h->p0,
                            eta * eta, abs_tol * abs_tol, h->s.pcg_max_iter, h->proj_flag, h->proj_n, h->partials,
                            h->sc, h->stream);
    if (h->tl_active) {
        launch_coarse_restrict<VT>(h->cargs, (VT*)h->r, h->tl_yc, h->stream);
        launch_tl_coarse_z<VT>(h->cargs, h->tl_ld, (const VT*)h->tl_Ainv, h->tl_yc, (VT*)h->r, (const VT*)h->Minv,
                               (VT*)h->z, 1, h->proj_flag, h->proj_n, h->partials, h->sc, h->stream);
    }
    CK(cudaGetLastError());
    int maxchunks = (h->s.pcg_max_iter + kPcgChunk - 1) / kPcgChunk + 1;
    for (int c = 0; c < maxchunks; c++) {
        int st = pcg_chunk<HT, VT>(h);
        if (st) return st;
        CK(cudaMemcpyAsync(h->sc_host, h->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        if (h->sc_host->done) break;
    }
    *iters = h->sc_host->it;
    if (h->sc_host->breakdown) {
        int st = record_curvature<VT>(h);
        if (st) return st;
    }
    // loose solves converge faster per decade and are not counted
    coarse_rate_check(h, refreshed);
    if (h->sc_host->breakdown && h->sc_host->it == 0 && !(h->s.project_spd == 2 && !h->proj_fallback))
        return fail(SORS_ERR_PCG_BREAKDOWN, "PCG breakdown: the Hessian is not positive definite");
    return SORS_OK;
}

// Solves H dx = -g (dx in h->x) by preconditioned MINRES: the Newton step of
// a symmetric indefinite Hessian, which the reference takes with LDL^T
// (cpp/src/solver.cpp:65-84).  Preconditioner: block Jacobi on |D_ii| and,
// with the two-level setting, the coarse correction of the SPD-projected
// Hessian (assembled at the current state when the coarse operator is
// rebuilt; the exact Hessian is then assembled again).  Tolerances as
// pcg_solve's, on the preconditioned residual norm.
// MINRES forcing cap: inexact Newton steps of an indefinite system stall at
// loose forcing (a bar compressed 10 %: 15 Newton iterations at 3e-2, 10 at
// 1e-2, 7 at 1e-3, 6 exact).
constexpr double kMinresEtaMax = 1e-3;

template <typename HT, typename VT>
int minres_solve(SorsHandle* h, double dt, double eta, double abs_tol, int* iters) {
    eta = std::min(eta, kMinresEtaMax);
    for (int k = 0; k < 2; k++)
        if (!h->mr_w[k]) {
            int st = dalloc(h, &h->mr_w[k], sizeof(VT) * 3 * (size_t)h->N);
            if (st) return st;
        }
    h->tl_active = h->s.two_level && h->cargs.nc > 0;
    bool refreshed = false;
    if (h->tl_active && (!h->tl_ready || !h->tl_proj)) {
        // the preconditioner must be SPD: the coarse operator of the projected Hessian
        int st;
        h->force_project = 1;
        st = eval_system<HT>(h, dt, true);
        h->force_project = -1;
        if (st) return st;
        if ((st = build_coarse<HT, VT>(h))) return st;
        h->tl_proj = true;
        if ((st = eval_system<HT>(h, dt, true))) return st;
        refreshed = true;
    }
    launch_block_jacobi_abs<HT, VT>(h->N, h->diag_slot, (const HT*)h->H, h->nnzb, (VT*)h->Minv, h->stream);
    const MinresBufs<VT> b = minres_bufs<VT>(h);
    const double eta2 = eta * eta, abs2 = abs_tol * abs_tol;
    launch_minres_init<VT>(h->N, h->g, b, !h->tl_active, eta2, abs2, h->s.pcg_max_iter, h->partials, h->sc,
                           h->stream);
    if (h->tl_active) {
        launch_coarse_restrict<VT>(h->cargs, b.V[1], h->tl_yc, h->stream);
        launch_minres_coarse_z<VT>(h->cargs, h->tl_ld, (const VT*)h->tl_Ainv, h->tl_yc, b, 1, 1, eta2, abs2,
                                   h->s.pcg_max_iter, h->partials, h->sc, h->stream);
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h->sc_host, h->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->mr_active = true;
    const int maxchunks = (h->s.pcg_max_iter + kPcgChunk - 1) / kPcgChunk + 1;
    for (int c = 0; c < maxchunks && !h->sc_host->done; c++) {
        int st = pcg_chunk<HT, VT>(h);
        if (st) { h->mr_active = false; return st; }
        CK(cudaMemcpyAsync(h->sc_host, h->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    h->mr_active = false;
    const int J = h->sc_host->it;
    if (h->sc_host->mr_pending) launch_minres_finish<VT>(h->N, b, (J + 1) & 1, h->sc, h->stream);
    CK(cudaGetLastError());
    *iters = J;
    if (verbose()) {
        // true residual ||H x + g|| of the returned solution (host copies)
        const size_t n = 3 * (size_t)h->N;
        std::vector<VT> xv(n);
        std::vector<HT> Hv(9 * (size_t)h->nnzb);
        std::vector<int> rp(h->N + 1), cl(h->nnzb);
        std::vector<double> gv(n);
        CK(cudaMemcpyAsync(xv.data(), h->x, sizeof(VT) * n, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaMemcpyAsync(Hv.data(), h->H, sizeof(HT) * Hv.size(), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaMemcpyAsync(rp.data(), h->row_ptr, sizeof(int) * rp.size(), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaMemcpyAsync(cl.data(), h->col, sizeof(int) * cl.size(), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaMemcpyAsync(gv.data(), h->g, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        double rr = 0.0, gg = 0.0, xx = 0.0;
        for (int i = 0; i < h->N; i++)
            for (int r = 0; r < 3; r++) {
                double acc = gv[3 * (size_t)i + r];
                for (int k = rp[i]; k < rp[i + 1]; k++)
                    for (int c = 0; c < 3; c++) {
                        // the lower triangle defines the operator
                        const int j = cl[k];
                        double a = (double)Hv[9 * (size_t)k + r * 3 + c];
                        if (j == i && c > r) a = (double)Hv[9 * (size_t)k + c * 3 + r];
                        acc += a * (double)xv[3 * (size_t)j + c];
                    }
                rr += acc * acc;
                gg += gv[3 * (size_t)i + r] * gv[3 * (size_t)i + r];
                xx += (double)xv[3 * (size_t)i + r] * (double)xv[3 * (size_t)i + r];
            }
        fprintf(stderr, "[sors] minres it=%d eta=%.2e |eta_M|/|b_M|=%.2e ||Hx+g||/||g||=%.2e |x|=%.3e bad=%d brk=%d\n",
                J, eta, sqrt(h->sc_host->rr / (h->sc_host->bnorm2 > 0 ? h->sc_host->bnorm2 : 1.0)),
                sqrt(rr / (gg > 0 ? gg : 1.0)), sqrt(xx), h->sc_host->mr_bad, h->sc_host->breakdown);
    }
    if (h->sc_host->mr_bad)
        return fail(SORS_ERR_PCG_BREAKDOWN, "MINRES breakdown: the preconditioner is not positive definite");
    coarse_rate_check(h, refreshed);
    return SORS_OK;
}

// The Newton system's solver of the settings: MINRES (linear_solver 1) for a
// plain Newton solve on one mesh, PCG otherwise.
template <typename HT, typename VT>
int newton_solve(SorsHandle* h, double dt, double eta, double abs_tol, int* iters) {
    if (h->s.linear_solver == 1 && h->batch.nmem <= 1 && !h->proj_flag)
        return minres_solve<HT, VT>(h, dt, eta, abs_tol, iters);
    return pcg_solve<HT, VT>(h, eta, abs_tol, iters);
}

int ensure_sqp_buffers(SorsHandle* h, int m);
template <typename HT, typename VT>
int adjoint_pairs(SorsHandle* h, double eta, std::vector<double>& lam, std::vector<double>& extra, int* iters);

// Adjoint of one backward-Euler step (see sors_adjoint_step).  At the step's
// solution q the residual g = grad Psi(q) - f + m (v - v_n)/dt - m grav +
// alpha m v (v = (q - q_n)/dt) vanishes on the subspace the held constraints
// leave free, and the held constraints fix the rest: Neumann DOFs at
// q_n + dt val (energy.cpp:296-306, neumannBC.cpp:4-21) and contact nodes on
// their plane or disk (n . (q_v - p) = 0).  With Z a basis of that subspace,
// lam = Z (Z^T H Z)^-1 Z^T b is a projected solve with the exact Hessian, and
//   dL/dtheta = -lam^T dg/dtheta  for the material, activations and old state,
//   r = b - H lam                 carries dL through the fixed DOFs' targets.
constexpr int kAdjointPressureIters = 200;

template <typename HT, typename VT>
int adjoint_impl(SorsHandle* h, const double* q_next, double dt, const double* b, const int* held_nodes,
                 const double* held_normals, int n_held, double* dq, double* dv, double* dE, double* dact,
                 double* dneu, SorsStepStats* stats, const double* bg_in = nullptr, double* bg_out = nullptr) {
    const int n = h->ndof, N = h->N, E = h->E;
    int st;
    if (!h->adj_l) {
        if ((st = dalloc_t(h, &h->adj_l, (size_t)n))) return st;
        if ((st = dalloc_t(h, &h->adj_y, (size_t)n))) return st;
        if ((st = dalloc_t(h, &h->adj_e, (size_t)2 * std::max(1, E)))) return st;
        if ((st = dalloc_t(h, &h->adj_q, (size_t)n))) return st;
    }
    h->adj_ready = false;
    if ((st = ensure_sqp_buffers(h, 0))) return st;
    CK(h2d(h, h->q, q_next, sizeof(double) * n));
    CK(cudaMemsetAsync(h->status, 0, sizeof(int), h->stream));
    // the exact Hessian: no SPD projection, every element term on every DOF
    struct ProjectionOff {
        SorsHandle* h;
        int saved;
        explicit ProjectionOff(SorsHandle* hh) : h(hh), saved(hh->s.project_spd) { h->s.project_spd = 0; }
        ~ProjectionOff() { h->s.project_spd = saved; }
    } projection_off(h);
    if ((st = eval_system<HT>(h, dt, true, kAsmFull))) return st;
    auto fixed = [&](int i) { return h->has_neumann && ((h->mask_h[i / 3] >> (i % 3)) & 1u); };
    h->pflag_h.assign(N, 0);
    if (h->has_neumann)
        for (int v = 0; v < N; v++) h->pflag_h[v] = h->mask_h[v] & 7u;
    for (int c = 0; c < n_held; c++) {
        const int v = held_nodes[c];
        if (v < 0 || v >= N) return fail(SORS_ERR_ARG, "held contact node out of range");
        if (h->pflag_h[v]) continue;  // Neumann nodes carry no contact
        h->pflag_h[v] = 8u;
        h->pn_h[v] = make_double4(held_normals[3 * c], held_normals[3 * c + 1], held_normals[3 * c + 2], 0.0);
    }
    CK(h2d(h, h->pflag_d, h->pflag_h.data(), (size_t)N));
    CK(h2d(h, h->pn_d, h->pn_h.data(), sizeof(double4) * N));
    std::vector<double> lam(n), rhs(b, b + n);
    const double eta = mixed(h) ? 1e-6 : std::max(1e-12, 0.01 * h->s.pcg_rel_tol);
    // Crank-Nicolson: the next step's residual holds 0.5 gi(q_next), gi the
    // internal force (gPrev), so its cotangent bg_in adds K^T bg_in to the
    // right-hand side; K = 2 (H - c M) with H the step's matrix (inertia c M
    // plus 0.5 K), evaluated by the SpMV of H.
    const bool cn = h->s.time_stepping == 1 && dt != 0.0;
    const double c_in = inertia_coef(h, dt);
    std::vector<double> bg;
    if (cn && bg_in) bg.assign(bg_in, bg_in + n);
    if (!bg.empty()) {
        CK(h2d(h, h->qp_dx, bg.data(), sizeof(double) * n));
        launch_spmv_plain<HT>(N, h->row_ptr, h->col, (const HT*)h->H, h->nnzb, h->qp_dx, h->adj_y, h->stream);
        std::vector<double> hb(n);
        CK(d2h(h, hb.data(), h->adj_y, sizeof(double) * n));
        for (int i = 0; i < n; i++) rhs[i] += 2.0 * (hb[i] - c_in * h->mass_h[i / 3] * bg[i]);
    }
    const std::vector<double> rhs0 = rhs;
    // lam = H^-1 rhs on the free subspace (H symmetric)
    auto solve = [&](const std::vector<double>& r) -> int {
        std::vector<double> g(n);
        for (int i = 0; i < n; i++) g[i] = -r[i];  // pcg_solve solves H x = -g
        CK(h2d(h, h->qp_g2, g.data(), sizeof(double) * n));
        int pit = 0;
        h->proj_flag = h->pflag_d;
        h->proj_n = h->pn_d;
        int s2 = pcg_solve<HT, VT>(h, eta, 0.0, &pit, h->qp_g2);
        h->proj_flag = nullptr;
        h->proj_n = nullptr;
        if (s2) return s2;
        if (h->sc_host->status & kFlagInverted) return fail(SORS_ERR_INVERTED, "Inverted Elements");
        if (stats) { stats->pcg_iters += pit; stats->residual_norm = sqrt(h->sc_host->rr); }
        if (sizeof(VT) == sizeof(double)) {
            CK(d2h(h, lam.data(), h->x, sizeof(double) * n));
        } else {
            std::vector<float> lf(n);
            CK(d2h(h, lf.data(), h->x, sizeof(float) * n));
            for (int i = 0; i < n; i++) lam[i] = lf[i];
        }
        CK(h2d(h, h->adj_l, lam.data(), sizeof(double) * n));
        return SORS_OK;
    };
    if ((st = solve(rhs))) return st;
    // Follower load: the residual's exact Jacobian K + T is not symmetric and
    // the Newton matrix holds K + S instead (k_pressure_adj_corr).  The
    // transpose system (K + T)^T lam = b is solved by the fixed point
    // lam <- H^-1 (b - (T^T - S) lam), which contracts when the load term is
    // small against stiffness and inertia.
    std::vector<double> corr;  // (T^T - S) lam at the final lam
    if (h->has_pressure) {
        const double tol = mixed(h) ? 1e-6 : 1e-11;
        corr.assign(n, 0.0);
        bool conv = false;
        for (int k = 0; k < kAdjointPressureIters && !conv; k++) {
            CK(cudaMemsetAsync(h->adj_y, 0, sizeof(double) * n, h->stream));
            launch_pressure_adj_corr(pressure_args(h), h->node_mask, method(h) == 0 ? pressure_jac_scale(h) : 0.0, h->adj_l, h->adj_y,
                                     h->stream);
            CK(d2h(h, corr.data(), h->adj_y, sizeof(double) * n));
            const std::vector<double> prev = lam;
            for (int i = 0; i < n; i++) rhs[i] = rhs0[i] - corr[i];
            if ((st = solve(rhs))) return st;
            double dd = 0.0, ll = 0.0;
            for (int i = 0; i < n; i++) { dd += (lam[i] - prev[i]) * (lam[i] - prev[i]); ll += lam[i] * lam[i]; }
            conv = dd <= tol * tol * ll;
        }
        if (!conv) return fail(SORS_ERR_NOT_CONVERGED, "the pressure-load adjoint fixed point did not converge");
        CK(cudaMemsetAsync(h->adj_y, 0, sizeof(double) * n, h->stream));
        launch_pressure_adj_corr(pressure_args(h), h->node_mask, method(h) == 0 ? pressure_jac_scale(h) : 0.0, h->adj_l, h->adj_y,
                                 h->stream);
        CK(d2h(h, corr.data(), h->adj_y, sizeof(double) * n));
    }
    std::vector<double> extra;  // forces of the held pairs' columns (empty: none)
    if (!h->adj_pairs.empty()) {
        int pp = 0;
        if ((st = adjoint_pairs<HT, VT>(h, eta, lam, extra, &pp))) return st;
        if (stats) stats->pcg_iters += pp;
    }
    // element contractions with lam (zero on fixed DOFs and along held normals);
    // Crank-Nicolson: the step's 0.5 gi(q_next) and the next step's gPrev =
    // gi(q_next), i.e. with 0.5 lam - bg_in
    const double* lam_elem = h->adj_l;
    if (cn) {
        std::vector<double> le(n);
        for (int i = 0; i < n; i++) le[i] = 0.5 * lam[i] - (bg.empty() ? 0.0 : bg[i]);
        CK(h2d(h, h->qp_dx, le.data(), sizeof(double) * n));
        lam_elem = h->qp_dx;
    }
    launch_adjoint_elem(E, h->nv, h->X, h->q, h->conn, h->mat, muscles(h), h->s.material, lam_elem, h->adj_e,
                        h->stream);
    std::vector<double> ge((size_t)2 * std::max(1, E));
    CK(d2h(h, ge.data(), h->adj_e, sizeof(double) * 2 * (size_t)E));
    std::vector<double> r(n, 0.0);
    if (h->has_neumann) {
        launch_spmv_plain<HT>(N, h->row_ptr, h->col, (const HT*)h->H, h->nnzb, h->adj_l, h->adj_y, h->stream);
        CK(d2h(h, r.data(), h->adj_y, sizeof(double) * n));
        for (int i = 0; i < n; i++)
            r[i] = rhs0[i] - r[i] + (extra.empty() ? 0.0 : extra[i]) - (corr.empty() ? 0.0 : corr[i]);
    }
    const double a = h->s.damping_alpha;
    for (int i = 0; i < n; i++) {
        const double m = h->mass_h[i / 3];
        const bool f = fixed(i);
        // d g / d q_n = -c M; d g / d v_n = -M / dt (backward Euler), -(2 / dt + alpha) M (Crank-Nicolson)
        const double inert = dt != 0.0 ? lam[i] * m * c_in : 0.0;
        if (dq) dq[i] = f ? r[i] : inert;
        if (dv) dv[i] = dt != 0.0 ? lam[i] * m * (cn ? 2.0 / dt + a : 1.0 / dt) : 0.0;
        if (dneu) dneu[i] = f ? r[i] * dt : 0.0;
        // the step's residual holds 0.5 gPrev
        if (bg_out) bg_out[i] = cn ? -0.5 * lam[i] : 0.0;
    }
    CK(cudaMemcpyAsync(h->adj_q, h->q, sizeof(double) * n, cudaMemcpyDeviceToDevice, h->stream));
    h->adj_ready = true;
    if (dE)
        for (int e = 0; e < E; e++) dE[e] = h->youngs_h[e] != 0.0 ? -ge[e] / h->youngs_h[e] : 0.0;
    if (dact) {
        for (int g = 0; g < h->n_mgroups; g++) dact[g] = 0.0;
        if (!h->mgroup_h.empty())
            for (int e = 0; e < E; e++)
                if (h->mgroup_h[e] >= 0) dact[h->mgroup_h[e]] -= ge[(size_t)E + e];
    }
    return SORS_OK;
}

template <typename HT, typename VT>
int minimize(SorsHandle* h, double dt, SorsStepStats* stats) {
    const int n = h->ndof;
    const int m = method(h);
    const double dx_tol = h->s.newton_dx_tol;
    const double res_tol = h->s.newton_res_tol;
    bool converged = false;
    int st = SORS_OK;
    double prev_g = -1.0, prev_eta = 0.5;
    CK(cudaMemsetAsync(h->status, 0, sizeof(int), h->stream));
    bool have_hess = false;
    for (int it = 0; it < h->s.newton_max_iter; it++) {
        bool want_hess = (m != 2) || !have_hess;  // frozen Hessian: assemble once
        if (want_hess) h->proj_fallback = (m == 2);  // adaptive: the frozen Hessian is the projected one
        // Near convergence (the inexact-Newton bound eta |g| of the last solve
        // within 1e3 res_tol) the gradient is evaluated alone first: the
        // iteration may stop there, and if it does not but |g| fell tenfold,
        // the step reuses the Hessian of the last assembly (a chord step, whose
        // error is second order in the last update); otherwise the Hessian is
        // assembled as usual.
        const bool probe = want_hess && have_hess && m != 2 && res_tol > 0.0 && prev_g > 0.0 &&
                           prev_eta * prev_g <= 1e3 * res_tol;
        if ((st = eval_system<HT>(h, dt, want_hess && !probe))) return st;
        if (want_hess && !probe) have_hess = true;
        CK(cudaMemcpyAsync(h->sc_host, h->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        if (h->sc_host->status & kFlagInverted)
            return fail(SORS_ERR_INVERTED, "Inverted Elements");
        double gn = sqrt(h->sc_host->gnorm2);
        if (stats) { stats->newton_iters++; stats->residual_norm = gn; }
        if (!(gn == gn)) break;  // NaN gradient: diverged
        if (res_tol > 0.0 && gn < res_tol) { converged = true; break; }
        if (probe && gn > 0.1 * prev_g) {
            if ((st = eval_system<HT>(h, dt, true))) return st;
            CK(cudaMemcpyAsync(h->sc_host, h->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, h->stream));
            CK(cudaStreamSynchronize(h->stream));
        }
        // forcing term: Eisenstat-Walker choice 2 with its safeguard, never
        // solving below what the residual target needs, floored at pcg_rel_tol
        // (and at 1e-6 for FP32 PCG vectors)
        double eta = 0.5;
        if (prev_g > 0.0) {
            const double ratio = gn / prev_g;
            eta = 0.9 * ratio * ratio;
            const double safe = 0.9 * prev_eta * prev_eta;
            if (safe > 0.1) eta = std::max(eta, safe);
            eta = std::min(eta, 0.5);
        }
        if (res_tol > 0.0) eta = std::max(eta, std::min(0.5, 0.5 * res_tol / gn));
        eta = std::max(eta, mixed(h) ? std::max(h->s.pcg_rel_tol, 1e-6) : h->s.pcg_rel_tol);
        prev_g = gn;
        prev_eta = eta;
        int pit = 0;
        if ((st = newton_solve<HT, VT>(h, dt, eta, res_tol > 0.0 ? 0.1 * res_tol : 0.0, &pit))) return st;
        if (stats) stats->pcg_iters += pit;
        if (h->s.project_spd == 2 && !h->proj_fallback && h->sc_host->breakdown) {
            // negative curvature in the exact Hessian: solve this iteration with the projected one
            h->proj_fallback = true;
            if ((st = eval_system<HT>(h, dt, true))) return st;
            if ((st = pcg_solve<HT, VT>(h, eta, res_tol > 0.0 ? 0.1 * res_tol : 0.0, &pit))) return st;
            if (stats) stats->pcg_iters += pit;
        }
        double alpha = 1.0;
        if (m == 1) {
            // Armijo backtracking (solver.cpp:201-264): c = 0.1, beta = 0.5
            CK(cudaMemcpyAsync(h->q0, h->q, sizeof(double) * n, cudaMemcpyDeviceToDevice, h->stream));
            launch_dot_gdx<VT>(n, h->g, (const VT*)h->x, h->partials, h->sc, h->stream);
            double e0;
            if ((st = eval_energy(h, dt, &e0))) return st;
            double gdx = h->sc_host->gdx;
            bool accepted = false;
            for (int ls = 0; ls < 64; ls++) {
                launch_newton_update<VT>(n, (const VT*)h->x, alpha, h->q, h->q0, h->partials, h->sc, 6, h->stream);
                double e1;
                if ((st = eval_energy(h, dt, &e1))) return st;
                if (e1 <= e0 + 0.1 * alpha * gdx) { accepted = true; break; }
                alpha *= 0.5;
            }
            if (!accepted) return fail(SORS_ERR_LINESEARCH, "line search did not find a decrease");
        } else {
            CK(cudaMemcpyAsync(h->q0, h->q, sizeof(double) * n, cudaMemcpyDeviceToDevice, h->stream));
            launch_newton_update<VT>(n, (const VT*)h->x, 1.0, h->q, h->q0, h->partials, h->sc, 6, h->stream);
            if (m == 0 && h->s.project_spd == 2 && h->s.newton_safeguard) {
                // Residual safeguard for the exact-Hessian Newton step: where the
                // full step raises ||g|| (far from the solution, or where PCG
                // met an indefinite Hessian without seeing it), halve it until
                // ||g(q + a dx)|| <= (1 - 1e-4 a) ||g(q)||.  Full steps that
                // decrease the residual are taken as the reference takes them.
                for (int ls = 0; ls < 12; ls++) {
                    if ((st = eval_system<HT>(h, dt, false))) return st;
                    CK(cudaMemcpyAsync(h->sc_host, h->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, h->stream));
                    CK(cudaStreamSynchronize(h->stream));
                    const double gt = sqrt(h->sc_host->gnorm2);
                    if (gt == gt && gt <= (1.0 - 1e-4 * alpha) * gn) break;
                    alpha *= 0.5;
                    launch_newton_update<VT>(n, (const VT*)h->x, alpha, h->q, h->q0, h->partials, h->sc, 6,
                                             h->stream);
                }
            }
        }
        CK(cudaMemcpyAsync(h->sc_host, h->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        double dxn = sqrt(h->sc_host->dxnorm2) / alpha;
        if (stats) stats->dx_norm = dxn;
        if (verbose())
            fprintf(stderr, "[sors] newton %d |g|=%.3e eta=%.2e pcg=%d |r|/|b|=%.2e |dx|=%.3e\n", it, gn, eta, pit,
                    sqrt(h->sc_host->rr / (h->sc_host->bnorm2 > 0 ? h->sc_host->bnorm2 : 1.0)), dxn);
        if (!(dxn == dxn)) break;  // "Newton's method diverged"
        if (dxn < dx_tol) { converged = true; break; }
    }
    if (!converged && m != 2) return fail(SORS_ERR_NOT_CONVERGED, "Newton's method did not converge");
    return SORS_OK;
}

// ---------------------------------------------------------------------------
// Contact active sets (host), restating PlaneContact/DiskContact::
// update_active_constraints (cpp/src/constraints/planeContact.cpp:89-124,
// diskContact.cpp:94-205) with the thresholds of cpp/headers/common.h:29-35.
// ---------------------------------------------------------------------------
constexpr double kPlaneThreshold = 0.01;
constexpr double kDiskPlaneThreshold = 0.01;
constexpr double kDiskRadialThreshold = 0.001;

void update_plane_contacts(SorsHandle* h, const double* q) {
    h->plane_mask.assign(h->plane_surf.size(), -1);
    for (size_t i = 0; i < h->plane_surf.size(); i++) {
        const double* x = q + 3 * (size_t)h->plane_surf[i];
        double best = std::numeric_limits<double>::max();
        int idx = -1;
        for (size_t k = 0; k < h->planes.size(); k++) {
            const auto& P = h->planes[k];
            const double d = P.n[0] * (x[0] - P.p[0]) + P.n[1] * (x[1] - P.p[1]) + P.n[2] * (x[2] - P.p[2]);
            if (d < kPlaneThreshold && d < best) { best = d; idx = (int)k; }
        }
        h->plane_mask[i] = idx;
    }
}

double disk_plane_dist(const SorsHandle::Disk& D, const double* x) {
    return D.n[0] * (x[0] - D.c[0]) + D.n[1] * (x[1] - D.c[1]) + D.n[2] * (x[2] - D.c[2]);
}
double disk_radial_dist(const SorsHandle::Disk& D, const double* x) {
    double v[3] = {x[0] - D.c[0], x[1] - D.c[1], x[2] - D.c[2]};
    const double d = D.n[0] * v[0] + D.n[1] * v[1] + D.n[2] * v[2];
    for (int k = 0; k < 3; k++) v[k] -= d * D.n[k];
    return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
}

void update_disk_group(SorsHandle* h, SorsHandle::DiskGroup& G, const double* q) {
    const size_t ns = G.surf.size();
    if (G.mask.size() != ns) G.mask.assign(ns, -1);
    const double clear = 3.0 * kDiskPlaneThreshold, depth = 5.0 * kDiskPlaneThreshold;
    if (G.frozen) {
        // keep the captured footprint until every vertex of it is clearly above its disk
        bool all_clear = true;
        for (size_t i = 0; i < ns && all_clear; i++) {
            const int d = G.mask[i];
            if (d < 0) continue;
            if (disk_plane_dist(h->disks[d], q + 3 * (size_t)G.surf[i]) < clear) all_clear = false;
        }
        if (all_clear) {
            G.frozen = false;
            std::fill(G.mask.begin(), G.mask.end(), -1);
        }
        return;
    }
    std::vector<char> hit(G.disks.size(), 0);
    bool any = false;
    for (size_t i = 0; i < ns; i++) {
        const double* x = q + 3 * (size_t)G.surf[i];
        for (size_t k = 0; k < G.disks.size(); k++) {
            const auto& D = h->disks[G.disks[k]];
            if (disk_plane_dist(D, x) >= kDiskPlaneThreshold) continue;
            if (disk_radial_dist(D, x) > D.r + kDiskRadialThreshold) continue;
            hit[k] = 1;
            any = true;
        }
    }
    std::fill(G.mask.begin(), G.mask.end(), -1);
    if (!any) return;
    int active = 0;
    for (size_t k = 0; k < G.disks.size(); k++) {
        if (!hit[k]) continue;
        const int d = G.disks[k];
        const auto& D = h->disks[d];
        for (size_t i = 0; i < ns; i++) {
            const double* x = q + 3 * (size_t)G.surf[i];
            const double pd = disk_plane_dist(D, x);
            if (pd > kDiskPlaneThreshold || pd < -depth) continue;
            if (disk_radial_dist(D, x) > D.r + kDiskRadialThreshold) continue;
            int& slot = G.mask[i];
            if (slot == -1) { slot = d; active++; }
            else if (fabs(pd) < fabs(disk_plane_dist(h->disks[slot], x))) slot = d;
        }
    }
    if (active > 0) G.frozen = true;
}

void update_disk_contacts(SorsHandle* h, const double* q) {
    for (auto& G : h->disk_groups) update_disk_group(h, G, q);
}

// Two-level set-up: nodes binned into about N / 2000 (at most 256) boxes of
// the undeformed bounding box, empty boxes dropped; each aggregate's coarse
// unknowns are its 3 translations and 3 rotations about its centroid, the
// rotations scaled by 1 / (box size).  The Galerkin matrix P^T H P is summed
// per aggregate pair over a fixed list of Hessian blocks (deterministic).
// Two-level aggregates: a grid of about N / 1000 (at most 512) near-cubic
// boxes over the bounding box of the undeformed positions.  The locality
// order numbers the nodes box by box, so that each aggregate is a contiguous
// node range.
struct AggBins {
    double lo[3], L[3], hb;
    int dim[3];
    void cell(const double* x, int (&c)[3]) const {
        for (int k = 0; k < 3; k++) c[k] = std::max(0, std::min(dim[k] - 1, (int)((x[k] - lo[k]) / L[k] * dim[k])));
    }
};
AggBins agg_bins(int N, const double* X) {
    AggBins b;
    double hi[3] = {-1e300, -1e300, -1e300};
    for (int k = 0; k < 3; k++) b.lo[k] = 1e300;
    for (int i = 0; i < N; i++)
        for (int k = 0; k < 3; k++) {
            b.lo[k] = std::min(b.lo[k], X[3 * (size_t)i + k]);
            hi[k] = std::max(hi[k], X[3 * (size_t)i + k]);
        }
    const int target = std::max(1, std::min(512, N / 1000));
    double vol = 1.0;
    for (int k = 0; k < 3; k++) b.L[k] = std::max(hi[k] - b.lo[k], 1e-12);
    const double lmax = std::max(b.L[0], std::max(b.L[1], b.L[2]));
    for (int k = 0; k < 3; k++) vol *= std::max(b.L[k], 1e-3 * lmax);
    b.hb = cbrt(vol / target);
    for (int k = 0; k < 3; k++) b.dim[k] = std::max(1, (int)llround(b.L[k] / b.hb));
    return b;
}

int setup_two_level(SorsHandle* h, const double* X) {
    const int N = h->N;
    AggBins ab = agg_bins(N, X);
    const double hb = ab.hb;
    const int* dim = ab.dim;
    std::vector<int> bin(N), remap((size_t)dim[0] * dim[1] * dim[2], -1);
    for (int i = 0; i < N; i++) {
        int c[3];
        ab.cell(X + 3 * (size_t)i, c);
        bin[i] = c[0] + dim[0] * (c[1] + dim[1] * c[2]);
    }
    // aggregates numbered in the order of their lowest node
    int nagg = 0;
    for (int i = 0; i < N; i++)
        if (remap[bin[i]] < 0) remap[bin[i]] = nagg++;
    std::vector<int> aid(N), cnt(nagg + 1, 0);
    for (int i = 0; i < N; i++) { aid[i] = remap[bin[i]]; cnt[aid[i] + 1]++; }
    for (int a = 0; a < nagg; a++) cnt[a + 1] += cnt[a];
    std::vector<int> nodes(N), fillp(cnt.begin(), cnt.end() - 1);
    for (int i = 0; i < N; i++) nodes[fillp[aid[i]]++] = i;
    std::vector<double4> cen(nagg);
    for (int a = 0; a < nagg; a++) {
        double c[3] = {0, 0, 0};
        for (int k = cnt[a]; k < cnt[a + 1]; k++)
            for (int d = 0; d < 3; d++) c[d] += X[3 * nodes[k] + d];
        const double n = std::max(1, cnt[a + 1] - cnt[a]);
        cen[a] = make_double4(c[0] / n, c[1] / n, c[2] / n, 1.0 / hb);
    }
    std::vector<float4> off(N);
    for (int i = 0; i < N; i++) {
        const double4 c = cen[aid[i]];
        off[i] = make_float4((float)((X[3 * i] - c.x) * c.w), (float)((X[3 * i + 1] - c.y) * c.w),
                             (float)((X[3 * i + 2] - c.z) * c.w), 0.0f);
    }
    // aggregate pairs and their Hessian blocks (counting sort by pair key)
    const long long nkeys = (long long)nagg * nagg;
    std::vector<int> keycnt((size_t)nkeys + 1, 0);
    const int64_t nnzb = h->nnzb;
    for (int i = 0; i < N; i++)
        for (int b = h->row_ptr_h[i]; b < h->row_ptr_h[i + 1]; b++) keycnt[(size_t)aid[i] * nagg + aid[h->col_h[b]] + 1]++;
    std::vector<int> pair_ptr{0};
    std::vector<int2> pair_ab;
    std::vector<long long> keypos((size_t)nkeys, -1);
    long long acc = 0;
    for (long long k = 0; k < nkeys; k++) {
        if (keycnt[k + 1] == 0) continue;
        keypos[k] = acc;
        acc += keycnt[k + 1];
        pair_ab.push_back(make_int2((int)(k / nagg), (int)(k % nagg)));
        pair_ptr.push_back((int)acc);
    }
    std::vector<int2> items((size_t)nnzb);
    for (int i = 0; i < N; i++)
        for (int b = h->row_ptr_h[i]; b < h->row_ptr_h[i + 1]; b++) {
            const long long k = (long long)aid[i] * nagg + aid[h->col_h[b]];
            items[(size_t)keypos[k]++] = make_int2(b, i);
        }
    int st;
    h->tl_npairs = (int)pair_ab.size();
    const int nc = 6 * nagg;
    int* aid_d = nullptr; double4* cen_d = nullptr; int* aggptr_d = nullptr; int* nodes_d = nullptr;
    if ((st = upload(h, &aid_d, aid.data(), (size_t)N))) return st;
    if ((st = upload(h, &cen_d, cen.data(), (size_t)nagg))) return st;
    float4* off_d = nullptr;
    if ((st = upload(h, &off_d, off.data(), (size_t)N))) return st;
    if ((st = upload(h, &aggptr_d, cnt.data(), (size_t)nagg + 1))) return st;
    if ((st = upload(h, &nodes_d, nodes.data(), (size_t)N))) return st;
    if ((st = upload(h, &h->tl_pair_ptr, pair_ptr.data(), pair_ptr.size()))) return st;
    if ((st = upload(h, &h->tl_ab, pair_ab.data(), pair_ab.size()))) return st;
    if ((st = upload(h, &h->tl_items, items.data(), items.size()))) return st;
    if ((st = dalloc_t(h, &h->tl_Ac, (size_t)nc * nc))) return st;
    // Ainv rows padded to a multiple of 16 bytes (zero padding, and zero tail in yc)
    const int w16 = 16 / (int)hsize(h);
    h->tl_ld = (nc + w16 - 1) / w16 * w16;
    if ((st = dalloc_t(h, &h->tl_yc, (size_t)h->tl_ld))) return st;
    CK(dzero(h, h->tl_yc, sizeof(double) * (size_t)h->tl_ld));
    if ((st = dalloc_t(h, &h->tl_rowk, (size_t)nc))) return st;
    if ((st = dalloc_t(h, &h->tl_colk, (size_t)nc))) return st;
    if ((st = dalloc(h, &h->tl_Ainv, (size_t)nc * h->tl_ld * hsize(h)))) return st;
    // contiguous aggregates (aid non-decreasing in node order): the runs of the
    // node-parallel restriction
    bool contiguous = true;
    for (int i = 1; i < N && contiguous; i++) contiguous = aid[i] >= aid[i - 1];
    if (contiguous && N > 0) {
        constexpr int kB = 256;  // kRunThreads
        const int nblk = (N + kB - 1) / kB;
        std::vector<int> run_start, block_ptr(nblk + 1, 0), agg_begin(nagg + 1, 0);
        for (int b = 0; b < nblk; b++) {
            block_ptr[b] = (int)run_start.size();
            const int i1 = std::min(N, (b + 1) * kB);
            for (int i = b * kB; i < i1; i++)
                if (i == b * kB || aid[i] != aid[i - 1]) run_start.push_back(i);
        }
        block_ptr[nblk] = (int)run_start.size();
        const int nruns = (int)run_start.size();
        for (int k = nruns - 1; k >= 0; k--) agg_begin[aid[run_start[k]]] = k;
        agg_begin[nagg] = nruns;
        run_start.push_back(N);
        int *rs_d = nullptr, *bp_d = nullptr, *ab_d = nullptr;
        double* part_d = nullptr;
        if ((st = upload(h, &rs_d, run_start.data(), run_start.size()))) return st;
        if ((st = upload(h, &bp_d, block_ptr.data(), block_ptr.size()))) return st;
        if ((st = upload(h, &ab_d, agg_begin.data(), agg_begin.size()))) return st;
        if ((st = dalloc_t(h, &part_d, (size_t)6 * nruns))) return st;
        h->cruns.run_start = rs_d; h->cruns.block_run_ptr = bp_d; h->cruns.agg_run_begin = ab_d;
        h->cruns.partial = part_d; h->cruns.nruns = nruns;
    }
    h->cargs.N = N; h->cargs.nagg = nagg; h->cargs.nc = nc;
    h->cargs.aid = aid_d; h->cargs.agg_c = cen_d; h->cargs.agg_ptr = aggptr_d; h->cargs.agg_nodes = nodes_d;
    h->cargs.fixed = h->node_mask; h->cargs.off = off_d;
    h->tl_ready = false;
    return SORS_OK;
}

int ensure_sqp_buffers(SorsHandle* h, int m) {
    int st;
    const size_t n = (size_t)h->ndof;
    if (!h->qp_x0) {
        double** v[] = {&h->qp_x0, &h->qp_y, &h->qp_g2, &h->qp_dx};
        for (double** p : v)
            if ((st = dalloc_t(h, p, n))) return st;
        if ((st = dalloc_t(h, &h->pflag_d, (size_t)h->N))) return st;
        if ((st = dalloc_t(h, &h->pn_d, (size_t)h->N))) return st;
        h->pn_h.assign(h->N, make_double4(0, 0, 0, 0));
    }
    if (m > h->c_cap) {
        const int cap = std::max(m, 2 * h->c_cap);
        if ((st = dalloc_t(h, &h->cnode_d, (size_t)cap))) return st;
        if ((st = dalloc_t(h, &h->cnb_d, (size_t)cap))) return st;
        if ((st = dalloc_t(h, &h->cout_d, (size_t)2 * cap))) return st;
        if ((st = dalloc_t(h, &h->cpos_d, (size_t)3 * cap))) return st;
        h->c_cap = cap;
    }
    return SORS_OK;
}

// Rows of the maxDistance pairs at the linearisation point x (maxDistance.cpp:
// 4-80): g_k = d_k - |x_i - x_j| >= 0, gradient -u at i and +u at j with
// u = (x_i - x_j) / |x_i - x_j|, so the QP row is a_k . dx >= l_k = |x_i - x_j| - d_k.
struct PairRows {
    std::vector<double> u, l;  // 3 per pair, 1 per pair
};

PairRows pair_rows(const SorsHandle* h, const std::vector<double>& xp) {
    const int np = (int)h->md_d.size();
    PairRows r;
    r.u.assign(3 * (size_t)np, 0.0);
    r.l.assign(np, 0.0);
    for (int k = 0; k < np; k++) {
        double d[3], L2 = 0.0;
        for (int c = 0; c < 3; c++) { d[c] = xp[6 * (size_t)k + c] - xp[6 * (size_t)k + 3 + c]; L2 += d[c] * d[c]; }
        const double L = sqrt(L2);
        if (L > 0.0)  // Eigen's normalized() leaves a zero vector unchanged
            for (int c = 0; c < 3; c++) r.u[3 * (size_t)k + c] = d[c] / L;
        r.l[k] = L - h->md_d[k];
    }
    return r;
}

// a_k . v with v given at the pair nodes (6 values per pair: v_i, v_j)
double pair_dot(const PairRows& R, int k, const double* v) {
    const double* u = &R.u[3 * (size_t)k];
    return -(u[0] * v[0] + u[1] * v[1] + u[2] * v[2]) + (u[0] * v[3] + u[1] * v[4] + u[2] * v[5]);
}

int ensure_pair_buffers(SorsHandle* h, int np) {
    if (np <= h->md_cap) return SORS_OK;
    int st;
    if ((st = dalloc_t(h, &h->md_nodes_d, 2 * (size_t)np))) return st;
    if ((st = dalloc_t(h, &h->md_pos_d, 6 * (size_t)np))) return st;
    if ((st = dalloc_t(h, &h->md_ij_d, (size_t)np))) return st;
    if ((st = dalloc_t(h, &h->md_coef_d, (size_t)np))) return st;
    h->md_cap = np;
    return SORS_OK;
}

// Small dense solve (Gaussian elimination, partial pivoting); false if singular.
bool dense_solve(int m, std::vector<double> A, std::vector<double>& b) {
    for (int c = 0; c < m; c++) {
        int piv = c;
        for (int r = c + 1; r < m; r++)
            if (fabs(A[(size_t)r * m + c]) > fabs(A[(size_t)piv * m + c])) piv = r;
        if (!(fabs(A[(size_t)piv * m + c]) > 0.0)) return false;
        if (piv != c) {
            for (int k = 0; k < m; k++) std::swap(A[(size_t)c * m + k], A[(size_t)piv * m + k]);
            std::swap(b[c], b[piv]);
        }
        for (int r = c + 1; r < m; r++) {
            const double f = A[(size_t)r * m + c] / A[(size_t)c * m + c];
            for (int k = c; k < m; k++) A[(size_t)r * m + k] -= f * A[(size_t)c * m + k];
            b[r] -= f * b[c];
        }
    }
    for (int c = m - 1; c >= 0; c--) {
        double s = b[c];
        for (int k = c + 1; k < m; k++) s -= A[(size_t)c * m + k] * b[k];
        b[c] = s / A[(size_t)c * m + c];
    }
    return true;
}

// The held maxDistance pairs on top of the node-projected QP solution dx0 (in
// qp_dx).  With P the projection of the held nodes, w_k = (P H P)^+ P a_k (one
// projected PCG solve per held pair) and dx = dx0 + sum_k mu_k w_k satisfies
// P (H dx + g - sum_k mu_k a_k) = 0; the held rows a_j . dx = l_j give the
// small system S mu = l - A dx0, S_jk = a_j . w_k.  Violated pairs join the
// working set, held pairs with mu < 0 leave.  On return qp_dx holds dx and
// mu[k] the multiplier of pair k (0 when not held).  Returns -1 when a solve met
// negative curvature with the exact Hessian (the caller falls back to the
// projected one).
template <typename HT, typename VT>
int solve_pairs(SorsHandle* h, const PairRows& R, double eta, std::vector<double>& mu, int* pcg_iters) {
    const int np = (int)h->md_d.size(), n = h->ndof;
    mu.assign(np, 0.0);
    std::vector<double> D0(6 * (size_t)np), Wh;   // dx0 and the w_k at the pair nodes
    launch_gather_nodes(2 * np, h->md_nodes_d, h->qp_dx, h->md_pos_d, h->stream);
    CK(d2h(h, D0.data(), h->md_pos_d, sizeof(double) * 6 * np));
    std::vector<int> slot(np, -1);  // pool index of w_k
    int used = 0;
    double l_scale = 0.0;
    for (int k = 0; k < np; k++) l_scale = std::max(l_scale, fabs(R.l[k]));
    const double tol_s = 1e-12 + 1e-9 * l_scale;
    std::vector<int> wl;
    for (int round = 0; round < 25; round++) {
        wl.clear();
        for (int k = 0; k < np; k++)
            if (h->md_work[k]) wl.push_back(k);
        for (int k : wl) {
            if (slot[k] >= 0) continue;
            if (used == (int)h->md_w.size()) {
                double* w = nullptr;
                int st;
                if ((st = dalloc_t(h, &w, (size_t)n))) return st;
                h->md_w.push_back(w);
            }
            // g = -a_k: the PCG solves P H P x = -P g
            const double4 coef = make_double4(R.u[3 * (size_t)k], R.u[3 * (size_t)k + 1], R.u[3 * (size_t)k + 2], -1.0);
            const int2 ij = make_int2(h->md_i[k], h->md_j[k]);
            CK(h2d(h, h->md_coef_d, &coef, sizeof(double4)));
            CK(h2d(h, h->md_ij_d, &ij, sizeof(int2)));
            CK(cudaMemsetAsync(h->qp_g2, 0, sizeof(double) * n, h->stream));
            launch_pair_axpy(1, h->md_ij_d, h->md_coef_d, h->qp_g2, h->stream);
            int pit = 0, st;
            if ((st = pcg_solve<HT, VT>(h, eta, 0.0, &pit, h->qp_g2))) return st;
            *pcg_iters += pit;
            if (h->s.project_spd == 2 && !h->proj_fallback && h->sc_host->breakdown) return -1;
            double* w = h->md_w[used];
            CK(cudaMemsetAsync(w, 0, sizeof(double) * n, h->stream));
            launch_add_vec<VT>(n, w, (const VT*)h->x, w, h->stream);
            Wh.resize(6 * (size_t)np * (used + 1));
            launch_gather_nodes(2 * np, h->md_nodes_d, w, h->md_pos_d, h->stream);
            CK(d2h(h, &Wh[6 * (size_t)np * used], h->md_pos_d, sizeof(double) * 6 * np));
            slot[k] = used++;
        }
        const int m = (int)wl.size();
        std::vector<double> S((size_t)m * m), rhs(m);
        for (int a = 0; a < m; a++) {
            rhs[a] = R.l[wl[a]] - pair_dot(R, wl[a], &D0[6 * (size_t)wl[a]]);
            for (int b = 0; b < m; b++)
                S[(size_t)a * m + b] = pair_dot(R, wl[a], &Wh[6 * (size_t)np * slot[wl[b]] + 6 * (size_t)wl[a]]);
        }
        for (int a = 0; a < m; a++)
            for (int b = 0; b < a; b++) S[(size_t)a * m + b] = S[(size_t)b * m + a] = 0.5 * (S[(size_t)a * m + b] + S[(size_t)b * m + a]);
        std::vector<double> sol = rhs;
        if (m && !dense_solve(m, S, sol)) return fail(SORS_ERR_NOT_CONVERGED, "max-distance pairs are dependent");
        mu.assign(np, 0.0);
        double mu_scale = 0.0;
        for (int a = 0; a < m; a++) { mu[wl[a]] = sol[a]; mu_scale = std::max(mu_scale, fabs(sol[a])); }
        const double tol_mu = 1e-14 + 1e-8 * mu_scale;
        bool changed = false;
        for (int k = 0; k < np; k++) {
            if (h->md_work[k]) {
                if (mu[k] < -tol_mu) { h->md_work[k] = 0; changed = true; }
                continue;
            }
            double v[6];
            for (int c = 0; c < 6; c++) {
                v[c] = D0[6 * (size_t)k + c];
                for (int a = 0; a < m; a++) v[c] += sol[a] * Wh[6 * (size_t)np * slot[wl[a]] + 6 * (size_t)k + c];
            }
            if (pair_dot(R, k, v) - R.l[k] < -tol_s) { h->md_work[k] = 1; changed = true; }
        }
        if (!changed) break;
    }
    for (int k = 0; k < np; k++) {
        if (!h->md_work[k] || slot[k] < 0) mu[k] = 0.0;
        if (mu[k] != 0.0) launch_axpy(n, mu[k], h->md_w[slot[k]], h->qp_dx, h->stream);
    }
    return SORS_OK;
}

// Held maxDistance pairs in the adjoint.  At a converged SQP step
// grad E(q) = sum_k mu_k grad g_k(q), so the step's sensitivity sees the
// Lagrangian Hessian H_L = H + sum_k (mu_k / L_k) (I - u_k u_k^T) on (x_i - x_j)
// (g_k = d_k - |x_i - x_j| has Hessian -(1/L)(I - u u^T) there) and the held
// rows a_k . lam = 0.  Both enter as columns c_q = (w at i, -w at j) on top of
// the node-projected solve lam0 = K^+ P b (K = P H P): the curvature as two
// columns per pair (w = t1, t2 spanning u-perp, weight mu/L), the row as one
// (w = -u).  With Y_q = K^+ P c_q, lam = lam0 + sum_q sigma_q z_q Y_q (sigma = -1
// for curvature columns, z = their force; +1 for rows, z = the multiplier) and a
// small dense system for z.  On return lam holds the result (host and adj_l)
// and extra (3N) the columns' forces sum_q sigma_q z_q c_q, which the
// reactions at fixed DOFs include.
template <typename HT, typename VT>
int adjoint_pairs(SorsHandle* h, double eta, std::vector<double>& lam, std::vector<double>& extra, int* iters) {
    const int n = h->ndof, np = (int)h->md_d.size();
    const int nh = (int)h->adj_pairs.size();
    std::vector<double> xp(6 * (size_t)np);
    launch_gather_nodes(2 * np, h->md_nodes_d, h->q, h->md_pos_d, h->stream);
    CK(d2h(h, xp.data(), h->md_pos_d, sizeof(double) * 6 * np));
    const PairRows R = pair_rows(h, xp);
    struct Col { int pair; double w[3]; double c; double sigma; };
    std::vector<Col> cols;
    for (int a = 0; a < nh; a++) {
        const int k = h->adj_pairs[a];
        const double* u = &R.u[3 * (size_t)k];
        const double L = R.l[k] + h->md_d[k];
        const double c = L > 0.0 ? h->adj_mu[a] / L : 0.0;
        if (c != 0.0) {
            double e[3] = {0, 0, 0};
            e[fabs(u[0]) < 0.9 ? 0 : 1] = 1.0;
            const double eu = e[0] * u[0] + e[1] * u[1] + e[2] * u[2];
            double t1[3] = {e[0] - eu * u[0], e[1] - eu * u[1], e[2] - eu * u[2]};
            const double tn = sqrt(t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2]);
            for (double& v : t1) v /= tn;
            const double t2[3] = {u[1] * t1[2] - u[2] * t1[1], u[2] * t1[0] - u[0] * t1[2], u[0] * t1[1] - u[1] * t1[0]};
            cols.push_back({k, {t1[0], t1[1], t1[2]}, c, -1.0});
            cols.push_back({k, {t2[0], t2[1], t2[2]}, c, -1.0});
        }
        cols.push_back({k, {-u[0], -u[1], -u[2]}, 0.0, 1.0});
    }
    const int m = (int)cols.size();
    while ((int)h->md_w.size() < m) {
        double* w = nullptr;
        int st;
        if ((st = dalloc_t(h, &w, (size_t)n))) return st;
        h->md_w.push_back(w);
    }
    // the columns at the pair nodes: col_p . v for v given there
    auto dot = [&](const Col& c, const double* v) {
        const double* vi = v + 6 * (size_t)c.pair;
        return c.w[0] * (vi[0] - vi[3]) + c.w[1] * (vi[1] - vi[4]) + c.w[2] * (vi[2] - vi[5]);
    };
    std::vector<double> y0(6 * (size_t)np), Y(6 * (size_t)np * m);
    launch_gather_nodes(2 * np, h->md_nodes_d, h->adj_l, h->md_pos_d, h->stream);
    CK(d2h(h, y0.data(), h->md_pos_d, sizeof(double) * 6 * np));
    h->proj_flag = h->pflag_d;
    h->proj_n = h->pn_d;
    for (int q = 0; q < m; q++) {
        // g = -c_q: the PCG solves K x = -P g
        const double4 coef = make_double4(cols[q].w[0], cols[q].w[1], cols[q].w[2], 1.0);
        const int2 ij = make_int2(h->md_i[cols[q].pair], h->md_j[cols[q].pair]);
        CK(h2d(h, h->md_coef_d, &coef, sizeof(double4)));
        CK(h2d(h, h->md_ij_d, &ij, sizeof(int2)));
        CK(cudaMemsetAsync(h->qp_g2, 0, sizeof(double) * n, h->stream));
        launch_pair_axpy(1, h->md_ij_d, h->md_coef_d, h->qp_g2, h->stream);
        int pit = 0, st = pcg_solve<HT, VT>(h, eta, 0.0, &pit, h->qp_g2);
        if (st) { h->proj_flag = nullptr; h->proj_n = nullptr; return st; }
        *iters += pit;
        CK(cudaMemsetAsync(h->md_w[q], 0, sizeof(double) * n, h->stream));
        launch_add_vec<VT>(n, h->md_w[q], (const VT*)h->x, h->md_w[q], h->stream);
        launch_gather_nodes(2 * np, h->md_nodes_d, h->md_w[q], h->md_pos_d, h->stream);
        CK(d2h(h, &Y[6 * (size_t)np * q], h->md_pos_d, sizeof(double) * 6 * np));
    }
    h->proj_flag = nullptr;
    h->proj_n = nullptr;
    std::vector<double> A((size_t)m * m), z(m);
    for (int p = 0; p < m; p++) {
        const bool curv = cols[p].sigma < 0.0;
        for (int q = 0; q < m; q++) {
            const double v = cols[q].sigma * dot(cols[p], &Y[6 * (size_t)np * q]);
            A[(size_t)p * m + q] = curv ? (p == q) - cols[p].c * v : v;
        }
        z[p] = curv ? cols[p].c * dot(cols[p], y0.data()) : -dot(cols[p], y0.data());
    }
    if (m && !dense_solve(m, A, z)) return fail(SORS_ERR_NOT_CONVERGED, "held max-distance pairs are dependent");
    extra.assign(n, 0.0);
    for (int q = 0; q < m; q++) {
        launch_axpy(n, cols[q].sigma * z[q], h->md_w[q], h->adj_l, h->stream);
        const int i = h->md_i[cols[q].pair], j = h->md_j[cols[q].pair];
        for (int c = 0; c < 3; c++) {
            extra[3 * (size_t)i + c] += cols[q].sigma * z[q] * cols[q].w[c];
            extra[3 * (size_t)j + c] -= cols[q].sigma * z[q] * cols[q].w[c];
        }
    }
    CK(d2h(h, lam.data(), h->adj_l, sizeof(double) * n));
    return SORS_OK;
}

// Solver::minimize_SQP (solver.cpp:109-197): at each iteration the QP
//   min 1/2 dx^T H dx + g^T dx  s.t.  dx_i = -(x_i - qPrev_i - dt val_i) (Neumann),
//                                     n_c . dx_v >= -n_c . (x_v - p_c)   (contact)
// is solved exactly by an active-set iteration: the working contacts are held
// as equalities (PCG on the subspace the constraints leave free, from a
// particular solution x0), violated contacts join, contacts with negative
// multipliers leave; x += dx until ||dx|| < DX_TOL.  (The reference solves the
// same QP with OSQP to its default 1e-3 tolerances.)
template <typename HT, typename VT>
int minimize_sqp(SorsHandle* h, double dt, SorsStepStats* stats) {
    const int n = h->ndof, N = h->N;
    int st;
    CK(cudaMemsetAsync(h->status, 0, sizeof(int), h->stream));
    // active constraints from the initial guess (solver.cpp:122-123)
    std::vector<double> qh(n);
    CK(d2h(h, qh.data(), h->q, sizeof(double) * n));
    if (!h->planes.empty()) update_plane_contacts(h, qh.data());
    if (!h->disks.empty()) update_disk_contacts(h, qh.data());
    std::vector<int> cnode;
    std::vector<double> cpt, cn;  // point and normal per constraint
    std::vector<char> taken(N, 0);
    auto add = [&](int v, const double* p, const double* nrm) {
        if (taken[v] || (h->has_neumann && h->mask_h[v])) return;  // one contact per node; Neumann nodes stay fixed
        taken[v] = 1;
        cnode.push_back(v);
        cpt.insert(cpt.end(), p, p + 3);
        cn.insert(cn.end(), nrm, nrm + 3);
    };
    for (size_t i = 0; i < h->plane_mask.size(); i++)
        if (h->plane_mask[i] >= 0) add(h->plane_surf[i], h->planes[h->plane_mask[i]].p, h->planes[h->plane_mask[i]].n);
    for (const auto& G : h->disk_groups)
        for (size_t i = 0; i < G.mask.size(); i++)
            if (G.mask[i] >= 0) add(G.surf[i], h->disks[G.mask[i]].c, h->disks[G.mask[i]].n);
    const int m = (int)cnode.size();
    const int np = (int)h->md_d.size();
    h->last_active = m;
    if ((st = ensure_sqp_buffers(h, m))) return st;
    std::vector<double> xpair(6 * (size_t)np), mu_pair;
    PairRows R;
    h->md_work.assign(np, 0);
    if (m) CK(h2d(h, h->cnode_d, cnode.data(), sizeof(int) * m));
    std::vector<char> inW(m, 0);
    std::vector<double> b(m), xc(3 * (size_t)m), chk(2 * (size_t)m);
    std::vector<double4> cnb(m);
    // projection: Neumann bits always; contact bits for the working set
    h->pflag_h.assign(N, 0);
    if (h->has_neumann)
        for (int v = 0; v < N; v++) h->pflag_h[v] = h->mask_h[v] & 7u;
    bool converged = false;
    // forcing: loose while the step is far from converged, tightened with the
    // squared contraction of ||dx|| (Eisenstat-Walker choice 2 on ||dx||)
    const double eta_min = mixed(h) ? std::max(h->s.pcg_rel_tol, 1e-6) : h->s.pcg_rel_tol;
    double eta = 1e-4, dx_prev = -1.0, dx_prev2 = -1.0;
    for (int it = 0; it < h->s.newton_max_iter; it++) {
        h->proj_fallback = false;
        if (dx_prev > 0.0 && dx_prev2 > 0.0) {
            const double ratio = dx_prev / dx_prev2;
            eta = std::min(1e-4, 0.9 * ratio * ratio);
        }
        eta = std::max(eta, eta_min);
        if (dx_prev > 0.0 && dx_prev < 1e3 * h->s.newton_dx_tol) eta = eta_min;  // the last iterations solve tight
        double abs_tol = 0.0;   // set by the first (cold) solve of this iteration
        if ((st = eval_system<HT>(h, dt, true, kAsmFull))) return st;
        launch_gather_nodes(m, h->cnode_d, h->q, h->cpos_d, h->stream);
        if (m) CK(d2h(h, xc.data(), h->cpos_d, sizeof(double) * 3 * m));
        CK(cudaMemcpyAsync(h->sc_host, h->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        if (h->sc_host->status & kFlagInverted) return fail(SORS_ERR_INVERTED, "Inverted Elements");
        for (int c = 0; c < m; c++) {
            const double* nn = &cn[3 * (size_t)c];
            const double* pp = &cpt[3 * (size_t)c];
            b[c] = -(nn[0] * (xc[3 * c] - pp[0]) + nn[1] * (xc[3 * c + 1] - pp[1]) + nn[2] * (xc[3 * c + 2] - pp[2]));
            cnb[c] = make_double4(nn[0], nn[1], nn[2], b[c]);
            if (it == 0) inW[c] = b[c] > 0.0;  // start with the constraints violated now
        }
        if (m) CK(h2d(h, h->cnb_d, cnb.data(), sizeof(double4) * m));
        if (np) {
            launch_gather_nodes(2 * np, h->md_nodes_d, h->q, h->md_pos_d, h->stream);
            CK(d2h(h, xpair.data(), h->md_pos_d, sizeof(double) * 6 * np));
            R = pair_rows(h, xpair);
            if (it == 0)
                for (int k = 0; k < np; k++) h->md_work[k] = R.l[k] > 0.0;  // violated now
        }
        if (stats) { stats->newton_iters++; stats->residual_norm = sqrt(h->sc_host->gnorm2); }
        int inner_used = 0, pcg_used = 0, adds = 0, drops = 0;
        for (int inner = 0; inner < 25; inner++) {
            inner_used++;
            for (int c = 0; c < m; c++) {
                const int v = cnode[c];
                h->pflag_h[v] = (uint8_t)((h->pflag_h[v] & 7u) | (inW[c] ? 8u : 0u));
                h->pn_h[v] = cnb[c];
            }
            CK(h2d(h, h->pflag_d, h->pflag_h.data(), (size_t)N));
            if (m) CK(h2d(h, h->pn_d, h->pn_h.data(), sizeof(double4) * N));
            // particular solution: the constraints alone on the first solve, the
            // previous step with the new working set imposed on re-solves
            if (inner == 0) launch_qp_x0(N, h->pflag_d, h->pn_d, h->q, h->qPrev, h->mval, dt, h->qp_x0, h->stream);
            else launch_qp_warm(N, h->pflag_d, h->pn_d, h->q, h->qPrev, h->mval, dt, h->qp_dx, h->qp_x0, h->stream);
            launch_spmv_plain<HT>(N, h->row_ptr, h->col, (const HT*)h->H, h->nnzb, h->qp_x0, h->qp_y, h->stream);
            launch_add_vec<double>(n, h->g, h->qp_y, h->qp_g2, h->stream);
            h->proj_flag = h->pflag_d;
            h->proj_n = h->pn_d;
            int pit = 0;
            // re-solves stop at the accuracy the cold solve asked for, in absolute terms
            st = pcg_solve<HT, VT>(h, inner == 0 ? eta : 0.0, abs_tol, &pit, h->qp_g2);
            if (inner == 0) abs_tol = eta * sqrt(h->sc_host->bnorm2);
            h->proj_flag = nullptr;
            h->proj_n = nullptr;
            if (st) return st;
            if (stats) stats->pcg_iters += pit;
            pcg_used += pit;
            if (h->s.project_spd == 2 && !h->proj_fallback && h->sc_host->breakdown) {
                // negative curvature in the exact Hessian: redo with the projected one
                h->proj_fallback = true;
                if ((st = eval_system<HT>(h, dt, true, kAsmFull))) return st;
                inner--;
                continue;
            }
            launch_add_vec<VT>(n, h->qp_x0, (const VT*)h->x, h->qp_dx, h->stream);
            if (np) {
                h->proj_flag = h->pflag_d;
                h->proj_n = h->pn_d;
                int pp = 0;
                st = solve_pairs<HT, VT>(h, R, eta, mu_pair, &pp);
                h->proj_flag = nullptr;
                h->proj_n = nullptr;
                if (stats) stats->pcg_iters += pp;
                pcg_used += pp;
                if (st == -1) {
                    h->proj_fallback = true;
                    if ((st = eval_system<HT>(h, dt, true, kAsmFull))) return st;
                    inner--;
                    continue;
                }
                if (st) return st;
            }
            if (m == 0) break;
            launch_spmv_plain<HT>(N, h->row_ptr, h->col, (const HT*)h->H, h->nnzb, h->qp_dx, h->qp_y, h->stream);
            if (np) {
                // the held pairs' forces: y = H dx - sum_k mu_k a_k
                std::vector<int2> ij;
                std::vector<double4> coef;
                for (int k = 0; k < np; k++)
                    if (mu_pair[k] != 0.0) {
                        ij.push_back(make_int2(h->md_i[k], h->md_j[k]));
                        coef.push_back(make_double4(R.u[3 * (size_t)k], R.u[3 * (size_t)k + 1], R.u[3 * (size_t)k + 2],
                                                    -mu_pair[k]));
                    }
                if (!ij.empty()) {
                    CK(h2d(h, h->md_ij_d, ij.data(), sizeof(int2) * ij.size()));
                    CK(h2d(h, h->md_coef_d, coef.data(), sizeof(double4) * coef.size()));
                    launch_pair_axpy((int)ij.size(), h->md_ij_d, h->md_coef_d, h->qp_y, h->stream);
                }
            }
            launch_qp_check(m, h->cnode_d, h->cnb_d, h->qp_dx, h->qp_y, h->g, h->cout_d, h->stream);
            CK(d2h(h, chk.data(), h->cout_d, sizeof(double) * 2 * m));
            double mu_scale = 0.0, b_scale = 0.0;
            for (int c = 0; c < m; c++) {
                mu_scale = std::max(mu_scale, fabs(chk[m + c]));
                b_scale = std::max(b_scale, fabs(b[c]));
            }
            const double tol_s = 1e-12 + 1e-9 * b_scale, tol_mu = 1e-14 + 1e-8 * mu_scale;
            bool changed = false;
            for (int c = 0; c < m; c++) {
                if (!inW[c] && chk[c] < -tol_s) { inW[c] = 1; changed = true; adds++; }
                else if (inW[c] && chk[m + c] < -tol_mu) { inW[c] = 0; changed = true; drops++; }
            }
            if (!changed) break;
        }
        CK(cudaMemcpyAsync(h->q0, h->q, sizeof(double) * n, cudaMemcpyDeviceToDevice, h->stream));
        double alpha = 1.0;
        if (it >= 1 && h->proj_fallback) {
            // A step from the projected Hessian (the exact one had negative
            // curvature) is a descent direction but not a Newton step: backtrack
            // on the energy (Armijo, c = 1e-4, halving), as full steps can cycle.
            // The held constraints are satisfied after the first iteration and
            // are linear, so every alpha in (0, 1] keeps them.
            double e0, e1;
            launch_dot_gdx<double>(n, h->g, h->qp_dx, h->partials, h->sc, h->stream);
            if ((st = eval_energy(h, dt, &e0))) return st;
            const double gdx = h->sc_host->gdx;
            if (gdx < 0.0) {
                for (int ls = 0; ls < 20; ls++) {
                    launch_newton_update<double>(n, h->qp_dx, alpha, h->q, h->q0, h->partials, h->sc, 6, h->stream);
                    if ((st = eval_energy(h, dt, &e1))) return st;
                    if (e1 <= e0 + 1e-4 * alpha * gdx) break;
                    alpha *= 0.5;
                }
            }
        }
        launch_newton_update<double>(n, h->qp_dx, alpha, h->q, h->q0, h->partials, h->sc, 6, h->stream);
        CK(cudaMemcpyAsync(h->sc_host, h->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        // convergence is judged on the full step, as the reference does
        const double dxn = sqrt(h->sc_host->dxnorm2) / alpha;
        dx_prev2 = dx_prev;
        dx_prev = dxn;
        if (stats) stats->dx_norm = dxn;
        if (verbose()) {
            int held = 0;
            for (int c = 0; c < m; c++) held += inW[c];
            fprintf(stderr, "sqp it %d |g| %.3e dx %.3e alpha %.3f contacts %d held %d inner %d (+%d -%d) pcg %d eta %.1e%s\n",
                    it, sqrt(h->sc_host->gnorm2), dxn, alpha, m, held, inner_used, adds, drops, pcg_used, eta,
                    h->proj_fallback ? " projected" : "");
        }
        if (!(dxn == dxn)) break;  // "SQP method diverged"
        if (dxn < h->s.newton_dx_tol) { converged = true; break; }
    }
    if (!converged) return fail(SORS_ERR_NOT_CONVERGED, "SQP method did not converge");
    h->held_pairs.clear();
    h->held_mu.clear();
    for (int k = 0; k < np; k++)
        if (h->md_work[k]) {
            h->held_pairs.push_back(k);
            h->held_mu.push_back(k < (int)mu_pair.size() ? mu_pair[k] : 0.0);
        }
    h->held_nodes.clear();
    h->held_normals.clear();
    for (int c = 0; c < m; c++)
        if (inW[c]) {
            h->held_nodes.push_back(cnode[c]);
            h->held_normals.insert(h->held_normals.end(), &cn[3 * (size_t)c], &cn[3 * (size_t)c] + 3);
        }
    return SORS_OK;
}

int run_minimize(SorsHandle* h, double dt, SorsStepStats* stats) {
    if (method(h) == 3) return mixed(h) ? minimize_sqp<float, float>(h, dt, stats) : minimize_sqp<double, double>(h, dt, stats);
    if (mixed(h)) return minimize<float, float>(h, dt, stats);
    return minimize<double, double>(h, dt, stats);
}

// CFL time step (solver.cpp:300-331): the shortest element edge at q and
// max |vPrev| reduced on the device, dt_CFL = l_min / v_max, at most dt.
int cfl_dt(SorsHandle* h, double dt, double* out) {
    launch_cfl(h->E, h->nv, h->q, h->conn, h->ndof, h->vPrev, h->partials, h->sc, h->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h->sc_host, h->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    const double dtc = h->sc_host->minedge / h->sc_host->vmax;
    *out = dtc < dt ? dtc : dt;
    return SORS_OK;
}

int step_resident(SorsHandle* h, double dt, int substeps, SorsStepStats* stats) {
    h->step_indefinite = 0;
    h->step_min_rq = INFINITY;
    if (dt == 0.0) dt = h->s.dt;
    if (substeps == 0) substeps = h->s.substeps;
    if (h->s.cfl) {
        double dtc;
        int st = cfl_dt(h, dt, &dtc);
        if (st) return st;
        substeps = (int)ceil(dt / dtc);
    }
    if (substeps < 1) return fail(SORS_ERR_ARG, "substeps must be >= 1");
    double dts = dt / substeps;
    if (stats) memset(stats, 0, sizeof(*stats));
    for (int j = 0; j < substeps; j++) {
        int st;
        if (h->s.newton_predictor && dts != 0.0 && method(h) != 3) {
            CK(cudaMemcpyAsync(h->q_save, h->q, sizeof(double) * h->ndof, cudaMemcpyDeviceToDevice, h->stream));
            launch_predict(h->ndof, h->q, h->vPrev, dts, h->stream);
            st = run_minimize(h, dts, stats);
            if (st == SORS_ERR_INVERTED) {
                // the predicted start inverted an element: restart from the given solution
                CK(cudaMemcpyAsync(h->q, h->q_save, sizeof(double) * h->ndof, cudaMemcpyDeviceToDevice, h->stream));
                st = run_minimize(h, dts, stats);
            }
        } else {
            st = run_minimize(h, dts, stats);
        }
        if (st) return st;
        launch_update_state(h->ndof, h->q, h->qPrev, h->vPrev, h->gPrev, h->gPrevTmp, dts, h->s.time_stepping,
                            h->stream);
        if (stats) stats->substeps++;
    }
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaGetLastError());
    return SORS_OK;
}

int set_device(SorsHandle* h) {
    CK(cudaSetDevice(h->device));
    set_grid_cap(h->s.max_blocks);
    return SORS_OK;
}

// Locality order of the nodes: connected components in the order of their
// lowest caller index (so that the meshes of a union keep their node ranges),
// within each the two-level aggregate boxes (agg_bins) in Morton order, and
// within a box the Morton order of the undeformed positions (21 bits per axis,
// one scale for all axes), so that every aggregate is a contiguous node range.
// SORS_NO_RENUMBER=1 keeps the caller's numbering (for comparison).
void locality_order(int N, int E, int nv, const double* X, const int32_t* conn, std::vector<int>& n2o) {
    std::vector<int> parent(N);
    for (int i = 0; i < N; i++) parent[i] = i;
    auto find = [&](int a) {
        while (parent[a] != a) a = parent[a] = parent[parent[a]];
        return a;
    };
    for (int e = 0; e < E; e++)
        for (int v = 1; v < nv; v++) {
            int a = find(conn[(size_t)e * nv]), b = find(conn[(size_t)e * nv + v]);
            if (a != b) parent[std::max(a, b)] = std::min(a, b);
        }
    std::vector<int> root(N);
    for (int i = 0; i < N; i++) root[i] = find(i);  // the component's lowest index
    double lo[3] = {X[0], X[1], X[2]}, hi[3] = {X[0], X[1], X[2]};
    for (int i = 0; i < N; i++)
        for (int k = 0; k < 3; k++) {
            lo[k] = std::min(lo[k], X[3 * (size_t)i + k]);
            hi[k] = std::max(hi[k], X[3 * (size_t)i + k]);
        }
    auto spread = [](uint64_t v) {
        v &= 0x1fffff;
        v = (v | v << 32) & 0x1f00000000ffffULL;
        v = (v | v << 16) & 0x1f0000ff0000ffULL;
        v = (v | v << 8) & 0x100f00f00f00f00fULL;
        v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
        v = (v | v << 2) & 0x1249249249249249ULL;
        return v;
    };
    const double ext = std::max(hi[0] - lo[0], std::max(hi[1] - lo[1], hi[2] - lo[2]));
    const AggBins ab = agg_bins(N, X);
    std::vector<std::tuple<int, uint64_t, uint64_t, int>> key(N);
    for (int i = 0; i < N; i++) {
        uint64_t code = 0, box = 0;
        int c[3];
        ab.cell(X + 3 * (size_t)i, c);
        for (int k = 0; k < 3; k++) {
            const double u = ext > 0 ? (X[3 * (size_t)i + k] - lo[k]) / ext : 0.0;
            code |= spread((uint64_t)std::min(2097151.0, std::max(0.0, u * 2097151.0))) << k;
            box |= spread((uint64_t)c[k]) << k;
        }
        key[i] = std::make_tuple(root[i], box, code, i);
    }
    std::sort(key.begin(), key.end());
    n2o.resize(N);
    for (int i = 0; i < N; i++) n2o[i] = std::get<3>(key[i]);
}

// Caller-numbered DOF vector (host or device) -> internal device vector.
int dof_in(SorsHandle* h, double* dst, const double* src, cudaMemcpyKind kind) {
    const size_t bytes = sizeof(double) * h->ndof;
    if (!h->renum) {
        CK(cudaMemcpyAsync(dst, src, bytes, kind, h->stream));
        return SORS_OK;
    }
    CK(cudaMemcpyAsync(h->perm_tmp, src, bytes, kind, h->stream));
    launch_gather_dofs(h->N, h->perm_tmp, h->n2o_d, dst, h->stream);
    return SORS_OK;
}

// Internal device vector -> caller-numbered DOF vector (host or device); the
// caller synchronises before reading a host destination.
int dof_out(SorsHandle* h, double* dst, const double* src, cudaMemcpyKind kind) {
    const size_t bytes = sizeof(double) * h->ndof;
    if (!h->renum) {
        CK(cudaMemcpyAsync(dst, src, bytes, kind, h->stream));
        return SORS_OK;
    }
    launch_gather_dofs(h->N, src, h->o2n_d, h->perm_tmp, h->stream);
    CK(cudaMemcpyAsync(dst, h->perm_tmp, bytes, kind, h->stream));
    return SORS_OK;
}

// Host-side conversions (set-up and diagnostic calls).
std::vector<double> dofs_to_internal(const SorsHandle* h, const double* src) {
    std::vector<double> out((size_t)h->ndof);
    for (int i = 0; i < h->N; i++)
        for (int k = 0; k < 3; k++) out[3 * (size_t)i + k] = src[3 * (size_t)(h->renum ? h->n2o[i] : i) + k];
    return out;
}
void dofs_to_caller(const SorsHandle* h, const double* src, double* dst) {
    for (int i = 0; i < h->N; i++)
        for (int k = 0; k < 3; k++) dst[3 * (size_t)(h->renum ? h->n2o[i] : i) + k] = src[3 * (size_t)i + k];
}
inline int node_in(const SorsHandle* h, int v) { return h->renum ? h->o2n[v] : v; }
inline int elem_out(const SorsHandle* h, int e) { return h->renum_e ? h->e2o[e] : e; }
inline int node_out(const SorsHandle* h, int v) { return h->renum ? h->n2o[v] : v; }

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

void sors_default_settings(SorsSettings* s) {
    memset(s, 0, sizeof(*s));
    s->time_stepping = 1;  // SimulationSettings default "crank_nicolson"
    s->solver_method = 0;
    s->dt = 0.0;
    s->substeps = 1;
    s->cfl = 0;
    s->damping_alpha = 0.0;
    s->precision = 0;
    s->project_spd = 2;
    s->material = 0;
    s->newton_dx_tol = 1e-9;
    s->newton_res_tol = 0.0;
    s->newton_max_iter = 100;
    s->pcg_rel_tol = 1e-10;
    s->pcg_max_iter = 20000;
    s->device = 0;
    s->newton_predictor = 1;
    s->max_blocks = 0;
    s->newton_safeguard = 0;
    s->two_level = 2;
    s->linear_solver = 0;
    s->pressure_jac_exact = 0;
}

int sors_last_error(char* buf, size_t n) {
    if (!buf || n == 0) return (int)g_last_error.size();
    size_t k = std::min(n - 1, g_last_error.size());
    memcpy(buf, g_last_error.data(), k);
    buf[k] = 0;
    return (int)k;
}

int sors_create(const double* X, int32_t n_nodes, const int32_t* conn, int32_t n_elems, int32_t nodes_per_elem,
                const double* density, const double* youngs, const double* poisson, const SorsSettings* settings,
                SorsHandle** out) {
    if (!out) return fail(SORS_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (nodes_per_elem != 4 && nodes_per_elem != 8) return fail(SORS_ERR_ARG, "nodes_per_elem must be 4 or 8");
    if (n_nodes <= 0 || n_elems < 0 || !X || (n_elems > 0 && (!conn || !density || !youngs || !poisson)))
        return fail(SORS_ERR_ARG, "empty mesh or NULL input");
    for (long long t = 0; t < (long long)n_elems * nodes_per_elem; t++)
        if (conn[t] < 0 || conn[t] >= n_nodes) return fail(SORS_ERR_ARG, "element index out of range");
    SorsHandle* h = new (std::nothrow) SorsHandle();
    if (!h) return fail(SORS_ERR_OOM, "host allocation failed");
    if (settings) h->s = *settings; else sors_default_settings(&h->s);
    h->N = n_nodes; h->E = n_elems; h->nv = nodes_per_elem; h->ndof = 3 * n_nodes;
    h->device = h->s.device;
    int st;
    auto bail = [&](int code) { sors_destroy(h); return code; };
    if ((st = set_device(h))) return bail(st);
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(SORS_ERR_CUDA, "stream creation failed"));
    const int N = n_nodes, E = n_elems, nv = nodes_per_elem;
    // the handle's node numbering (locality order); the rest of the set-up
    // reads the renumbered positions and connectivity
    std::vector<double> X_int, rho_int, youngs_int, poisson_int;
    std::vector<int32_t> conn_int;
    {
        const char* env = getenv("SORS_NO_RENUMBER");
        const bool off = env && *env && *env != '0';
        if (!off) locality_order(N, E, nv, X, conn, h->n2o);
        h->renum = false;
        if (!off)
            for (int i = 0; i < N && !h->renum; i++) h->renum = h->n2o[i] != i;
        if (h->renum) {
            h->o2n.assign(N, 0);
            for (int i = 0; i < N; i++) h->o2n[h->n2o[i]] = i;
            X_int.resize((size_t)3 * N);
            for (int i = 0; i < N; i++)
                for (int k = 0; k < 3; k++) X_int[3 * (size_t)i + k] = X[3 * (size_t)h->n2o[i] + k];
            // elements in the order of their lowest internal vertex
            std::vector<std::pair<int, int>> ek((size_t)E);
            for (int e = 0; e < E; e++) {
                int mn = N;
                for (int v = 0; v < nv; v++) mn = std::min(mn, h->o2n[conn[(size_t)e * nv + v]]);
                ek[e] = {mn, e};
            }
            std::sort(ek.begin(), ek.end());
            h->e2o.resize(E);
            for (int e = 0; e < E; e++) {
                h->e2o[e] = ek[e].second;
                h->renum_e |= h->e2o[e] != e;
            }
            conn_int.resize((size_t)E * nv);
            for (int e = 0; e < E; e++)
                for (int v = 0; v < nv; v++)
                    conn_int[(size_t)e * nv + v] = h->o2n[conn[(size_t)h->e2o[e] * nv + v]];
            X = X_int.data();
            conn = conn_int.data();
            if (h->renum_e) {
                rho_int.resize(E); youngs_int.resize(E); poisson_int.resize(E);
                for (int e = 0; e < E; e++) {
                    rho_int[e] = density[h->e2o[e]];
                    youngs_int[e] = youngs[h->e2o[e]];
                    poisson_int[e] = poisson[h->e2o[e]];
                }
                density = rho_int.data(); youngs = youngs_int.data(); poisson = poisson_int.data();
            }
            if ((st = upload(h, &h->n2o_d, h->n2o.data(), (size_t)N))) return bail(st);
            if ((st = upload(h, &h->o2n_d, h->o2n.data(), (size_t)N))) return bail(st);
            if ((st = dalloc_t(h, &h->perm_tmp, (size_t)3 * N))) return bail(st);
        } else {
            h->n2o.clear();
        }
    }
    // per-element Lame parameters (neoHookean.cpp:10-11) and lumped mass (energy.cpp:176-189)
    std::vector<double2> mat(E > 0 ? E : 1);
    std::vector<double> mass(N, 0.0);
    for (int e = 0; e < E; e++) {
        mat[e] = lame_params(youngs[e], poisson[e], h->s.material);
        double m = density[e] * elem_volume(X, conn + (size_t)e * nv, nv);
        for (int v = 0; v < nv; v++) mass[conn[(size_t)e * nv + v]] += m / nv;
    }
    h->youngs_h.assign(youngs, youngs + E);
    h->poisson_h.assign(poisson, poisson + E);
    h->mass_h = mass;
    if ((st = upload(h, &h->X, X, (size_t)3 * N))) return bail(st);
    if ((st = upload(h, &h->conn, conn, (size_t)E * nv))) return bail(st);
    if ((st = upload(h, &h->mat, mat.data(), (size_t)E))) return bail(st);
    if ((st = upload(h, &h->mass, mass.data(), (size_t)N))) return bail(st);
    if (nv == 4) {
        if ((st = dalloc_t(h, &h->tshape, (size_t)10 * std::max(1, E)))) return bail(st);
        launch_tet_shapes(E, h->X, h->conn, h->tshape, h->stream);
        CK(cudaStreamSynchronize(h->stream));
    }
    {
        PatternHost ph;
        if ((st = build_pattern(h, conn, &ph))) return bail(st);
        if ((st = build_tet_chunks(h, conn, X, ph))) return bail(st);
    }
    if (nv == 8 && E > 0 && (h->s.material == 0 || h->s.material == 2)) {
        // element tiles of the element-owner hex assembly
        if ((st = dalloc(h, &h->hex_tile, (size_t)E * 36 * 9 * hsize(h)))) return bail(st);
        if ((st = dalloc_t(h, &h->hex_gtile, (size_t)E * 24))) return bail(st);
        std::vector<int> br((size_t)h->nnzb);
        for (int i = 0; i < N; i++)
            for (int b = h->row_ptr_h[i]; b < h->row_ptr_h[i + 1]; b++) br[b] = i;
        if ((st = upload(h, &h->hex_blk_row, br.data(), br.size()))) return bail(st);
    }
    const size_t nd = (size_t)3 * N;
    double** vecs[] = {&h->q, &h->q0, &h->qPrev, &h->vPrev, &h->gPrev, &h->gPrevTmp, &h->g, &h->g_int, &h->f_ext,
                       &h->mval, &h->vforce, &h->q_save};
    for (double** p : vecs) {
        if ((st = dalloc_t(h, p, nd))) return bail(st);
        CK(dzero(h, *p, nd * sizeof(double)));
    }
    // TimeIntegrator(settings, undeformed vertices): qPrev = X (integrator.h:155-161)
    CK(h2d(h, h->qPrev, X, nd * sizeof(double)));
    CK(h2d(h, h->q, X, nd * sizeof(double)));
    h->mask_h.assign(N, 0);
    if ((st = upload(h, &h->node_mask, h->mask_h.data(), (size_t)N))) return bail(st);
    // two_level 2 ("auto"): on for meshes of 20,000 nodes or more, where the
    // coarse correction's three extra kernels per iteration pay for themselves
    if (h->s.two_level == 2) h->s.two_level = N >= 20000 ? 1 : 0;
    if (h->s.two_level && (st = setup_two_level(h, X))) return bail(st);
    size_t hs = hsize(h);
    // 160 bytes of padding: the SpMV reads values in 144-byte groups, the last of
    // which may run past the last block
    if ((st = dalloc(h, &h->H, (size_t)h->nnzb * 9 * hs + 160))) return bail(st);
    CK(dzero(h, (char*)h->H + (size_t)h->nnzb * 9 * hs, 160));
    if ((st = dalloc(h, &h->Minv, (size_t)N * 9 * hs))) return bail(st);
    void** vv[] = {&h->x, &h->r, &h->z, &h->p0, &h->p1, &h->qv};
    for (void** p : vv) {
        // the search directions p0, p1 are padded to 4 values per node
        const size_t bytes = (p == &h->p0 || p == &h->p1) ? (size_t)N * 4 * hs : nd * hs;
        if ((st = dalloc(h, p, bytes))) return bail(st);
        CK(dzero(h, *p, bytes));
    }
    if ((st = dalloc_t(h, &h->partials, (size_t)kRedBlocks * kMaxScalars))) return bail(st);
    if ((st = dalloc_t(h, &h->sc, 1))) return bail(st);
    CK(dzero(h, h->sc, sizeof(DevScalars)));
    h->status = &h->sc->status;
    if (cudaMallocHost((void**)&h->sc_host, sizeof(DevScalars)) != cudaSuccess)
        return bail(fail(SORS_ERR_OOM, "pinned allocation failed"));
    if ((st = dalloc_t(h, &h->pressure_d, 1))) return bail(st);
    // synchronous copies above ran on the legacy stream; no device-wide sync here,
    // so that a handle created while others are capturing PCG graphs does not
    // invalidate their capture
    CK(cudaStreamSynchronize(h->stream));
    *out = h;
    return SORS_OK;
}

void sors_destroy(SorsHandle* h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->pcg_exec) cudaGraphExecDestroy(h->pcg_exec);
    for (void* p : h->allocs) cudaFree(p);
    if (h->sc_host) cudaFreeHost(h->sc_host);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

int sors_set_neumann(SorsHandle* h, const int32_t* mask, const double* value) {
    if (!h || !mask || !value) return fail(SORS_ERR_ARG, "NULL argument");
    int st;
    if ((st = set_device(h))) return st;
    for (int i = 0; i < h->N; i++) {
        uint8_t m = 0;
        const int o = node_out(h, i);
        for (int k = 0; k < 3; k++)
            if (mask[3 * o + k] == 1) m |= (uint8_t)(1u << k);
        h->mask_h[i] = m;
    }
    CK(h2d(h, h->node_mask, h->mask_h.data(), h->N));
    {
        const std::vector<double> vi = dofs_to_internal(h, value);
        CK(h2d(h, h->mval, vi.data(), sizeof(double) * h->ndof));
    }
    h->has_neumann = true;
    h->tl_ready = false;  // the coarse space drops held DOFs
    return SORS_OK;
}

int sors_set_pressure_faces(SorsHandle* h, const int32_t* faces, int32_t n_faces, int32_t verts_per_face,
                            const int32_t* groups, int32_t n_groups) {
    if (!h || (n_faces > 0 && (!faces || !groups))) return fail(SORS_ERR_ARG, "NULL argument");
    if (verts_per_face != 3 && verts_per_face != 4) return fail(SORS_ERR_ARG, "faces must have 3 or 4 vertices");
    if ((h->nv == 4) != (verts_per_face == 3))
        return fail(SORS_ERR_ARG, "tet meshes take triangles, hex meshes take quads");
    int st;
    if ((st = set_device(h))) return st;
    for (long long t = 0; t < (long long)n_faces * verts_per_face; t++)
        if (faces[t] < 0 || faces[t] >= h->N) return fail(SORS_ERR_ARG, "face vertex out of range");
    for (int f = 0; f < n_faces; f++)
        if (groups[f] < 0 || groups[f] >= n_groups) return fail(SORS_ERR_ARG, "face group out of range");
    std::vector<int32_t> faces_int((size_t)n_faces * verts_per_face);
    for (size_t t = 0; t < faces_int.size(); t++) faces_int[t] = node_in(h, faces[t]);
    faces = faces_int.data();
    // surface rows: node -> (face, local index)
    std::vector<std::vector<int>> inc(h->N);
    for (int f = 0; f < n_faces; f++)
        for (int k = 0; k < verts_per_face; k++) inc[faces[(size_t)f * verts_per_face + k]].push_back(f * 4 + k);
    std::vector<int> surf, ptr(1, 0), fl;
    for (int i = 0; i < h->N; i++)
        if (!inc[i].empty()) {
            surf.push_back(i);
            fl.insert(fl.end(), inc[i].begin(), inc[i].end());
            ptr.push_back((int)fl.size());
        }
    h->n_faces = n_faces; h->fnv = verts_per_face; h->n_groups = n_groups; h->nsurf = (int)surf.size();
    if ((st = upload(h, &h->faces, faces, (size_t)n_faces * verts_per_face))) return st;
    if ((st = upload(h, &h->face_group, groups, (size_t)n_faces))) return st;
    if ((st = upload(h, &h->surf_nodes, surf.data(), surf.size()))) return st;
    if ((st = upload(h, &h->sface_ptr, ptr.data(), ptr.size()))) return st;
    if ((st = upload(h, &h->sface_fl, fl.data(), fl.size()))) return st;
    if ((st = dalloc_t(h, &h->pressure_d, (size_t)std::max(1, n_groups)))) return st;
    CK(dzero(h, h->pressure_d, sizeof(double) * std::max(1, n_groups)));
    h->has_pressure = true;
    return SORS_OK;
}

int sors_enable_vertex_force(SorsHandle* h, int32_t enable) {
    if (!h) return fail(SORS_ERR_ARG, "NULL handle");
    h->has_vforce = enable != 0;
    return SORS_OK;
}

int sors_set_actuation(SorsHandle* h, const char* name, const double* values, int64_t n) {
    if (!h || !name || (n > 0 && !values)) return fail(SORS_ERR_ARG, "NULL argument");
    int st;
    if ((st = set_device(h))) return st;
    std::string nm(name);
    if (nm == "pressure") {
        if (!h->has_pressure) return SORS_OK;  // unused actuation entries are ignored
        if (n < h->n_groups) return fail(SORS_ERR_ARG, "pressure actuation has fewer entries than surface groups");
        CK(h2d(h, h->pressure_d, values, sizeof(double) * h->n_groups));
        return SORS_OK;
    }
    if (nm == "vertexForce") {
        if (n != h->ndof) return fail(SORS_ERR_ARG, "vertexForce actuation must have 3N entries");
        if ((st = dof_in(h, h->vforce, values, cudaMemcpyHostToDevice))) return st;
        CK(cudaStreamSynchronize(h->stream));
        return SORS_OK;
    }
    if (nm == "softconMuscle") {
        if (!h->mgroup) return SORS_OK;  // no element carries a fibre term
        if (n < h->n_mgroups) return fail(SORS_ERR_ARG, "softconMuscle actuation has fewer entries than muscle groups");
        CK(h2d(h, h->mact, values, sizeof(double) * h->n_mgroups));
        return SORS_OK;
    }
    return SORS_OK;  // other Params keys are not used by this mesh's energies
}

int sors_set_muscles(SorsHandle* h, const int32_t* group, const double* stiffness, const double* direction,
                     int32_t n_groups) {
    if (!h || !group || !stiffness || !direction) return fail(SORS_ERR_ARG, "NULL argument");
    if (n_groups < 1) return fail(SORS_ERR_ARG, "n_groups must be positive");
    int st;
    if ((st = set_device(h))) return st;
    std::vector<double4> prm((size_t)std::max(1, h->E));
    std::vector<int32_t> grp_int((size_t)std::max(1, h->E));
    for (int e = 0; e < h->E; e++) {
        const int o = elem_out(h, e);
        if (group[o] >= n_groups || group[o] < -1) return fail(SORS_ERR_ARG, "muscle group out of range");
        prm[e] = make_double4(direction[3 * (size_t)o], direction[3 * (size_t)o + 1], direction[3 * (size_t)o + 2],
                              stiffness[o]);
        grp_int[e] = group[o];
    }
    group = grp_int.data();
    if (!h->mgroup) {
        if ((st = dalloc_t(h, &h->mgroup, (size_t)std::max(1, h->E)))) return st;
        if ((st = dalloc_t(h, &h->mparam, (size_t)std::max(1, h->E)))) return st;
    }
    if (n_groups > h->n_mgroups) {
        if ((st = dalloc_t(h, &h->mact, (size_t)n_groups))) return st;
        CK(dzero(h, h->mact, sizeof(double) * n_groups));
    }
    h->n_mgroups = std::max(h->n_mgroups, (int)n_groups);
    h->mgroup_h.assign(group, group + h->E);
    if (h->E) {
        CK(h2d(h, h->mgroup, group, sizeof(int) * h->E));
        CK(h2d(h, h->mparam, prm.data(), sizeof(double4) * h->E));
    }
    return SORS_OK;
}

int sors_set_initial_deformation(SorsHandle* h, const double* q) {
    if (!h || !q) return fail(SORS_ERR_ARG, "NULL argument");
    int st;
    if ((st = set_device(h))) return st;
    if ((st = dof_in(h, h->qPrev, q, cudaMemcpyHostToDevice))) return st;
    CK(cudaStreamSynchronize(h->stream));
    return SORS_OK;
}

int sors_set_initial_velocity(SorsHandle* h, const double* v) {
    if (!h || !v) return fail(SORS_ERR_ARG, "NULL argument");
    int st;
    if ((st = set_device(h))) return st;
    if ((st = dof_in(h, h->vPrev, v, cudaMemcpyHostToDevice))) return st;
    CK(cudaStreamSynchronize(h->stream));
    return SORS_OK;
}

int sors_get_state(SorsHandle* h, double* q_prev, double* v_prev) {
    if (!h) return fail(SORS_ERR_ARG, "NULL handle");
    int st;
    if ((st = set_device(h))) return st;
    if (q_prev && (st = dof_out(h, q_prev, h->qPrev, cudaMemcpyDeviceToHost))) return st;
    CK(cudaStreamSynchronize(h->stream));
    if (v_prev && (st = dof_out(h, v_prev, h->vPrev, cudaMemcpyDeviceToHost))) return st;
    CK(cudaStreamSynchronize(h->stream));
    return SORS_OK;
}

int sors_energy(SorsHandle* h, const double* q, double dt, double* out) {
    if (!h || !q || !out) return fail(SORS_ERR_ARG, "NULL argument");
    int st;
    if ((st = set_device(h))) return st;
    if ((st = dof_in(h, h->q, q, cudaMemcpyHostToDevice))) return st;
    return eval_energy(h, dt, out);
}

int sors_gradient(SorsHandle* h, const double* q, double dt, double* g) {
    if (!h || !q || !g) return fail(SORS_ERR_ARG, "NULL argument");
    int st;
    if ((st = set_device(h))) return st;
    if ((st = dof_in(h, h->q, q, cudaMemcpyHostToDevice))) return st;
    st = mixed(h) ? eval_system<float>(h, dt, false) : eval_system<double>(h, dt, false);
    if (st) return st;
    if ((st = dof_out(h, g, h->g, cudaMemcpyDeviceToHost))) return st;
    CK(cudaStreamSynchronize(h->stream));
    return SORS_OK;
}

int sors_hessian_bsr(SorsHandle* h, const double* q, double dt, int32_t* row_ptr, int32_t* col, double* val,
                     int64_t* nnzb) {
    if (!h) return fail(SORS_ERR_ARG, "NULL handle");
    if (nnzb) *nnzb = h->nnzb;
    if (!row_ptr && !col && !val) return SORS_OK;
    int st;
    if ((st = set_device(h))) return st;
    if (h->renum && h->caller_blk.empty()) {
        // the pattern in the caller's numbering: caller row o is internal row
        // o2n[o]; its blocks sorted by caller column
        const int N = h->N;
        h->caller_row_ptr.assign(N + 1, 0);
        h->caller_col.resize(h->nnzb);
        h->caller_blk.resize(h->nnzb);
        std::vector<std::pair<int, int>> tmp;
        for (int o = 0; o < N; o++) {
            const int i = h->o2n[o];
            tmp.clear();
            for (int b = h->row_ptr_h[i]; b < h->row_ptr_h[i + 1]; b++) tmp.push_back({h->n2o[h->col_h[b]], b});
            std::sort(tmp.begin(), tmp.end());
            const int b0 = h->caller_row_ptr[o];
            for (size_t k = 0; k < tmp.size(); k++) {
                h->caller_col[b0 + k] = tmp[k].first;
                h->caller_blk[b0 + k] = tmp[k].second;
            }
            h->caller_row_ptr[o + 1] = b0 + (int)tmp.size();
        }
    }
    const int* rp_out = h->renum ? h->caller_row_ptr.data() : h->row_ptr_h.data();
    const int* col_out = h->renum ? h->caller_col.data() : h->col_h.data();
    if (row_ptr) memcpy(row_ptr, rp_out, sizeof(int) * (h->N + 1));
    if (col) memcpy(col, col_out, sizeof(int) * h->nnzb);
    if (!val) return SORS_OK;
    if (!q) return fail(SORS_ERR_ARG, "q is NULL");
    if ((st = dof_in(h, h->q, q, cudaMemcpyHostToDevice))) return st;
    CK(cudaMemsetAsync(h->status, 0, sizeof(int), h->stream));
    st = mixed(h) ? eval_system<float>(h, dt, true) : eval_system<double>(h, dt, true);
    if (st) return st;
    size_t n = (size_t)h->nnzb * 9;
    std::vector<double> raw(n);
    if (mixed(h)) {
        std::vector<float> tmp(n);
        CK(cudaMemcpyAsync(tmp.data(), h->H, n * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        for (size_t k = 0; k < n; k++) raw[k] = tmp[k];
    } else {
        CK(cudaMemcpyAsync(raw.data(), h->H, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    // the ABI returns each block's 9 values contiguously, row-major
    const size_t nb = (size_t)h->nnzb;
    for (size_t b = 0; b < nb; b++) {
        const size_t bi = h->renum ? (size_t)h->caller_blk[b] : b;
        for (int rc = 0; rc < 9; rc++) val[b * 9 + rc] = raw[hval(bi, rc, nb)];
    }
    int flag = 0;
    CK(d2h(h, &flag, h->status, sizeof(int)));
    if (flag & kFlagInverted) return fail(SORS_ERR_INVERTED, "Inverted Elements");
    return SORS_OK;
}

int sors_elem_eval(SorsHandle* h, const double* q, int32_t project, double* psi, double* grad, double* hess) {
    if (!h || !q) return fail(SORS_ERR_ARG, "NULL argument");
    int st;
    if ((st = set_device(h))) return st;
    const int n = 3 * h->nv;
    double *dpsi = nullptr, *dgrad = nullptr, *dhess = nullptr;
    auto cleanup = [&]() { cudaFree(dpsi); cudaFree(dgrad); cudaFree(dhess); };
    if (psi && cudaMalloc(&dpsi, sizeof(double) * std::max(1, h->E)) != cudaSuccess) { cleanup(); return fail(SORS_ERR_OOM, "alloc"); }
    if (grad && cudaMalloc(&dgrad, sizeof(double) * (size_t)std::max(1, h->E) * n) != cudaSuccess) { cleanup(); return fail(SORS_ERR_OOM, "alloc"); }
    if (hess && cudaMalloc(&dhess, sizeof(double) * (size_t)std::max(1, h->E) * n * n) != cudaSuccess) { cleanup(); return fail(SORS_ERR_OOM, "alloc"); }
    if ((st = dof_in(h, h->q, q, cudaMemcpyHostToDevice))) { cleanup(); return st; }
    cudaMemsetAsync(h->status, 0, sizeof(int), h->stream);
    if (mixed(h))
        launch_elem_rows<float>(h->E, h->nv, h->X, h->q, h->conn, h->mat, h->tshape, muscles(h), h->s.material, project, dpsi, dgrad, dhess,
                                h->status, h->stream);
    else
        launch_elem_rows<double>(h->E, h->nv, h->X, h->q, h->conn, h->mat, h->tshape, muscles(h), h->s.material, project, dpsi, dgrad, dhess,
                                 h->status, h->stream);
    cudaError_t e = cudaStreamSynchronize(h->stream);
    // per-element outputs in the caller's element order
    auto fetch = [&](double* dst, const double* src, size_t per) {
        if (!h->renum_e) return d2h(h, dst, src, sizeof(double) * (size_t)h->E * per);
        std::vector<double> tmp((size_t)h->E * per);
        cudaError_t r = d2h(h, tmp.data(), src, sizeof(double) * tmp.size());
        for (int el = 0; el < h->E && r == cudaSuccess; el++)
            memcpy(dst + (size_t)h->e2o[el] * per, tmp.data() + (size_t)el * per, sizeof(double) * per);
        return r;
    };
    if (e == cudaSuccess && psi) e = fetch(psi, dpsi, 1);
    if (e == cudaSuccess && grad) e = fetch(grad, dgrad, (size_t)n);
    if (e == cudaSuccess && hess) e = fetch(hess, dhess, (size_t)n * n);
    int flag = 0;
    if (e == cudaSuccess) e = d2h(h, &flag, h->status, sizeof(int));
    cleanup();
    if (e != cudaSuccess) return fail(SORS_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e));
    if (flag & kFlagInverted) return fail(SORS_ERR_INVERTED, "Inverted Elements");
    return SORS_OK;
}

int sors_set_plane_contact(SorsHandle* h, const double* points, const double* normals, int32_t n_planes,
                           const int32_t* surface_vertices, int32_t n_surface) {
    if (!h || (n_planes > 0 && (!points || !normals)) || (n_surface > 0 && !surface_vertices))
        return fail(SORS_ERR_ARG, "NULL argument");
    if (n_planes < 0 || n_surface < 0) return fail(SORS_ERR_ARG, "negative count");
    h->planes.clear();
    for (int k = 0; k < n_planes; k++) {
        SorsHandle::Plane P;
        for (int c = 0; c < 3; c++) { P.p[c] = points[3 * k + c]; P.n[c] = normals[3 * k + c]; }
        h->planes.push_back(P);
    }
    for (int i = 0; i < n_surface; i++)
        if (surface_vertices[i] < 0 || surface_vertices[i] >= h->N) return fail(SORS_ERR_ARG, "surface vertex out of range");
    h->plane_surf.resize(n_surface);
    for (int i = 0; i < n_surface; i++) h->plane_surf[i] = node_in(h, surface_vertices[i]);
    h->plane_mask.assign(n_surface, -1);
    return SORS_OK;
}

int sors_set_disk_contact(SorsHandle* h, const double* centers, const double* normals, const double* radii,
                          int32_t n_disks, const int32_t* surface_vertices, int32_t n_surface) {
    if (!h || (n_disks > 0 && (!centers || !normals || !radii)) || (n_surface > 0 && !surface_vertices))
        return fail(SORS_ERR_ARG, "NULL argument");
    if (n_disks < 0 || n_surface < 0) return fail(SORS_ERR_ARG, "negative count");
    h->disks.clear();
    for (int k = 0; k < n_disks; k++) {
        SorsHandle::Disk D;
        double nn = sqrt(normals[3 * k] * normals[3 * k] + normals[3 * k + 1] * normals[3 * k + 1] +
                         normals[3 * k + 2] * normals[3 * k + 2]);
        if (!(nn > 0)) return fail(SORS_ERR_ARG, "zero disk normal");
        for (int c = 0; c < 3; c++) { D.c[c] = centers[3 * k + c]; D.n[c] = normals[3 * k + c] / nn; }
        D.r = radii[k];
        h->disks.push_back(D);
    }
    for (int i = 0; i < n_surface; i++)
        if (surface_vertices[i] < 0 || surface_vertices[i] >= h->N) return fail(SORS_ERR_ARG, "surface vertex out of range");
    h->disk_groups.assign(1, SorsHandle::DiskGroup{});
    auto& G = h->disk_groups[0];
    for (int k = 0; k < n_disks; k++) G.disks.push_back(k);
    G.surf.resize(n_surface);
    for (int i = 0; i < n_surface; i++) G.surf[i] = node_in(h, surface_vertices[i]);
    G.mask.assign(n_surface, -1);
    return SORS_OK;
}

int sors_set_disk_contact_groups(SorsHandle* h, const double* centers, const double* normals, const double* radii,
                                 int32_t n_disks, const int32_t* surface_vertices, const int32_t* surface_ptr) {
    if (!h || !surface_ptr || (n_disks > 0 && (!centers || !normals || !radii))) return fail(SORS_ERR_ARG, "NULL argument");
    const int total = n_disks > 0 ? surface_ptr[n_disks] : 0;
    if (total > 0 && !surface_vertices) return fail(SORS_ERR_ARG, "NULL argument");
    for (int k = 0; k < n_disks; k++)
        if (surface_ptr[k] > surface_ptr[k + 1] || surface_ptr[k] < 0) return fail(SORS_ERR_ARG, "surface_ptr not monotone");
    int st = sors_set_disk_contact(h, centers, normals, radii, n_disks, surface_vertices, total);
    if (st) return st;
    h->disk_groups.assign(n_disks, SorsHandle::DiskGroup{});
    for (int k = 0; k < n_disks; k++) {
        auto& G = h->disk_groups[k];
        G.disks = {k};
        G.surf.clear();
        for (int i = surface_ptr[k]; i < surface_ptr[k + 1]; i++) G.surf.push_back(node_in(h, surface_vertices[i]));
        G.mask.assign(G.surf.size(), -1);
    }
    return SORS_OK;
}

int sors_set_disk(SorsHandle* h, int32_t disk_idx, const double* center, const double* normal, double radius) {
    if (!h || !center || !normal) return fail(SORS_ERR_ARG, "NULL argument");
    if (disk_idx < 0 || disk_idx >= (int)h->disks.size()) return fail(SORS_ERR_ARG, "diskIdx out of range in set_disk()");
    auto& D = h->disks[disk_idx];
    double nn = sqrt(normal[0] * normal[0] + normal[1] * normal[1] + normal[2] * normal[2]);
    if (!(nn > 0)) return fail(SORS_ERR_ARG, "zero disk normal");
    for (int c = 0; c < 3; c++) { D.c[c] = center[c]; D.n[c] = normal[c] / nn; }
    D.r = radius;
    return SORS_OK;
}

int sors_set_max_distance(SorsHandle* h, const int32_t* vertex1, const int32_t* vertex2, const double* max_distance,
                          int32_t n_pairs) {
    if (!h || (n_pairs > 0 && (!vertex1 || !vertex2 || !max_distance))) return fail(SORS_ERR_ARG, "NULL argument");
    if (n_pairs < 0) return fail(SORS_ERR_ARG, "negative count");
    for (int k = 0; k < n_pairs; k++)
        if (vertex1[k] < 0 || vertex1[k] >= h->N || vertex2[k] < 0 || vertex2[k] >= h->N)
            return fail(SORS_ERR_ARG, "max-distance vertex out of range");
    int st;
    if ((st = ensure_pair_buffers(h, n_pairs))) return st;
    h->md_i.resize(n_pairs);
    h->md_j.resize(n_pairs);
    for (int k = 0; k < n_pairs; k++) { h->md_i[k] = node_in(h, vertex1[k]); h->md_j[k] = node_in(h, vertex2[k]); }
    h->md_d.assign(max_distance, max_distance + n_pairs);
    h->md_work.assign(n_pairs, 0);
    h->held_pairs.clear();
    std::vector<int> nodes(2 * (size_t)n_pairs);
    for (int k = 0; k < n_pairs; k++) { nodes[2 * k] = h->md_i[k]; nodes[2 * k + 1] = h->md_j[k]; }
    if (n_pairs) CK(h2d(h, h->md_nodes_d, nodes.data(), sizeof(int) * nodes.size()));
    return SORS_OK;
}

int32_t sors_held_pairs(SorsHandle* h, int32_t* pairs, double* multipliers, int32_t cap) {
    if (!h) return 0;
    const int k = (int)h->held_pairs.size();
    for (int c = 0; c < k && c < cap; c++) {
        if (pairs) pairs[c] = h->held_pairs[c];
        if (multipliers) multipliers[c] = h->held_mu[c];
    }
    return k;
}

int sors_adjoint_set_pairs(SorsHandle* h, const int32_t* pairs, const double* multipliers, int32_t n) {
    if (!h || (n > 0 && (!pairs || !multipliers))) return fail(SORS_ERR_ARG, "NULL argument");
    if (n < 0) return fail(SORS_ERR_ARG, "negative count");
    for (int c = 0; c < n; c++)
        if (pairs[c] < 0 || pairs[c] >= (int)h->md_d.size()) return fail(SORS_ERR_ARG, "held pair out of range");
    h->adj_pairs.assign(pairs, pairs + n);
    h->adj_mu.assign(multipliers, multipliers + n);
    return SORS_OK;
}

int32_t sors_active_contacts(SorsHandle* h) { return h ? h->last_active : 0; }

int32_t sors_held_contacts(SorsHandle* h, int32_t* nodes, double* normals, int32_t cap) {
    if (!h) return 0;
    const int k = (int)h->held_nodes.size();
    for (int c = 0; c < k && c < cap; c++) {
        if (nodes) nodes[c] = node_out(h, h->held_nodes[c]);
        if (normals)
            for (int j = 0; j < 3; j++) normals[3 * c + j] = h->held_normals[3 * (size_t)c + j];
    }
    return k;
}

int32_t sors_get_contact_state(SorsHandle* h, int32_t* state, int32_t cap) {
    if (!h) return 0;
    int k = 0;
    for (const auto& G : h->disk_groups) k += 1 + (int)G.mask.size();
    if (state && cap >= k) {
        int o = 0;
        for (const auto& G : h->disk_groups) {
            state[o++] = G.frozen ? 1 : 0;
            for (int m : G.mask) state[o++] = m;
        }
    }
    return k;
}

int sors_set_contact_state(SorsHandle* h, const int32_t* state, int32_t n) {
    if (!h || (n > 0 && !state)) return fail(SORS_ERR_ARG, "NULL argument");
    int k = 0;
    for (const auto& G : h->disk_groups) k += 1 + (int)G.mask.size();
    if (n != k) return fail(SORS_ERR_ARG, "contact state size mismatch");
    int o = 0;
    for (auto& G : h->disk_groups) {
        G.frozen = state[o++] != 0;
        for (auto& m : G.mask) m = state[o++];
    }
    return SORS_OK;
}

int sors_set_material(SorsHandle* h, const double* youngs, const double* poisson) {
    if (!h || !youngs || !poisson) return fail(SORS_ERR_ARG, "NULL argument");
    int st;
    if ((st = set_device(h))) return st;
    std::vector<double2> mat((size_t)std::max(1, h->E));
    h->youngs_h.resize(h->E);
    h->poisson_h.resize(h->E);
    for (int e = 0; e < h->E; e++) {
        const int o = elem_out(h, e);
        mat[e] = lame_params(youngs[o], poisson[o], h->s.material);
        h->youngs_h[e] = youngs[o];
        h->poisson_h[e] = poisson[o];
    }
    if (h->E) CK(h2d(h, h->mat, mat.data(), sizeof(double2) * h->E));
    return SORS_OK;
}

int sors_adjoint_step(SorsHandle* h, const double* q_next, double dt, const double* dL_dq_next,
                      const int32_t* held_nodes, const double* held_normals, int32_t n_held, double* dL_dq_prev,
                      double* dL_dv_prev, double* dL_dyoungs, double* dL_dact, double* dL_dneumann,
                      SorsStepStats* stats) {
    if (!h || !q_next || !dL_dq_next) return fail(SORS_ERR_ARG, "NULL argument");
    if (n_held < 0 || (n_held > 0 && (!held_nodes || !held_normals))) return fail(SORS_ERR_ARG, "held contacts");
    int st;
    if ((st = set_device(h))) return st;
    if (dt == 0.0) dt = h->s.dt;
    if (h->s.time_stepping != 0 && dt != 0.0)
        return fail(SORS_ERR_UNSUPPORTED, "Crank-Nicolson steps are differentiated by sors_adjoint_step_cn");
    if (h->has_pressure && !h->adj_pairs.empty())
        return fail(SORS_ERR_UNSUPPORTED, "the adjoint does not combine pressure loads with held max-distance pairs");
    if (h->s.material == 1) return fail(SORS_ERR_UNSUPPORTED, "the adjoint is built for Neo-Hookean elements");
    if (stats) *stats = SorsStepStats{};
    if (!h->renum && !h->renum_e)
        return mixed(h) ? adjoint_impl<float, float>(h, q_next, dt, dL_dq_next, held_nodes, held_normals, n_held,
                                                     dL_dq_prev, dL_dv_prev, dL_dyoungs, dL_dact, dL_dneumann, stats)
                        : adjoint_impl<double, double>(h, q_next, dt, dL_dq_next, held_nodes, held_normals, n_held,
                                                       dL_dq_prev, dL_dv_prev, dL_dyoungs, dL_dact, dL_dneumann,
                                                       stats);
    // the handle's numbering inside, the caller's at the boundary
    const std::vector<double> qn = dofs_to_internal(h, q_next), bq = dofs_to_internal(h, dL_dq_next);
    std::vector<int32_t> hn(n_held);
    for (int c = 0; c < n_held; c++) hn[c] = node_in(h, held_nodes[c]);
    std::vector<double> oq(dL_dq_prev ? h->ndof : 0), ov(dL_dv_prev ? h->ndof : 0), on(dL_dneumann ? h->ndof : 0);
    std::vector<double> oe(dL_dyoungs ? h->E : 0);
    st = mixed(h) ? adjoint_impl<float, float>(h, qn.data(), dt, bq.data(), hn.data(), held_normals, n_held,
                                               dL_dq_prev ? oq.data() : nullptr, dL_dv_prev ? ov.data() : nullptr,
                                               dL_dyoungs ? oe.data() : nullptr, dL_dact,
                                               dL_dneumann ? on.data() : nullptr, stats)
                  : adjoint_impl<double, double>(h, qn.data(), dt, bq.data(), hn.data(), held_normals, n_held,
                                                 dL_dq_prev ? oq.data() : nullptr, dL_dv_prev ? ov.data() : nullptr,
                                                 dL_dyoungs ? oe.data() : nullptr, dL_dact,
                                                 dL_dneumann ? on.data() : nullptr, stats);
    if (st) return st;
    if (dL_dyoungs)
        for (int e = 0; e < h->E; e++) dL_dyoungs[elem_out(h, e)] = oe[e];
    if (dL_dq_prev) dofs_to_caller(h, oq.data(), dL_dq_prev);
    if (dL_dv_prev) dofs_to_caller(h, ov.data(), dL_dv_prev);
    if (dL_dneumann) dofs_to_caller(h, on.data(), dL_dneumann);
    return SORS_OK;
}

int sors_adjoint_step_cn(SorsHandle* h, const double* q_next, double dt, const double* dL_dq_next,
                         const double* dL_dgprev_next, const int32_t* held_nodes, const double* held_normals,
                         int32_t n_held, double* dL_dq_prev, double* dL_dv_prev, double* dL_dgprev_prev,
                         double* dL_dyoungs, double* dL_dact, double* dL_dneumann, SorsStepStats* stats) {
    if (!h || !q_next || !dL_dq_next) return fail(SORS_ERR_ARG, "NULL argument");
    if (n_held < 0 || (n_held > 0 && (!held_nodes || !held_normals))) return fail(SORS_ERR_ARG, "held contacts");
    int st;
    if ((st = set_device(h))) return st;
    if (dt == 0.0) dt = h->s.dt;
    if (h->s.time_stepping != 1 || dt == 0.0)
        return fail(SORS_ERR_ARG, "sors_adjoint_step_cn differentiates Crank-Nicolson steps (dt > 0)");
    if (h->has_pressure || !h->adj_pairs.empty() || h->s.material == 1)
        return fail(SORS_ERR_UNSUPPORTED,
                    "the Crank-Nicolson adjoint is built for Neo-Hookean elements without pressure loads or held pairs");
    if (stats) *stats = SorsStepStats{};
    const int n = h->ndof;
    const std::vector<double> qn = dofs_to_internal(h, q_next), bq = dofs_to_internal(h, dL_dq_next);
    std::vector<double> bgi;
    // (every output is computed in the handle's numbering, then converted)
    if (dL_dgprev_next) bgi = dofs_to_internal(h, dL_dgprev_next);
    std::vector<int32_t> hn(n_held);
    for (int c = 0; c < n_held; c++) hn[c] = node_in(h, held_nodes[c]);
    std::vector<double> oq(n), ov(n), og(n), on(n), oe(h->E);
    st = mixed(h) ? adjoint_impl<float, float>(h, qn.data(), dt, bq.data(), hn.data(), held_normals, n_held,
                                               oq.data(), ov.data(), oe.data(), dL_dact, on.data(), stats,
                                               bgi.empty() ? nullptr : bgi.data(), og.data())
                  : adjoint_impl<double, double>(h, qn.data(), dt, bq.data(), hn.data(), held_normals, n_held,
                                                 oq.data(), ov.data(), oe.data(), dL_dact, on.data(), stats,
                                                 bgi.empty() ? nullptr : bgi.data(), og.data());
    if (st) return st;
    if (dL_dyoungs)
        for (int e = 0; e < h->E; e++) dL_dyoungs[elem_out(h, e)] = oe[e];
    if (dL_dq_prev) dofs_to_caller(h, oq.data(), dL_dq_prev);
    if (dL_dv_prev) dofs_to_caller(h, ov.data(), dL_dv_prev);
    if (dL_dgprev_prev) dofs_to_caller(h, og.data(), dL_dgprev_prev);
    if (dL_dneumann) dofs_to_caller(h, on.data(), dL_dneumann);
    return SORS_OK;
}

int sors_get_prev_force(SorsHandle* h, double* g_prev) {
    if (!h || !g_prev) return fail(SORS_ERR_ARG, "NULL argument");
    int st;
    if ((st = set_device(h))) return st;
    if ((st = dof_out(h, g_prev, h->gPrev, cudaMemcpyDeviceToHost))) return st;
    CK(cudaStreamSynchronize(h->stream));
    return SORS_OK;
}

int sors_set_prev_force(SorsHandle* h, const double* g_prev) {
    if (!h || !g_prev) return fail(SORS_ERR_ARG, "NULL argument");
    int st;
    if ((st = set_device(h))) return st;
    if ((st = dof_in(h, h->gPrev, g_prev, cudaMemcpyHostToDevice))) return st;
    CK(cudaStreamSynchronize(h->stream));
    return SORS_OK;
}

int sors_adjoint_pressure_grad(SorsHandle* h, double* dL_dpressure, int32_t n_groups) {
    if (!h || !dL_dpressure) return fail(SORS_ERR_ARG, "NULL argument");
    if (!h->has_pressure || n_groups != h->n_groups)
        return fail(SORS_ERR_ARG, "n_groups must equal the number of pressure groups");
    if (!h->adj_ready) return fail(SORS_ERR_ARG, "no adjoint step to differentiate");
    int st;
    if ((st = set_device(h))) return st;
    const int n = h->ndof;
    if (!h->adj_pg && (st = dalloc_t(h, &h->adj_pg, (size_t)std::max(1, n_groups)))) return st;
    std::vector<double> lam(n), f(n), e(n_groups);
    CK(d2h(h, lam.data(), h->adj_l, sizeof(double) * n));
    // dL/dp_g = -lam . dg/dp_g = lam . f_g, f_g the follower load of group g at unit pressure
    for (int g = 0; g < n_groups; g++) {
        std::fill(e.begin(), e.end(), 0.0);
        e[g] = 1.0;
        CK(h2d(h, h->adj_pg, e.data(), sizeof(double) * n_groups));
        CK(cudaMemsetAsync(h->adj_y, 0, sizeof(double) * n, h->stream));
        PressureArgs p = pressure_args(h);
        p.pressure = h->adj_pg;
        p.q = h->adj_q;
        p.f_ext = h->adj_y;
        launch_pressure_force(p, h->stream);
        CK(cudaGetLastError());
        CK(d2h(h, f.data(), h->adj_y, sizeof(double) * n));
        double acc = 0.0;
        for (int i = 0; i < n; i++) acc += lam[i] * f[i];
        dL_dpressure[g] = acc;
    }
    return SORS_OK;
}

int sors_step(SorsHandle* h, const double* q_in, double* q_out, double dt, int32_t substeps, SorsStepStats* stats) {
    if (!h || !q_in || !q_out) return fail(SORS_ERR_ARG, "NULL argument");
    int st;
    if ((st = set_device(h))) return st;
    if ((st = dof_in(h, h->q, q_in, cudaMemcpyHostToDevice))) return st;
    st = step_resident(h, dt, substeps, stats);
    if (st) return st;
    if ((st = dof_out(h, q_out, h->q, cudaMemcpyDeviceToHost))) return st;
    CK(cudaStreamSynchronize(h->stream));
    return SORS_OK;
}

int sors_step_device(SorsHandle* h, double* q_device, double dt, int32_t substeps, SorsStepStats* stats) {
    if (!h || !q_device) return fail(SORS_ERR_ARG, "NULL argument");
    int st;
    if ((st = set_device(h))) return st;
    if ((st = dof_in(h, h->q, q_device, cudaMemcpyDeviceToDevice))) return st;
    st = step_resident(h, dt, substeps, stats);
    if (st) return st;
    if ((st = dof_out(h, q_device, h->q, cudaMemcpyDeviceToDevice))) return st;
    CK(cudaStreamSynchronize(h->stream));
    return SORS_OK;
}

int sors_update_state(SorsHandle* h, const double* q, double dt) {
    if (!h || !q) return fail(SORS_ERR_ARG, "NULL argument");
    int st;
    if ((st = set_device(h))) return st;
    if ((st = dof_in(h, h->q, q, cudaMemcpyHostToDevice))) return st;
    launch_update_state(h->ndof, h->q, h->qPrev, h->vPrev, h->gPrev, h->gPrevTmp, dt, h->s.time_stepping, h->stream);
    CK(cudaStreamSynchronize(h->stream));
    return SORS_OK;
}

int64_t sors_device_bytes(const SorsHandle* h) { return h ? (int64_t)h->bytes : 0; }

int sors_sizes(const SorsHandle* h, int64_t* n_nodes, int64_t* n_elems, int64_t* nnzb) {
    if (!h) return fail(SORS_ERR_ARG, "NULL handle");
    if (n_nodes) *n_nodes = h->N;
    if (n_elems) *n_elems = h->E;
    if (nnzb) *nnzb = h->nnzb;
    return SORS_OK;
}

void* sors_stream(SorsHandle* h) { return h ? (void*)h->stream : nullptr; }

int64_t sors_kernel_launch_count(void) { return (int64_t)g_kernel_launches.load(); }

int sors_set_assembly_variant(SorsHandle* h, int32_t variant) {
    if (!h) return fail(SORS_ERR_ARG, "NULL handle");
    if (variant < 0 || variant > 2) return fail(SORS_ERR_ARG, "assembly variant must be 0, 1 or 2");
    if (variant == 2 && h->chunks.nchunks > 0 && !h->chunk_gen) {
        int st;
        if ((st = set_device(h))) return st;
        const size_t rec = h->s.material == 2 ? 40 : 28;  // generator fields padded to 16 bytes
        if ((st = dalloc(h, &h->chunk_gen, (size_t)h->E * rec * hsize(h)))) return st;
        if ((st = dalloc_t(h, &h->chunk_gradg, (size_t)h->E * 12))) return st;
    }
    h->asm_variant = variant;
    return SORS_OK;
}

int64_t sors_assembly_chunks(SorsHandle* h) { return h ? (int64_t)h->chunks.nchunks : 0; }

int sors_set_members(SorsHandle* h, const int32_t* node_offsets, int32_t n_members) {
    if (!h || (n_members > 0 && !node_offsets)) return fail(SORS_ERR_ARG, "NULL argument");
    int st;
    if ((st = set_device(h))) return st;
    if (n_members <= 1) {
        h->batch.nmem = 0;
        return SORS_OK;
    }
    if (node_offsets[0] != 0 || node_offsets[n_members] != h->N)
        return fail(SORS_ERR_ARG, "member node offsets must run from 0 to the node count");
    for (int k = 0; k < n_members; k++)
        if (node_offsets[k + 1] <= node_offsets[k]) return fail(SORS_ERR_ARG, "member node offsets must increase");
    // the handle orders nodes by connected component (lowest caller index
    // first), so independent meshes keep their caller node ranges
    if (h->renum)
        for (int k = 0; k < n_members; k++)
            for (int i = node_offsets[k]; i < node_offsets[k + 1]; i++)
                if (h->n2o[i] < node_offsets[k] || h->n2o[i] >= node_offsets[k + 1])
                    return fail(SORS_ERR_ARG, "an element joins two members");
    // no element may couple two members
    std::vector<int> conn((size_t)h->E * h->nv);
    if (!conn.empty()) CK(d2h(h, conn.data(), h->conn, sizeof(int) * conn.size()));
    std::vector<int> mem_of(h->N);
    for (int k = 0; k < n_members; k++)
        for (int i = node_offsets[k]; i < node_offsets[k + 1]; i++) mem_of[i] = k;
    for (int e = 0; e < h->E; e++)
        for (int v = 1; v < h->nv; v++)
            if (mem_of[conn[(size_t)e * h->nv + v]] != mem_of[conn[(size_t)e * h->nv]])
                return fail(SORS_ERR_ARG, "an element joins two members");
    std::vector<int> blk0(n_members + 1, 0), blk_mem;
    for (int k = 0; k < n_members; k++) {
        const int nb = (node_offsets[k + 1] - node_offsets[k] + kBatchThreads - 1) / kBatchThreads;
        blk0[k + 1] = blk0[k] + nb;
        for (int b = 0; b < nb; b++) blk_mem.push_back(k);
    }
    BatchArgs& b = h->batch;
    int *d_node0 = nullptr, *d_blk0 = nullptr, *d_blkmem = nullptr;
    if ((st = upload(h, &d_node0, node_offsets, (size_t)n_members + 1))) return st;
    if ((st = upload(h, &d_blk0, blk0.data(), blk0.size()))) return st;
    if ((st = upload(h, &d_blkmem, blk_mem.data(), blk_mem.size()))) return st;
    MemberScalars* d_ms = nullptr;
    double* d_part = nullptr;
    if ((st = dalloc_t(h, &d_ms, (size_t)n_members))) return st;
    CK(dzero(h, d_ms, sizeof(MemberScalars) * n_members));
    if ((st = dalloc_t(h, &d_part, (size_t)2 * blk_mem.size()))) return st;
    b.mem_node0 = d_node0; b.mem_blk0 = d_blk0; b.blk_mem = d_blkmem; b.ms = d_ms; b.partials = d_part;
    b.nblocks = (int)blk_mem.size();
    b.nmem = n_members;
    b.max_row_blocks = h->max_row_blocks;
    h->mem_node0_h.assign(node_offsets, node_offsets + n_members + 1);
    h->ms_h.assign(n_members, MemberScalars{});
    CK(cudaStreamSynchronize(h->stream));
    return SORS_OK;
}

int sors_last_step_curvature(SorsHandle* h, double* min_rayleigh, int32_t* indefinite_solves) {
    if (!h || !min_rayleigh || !indefinite_solves) return fail(SORS_ERR_ARG, "NULL argument");
    *min_rayleigh = h->step_min_rq;
    *indefinite_solves = h->step_indefinite;
    return SORS_OK;
}

int64_t sors_evaluation_count(SorsHandle* h, int32_t with_hessian) {
    if (!h) return 0;
    return with_hessian ? h->n_hess_evals : h->n_grad_evals;
}

}  // extern "C"

namespace {
template <typename HT, typename VT>
int profile_impl(SorsHandle* h, int iters, SorsKernelProfile* out) {
    const size_t hs = sizeof(HT), vs = sizeof(VT);
    const double N = h->N, E = h->E, nnzb = (double)h->nnzb, nv = h->nv;
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    float ms = 0.f;
    const double dt = h->s.dt;
    // assembly of gradient rows + Hessian block-rows at the current iterate
    int st = eval_system<HT>(h, dt, true);
    if (st) return st;
    // as a step assembles (the adaptive projection's first try is the exact Hessian)
    AsmArgs<HT> aa = asm_args<HT>(h, dt, true, kAsmStep, h->s.project_spd == 1);
    CK(cudaEventRecord(a, h->stream));
    for (int i = 0; i < iters; i++) launch_assemble<HT>(aa, h->max_pairs, h->stream);
    CK(cudaEventRecord(b, h->stream));
    CK(cudaEventSynchronize(b));
    CK(cudaEventElapsedTime(&ms, a, b));
    out->assemble_ms = ms / iters;
    {
        AsmArgs<HT> ag = aa;
        ag.want_hess = 0;
        CK(cudaEventRecord(a, h->stream));
        for (int i = 0; i < iters; i++) launch_assemble<HT>(ag, h->max_pairs, h->stream);
        CK(cudaEventRecord(b, h->stream));
        CK(cudaEventSynchronize(b));
        CK(cudaEventElapsedTime(&ms, a, b));
        out->assemble_grad_ms = ms / iters;
    }
    if (aa.ch.nchunks > 0 && nv == 4 && !aa.project && !aa.mus.group) {
        // chunked element-owner kernel, each compulsory input and output once:
        // conn, shape gradients + volume, (mu, lambda); q, mask, mass; chunk rows
        // and element lists with their owned-vertex slots; pair counts, pattern
        // and slot items; H and gradient out
        const double ch_elems = (double)h->chunk_elem_total;
        out->assemble_bytes = E * (16 + 80 + 16) + N * (24 + 1 + 8) + (N + 4 * (double)h->chunks.nchunks) * 4 +
                              ch_elems * (4 + 8) + (N + 1) * 4 * 2 + (nnzb + 1) * 4 + nnzb * 4 + E * nv * nv * 2 +
                              nnzb * 9 * hs + N * 24;
    } else {
        // compulsory bytes: conn, (mu,lambda), X, q, mask, mass, pair lists, slot maps, pattern; H and gradient out
        out->assemble_bytes = E * nv * 4 + E * 16 + N * 24 * 2 + N * 1 + N * 8 + (N + 1) * 4 + E * nv * 4 +
                              (nnzb + 1) * 4 + E * nv * nv * 2 + (N + 1) * 4 + nnzb * 4 + nnzb * 9 * hs + N * 24;
    }
    // PCG kernels on the assembled system, on nonzero vectors (p = r = 1) so
    // that no launch meets a zero curvature or a converged residual and exits early
    launch_block_jacobi<HT, VT>(h->N, h->row_ptr, h->diag_slot, (const HT*)h->H, h->nnzb, (VT*)h->Minv, h->stream);
    launch_pcg_init<HT, VT>(h->N, h->g, (const VT*)h->Minv, (VT*)h->x, (VT*)h->r, (VT*)h->z, (VT*)h->p0, 0.0, 0.0,
                            1 << 30, nullptr, nullptr, h->partials, h->sc, h->stream);
    {
        std::vector<VT> ones(4 * (size_t)h->N, VT(1));
        for (size_t i = 3; i < ones.size(); i += 4) ones[i] = VT(0);
        CK(cudaMemcpyAsync(h->p0, ones.data(), sizeof(VT) * ones.size(), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(h->p1, ones.data(), sizeof(VT) * ones.size(), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(h->r, ones.data(), sizeof(VT) * 3 * (size_t)h->N, cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(h->z, ones.data(), sizeof(VT) * 3 * (size_t)h->N, cudaMemcpyHostToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    CK(cudaMemsetAsync(&h->sc->done, 0, sizeof(int), h->stream));
    CK(cudaEventRecord(a, h->stream));
    for (int i = 0; i < iters; i++)
        launch_pcg_spmv<HT, VT>(h->N, h->max_row_blocks, h->row_ptr, h->col, (const HT*)h->H, h->nnzb, (VT*)h->p1,
                                (VT*)h->qv, h->partials, h->sc, h->stream);
    CK(cudaEventRecord(b, h->stream));
    CK(cudaEventSynchronize(b));
    CK(cudaEventElapsedTime(&ms, a, b));
    out->spmv_ms = ms / iters;
    // values + block columns + row pointers + p (padded, read) + q (written)
    out->spmv_bytes = nnzb * 9 * hs + nnzb * 4 + (N + 1) * 4 + 4 * N * vs + 3 * N * vs;
    CK(cudaMemsetAsync(&h->sc->done, 0, sizeof(int), h->stream));
    CK(cudaEventRecord(a, h->stream));
    for (int i = 0; i < iters; i++)
        launch_form_p<VT>(h->N, (VT*)h->z, (VT*)(i & 1 ? h->p1 : h->p0), (VT*)(i & 1 ? h->p0 : h->p1), h->sc,
                          h->stream);
    CK(cudaEventRecord(b, h->stream));
    CK(cudaEventSynchronize(b));
    CK(cudaEventElapsedTime(&ms, a, b));
    out->form_p_ms = ms / iters;
    // z and p_old read, p_new written (padded)
    out->form_p_bytes = 3 * N * vs + 8 * N * vs;
    CK(cudaMemsetAsync(&h->sc->done, 0, sizeof(int), h->stream));
    CK(cudaEventRecord(a, h->stream));
    for (int i = 0; i < iters; i++)
        launch_pcg_update<VT>(h->N, (VT*)h->p1, (VT*)h->qv, (VT*)h->Minv, (VT*)h->x, (VT*)h->r, (VT*)h->z,
                              nullptr, nullptr, h->partials, h->sc, h->stream);
    CK(cudaEventRecord(b, h->stream));
    CK(cudaEventSynchronize(b));
    CK(cudaEventElapsedTime(&ms, a, b));
    out->pcg_update_ms = ms / iters;
    // p, q, Minv read; x, r read+written; z written
    out->pcg_update_bytes = 3 * N * vs * 2 + 9 * N * vs + 3 * N * vs * 4 + 3 * N * vs;
    if (h->cargs.nc > 0) {
        // two-level iteration kernels (their values are not used: timing only)
        CK(cudaMemsetAsync(&h->sc->done, 0, sizeof(int), h->stream));
        CK(cudaEventRecord(a, h->stream));
        for (int i = 0; i < iters; i++) {
            if (h->cruns.nruns > 0)
                launch_tl_update_restrict_runs<VT>(h->cargs, h->cruns, (VT*)h->p1, (VT*)h->qv, (VT*)h->x,
                                                   (VT*)h->r, nullptr, nullptr, h->tl_yc, h->sc, h->stream);
            else
                launch_tl_update_restrict<VT>(h->cargs, (VT*)h->p1, (VT*)h->qv, (VT*)h->x, (VT*)h->r, nullptr,
                                              nullptr, h->tl_yc, h->sc, h->stream);
        }
        CK(cudaEventRecord(b, h->stream));
        CK(cudaEventSynchronize(b));
        CK(cudaEventElapsedTime(&ms, a, b));
        out->tl_restrict_ms = ms / iters;
        // p, q, x, r read; x, r written; offsets (16 B) and the node list or
        // the aggregate id (4 B) per node
        out->tl_restrict_bytes = 18 * N * vs + 20 * N;
        CK(cudaMemsetAsync(&h->sc->done, 0, sizeof(int), h->stream));
        CK(cudaEventRecord(a, h->stream));
        for (int i = 0; i < iters; i++)
            launch_tl_coarse_z<VT>(h->cargs, h->tl_ld, (const VT*)h->tl_Ainv, h->tl_yc, (VT*)h->r, (const VT*)h->Minv,
                                   (VT*)h->z, 1, nullptr, nullptr, h->partials, h->sc, h->stream);
        CK(cudaEventRecord(b, h->stream));
        CK(cudaEventSynchronize(b));
        CK(cudaEventElapsedTime(&ms, a, b));
        out->tl_coarse_z_ms = ms / iters;
        // the coarse inverse once, r and Minv read, z written, offsets and node list
        out->tl_coarse_z_bytes = (double)h->cargs.nc * h->tl_ld * vs + 15 * N * vs + 20 * N;
    }
    CK(cudaEventRecord(a, h->stream));
    for (int i = 0; i < iters; i++)
        launch_elem_energy(h->E, h->nv, h->X, h->q, h->conn, h->mat, muscles(h), h->s.material, h->partials, h->sc, h->stream);
    CK(cudaEventRecord(b, h->stream));
    CK(cudaEventSynchronize(b));
    CK(cudaEventElapsedTime(&ms, a, b));
    out->energy_ms = ms / iters;
    out->energy_bytes = E * nv * 4 + E * 16 + N * 48;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    CK(cudaGetLastError());
    return SORS_OK;
}
}  // namespace

extern "C" {

int sors_profile_kernels(SorsHandle* h, int32_t iters, SorsKernelProfile* out) {
    if (!h || !out || iters <= 0) return fail(SORS_ERR_ARG, "bad argument");
    int st;
    if ((st = set_device(h))) return st;
    memset(out, 0, sizeof(*out));
    return mixed(h) ? profile_impl<float, float>(h, iters, out) : profile_impl<double, double>(h, iters, out);
}

}  // extern "C"
