// Host orchestration of the engine behind the C ABI (include/fmmx.h).
//
// fmmx_build   = Fmm::new / refresh (fmm.rs:26-56): bounding box, Morton keys,
//                key sort, level-by-level node creation, depth-first
//                renumbering, body gather, cell geometry.
// fmmx_evaluate = Fmm::run (fmm.rs:60-142): gather, f pre-pass, P2M/M2M and
//                multipole power, dual walk, directed lists, M2L, L2L, P2P,
//                L2P + scatter.
//
// All work runs on one stream; the host waits on it only where a size must be
// known (node count after the build, list lengths after the walk).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "kernels.h"
#include "rotw.h"
#include "sort.h"

using namespace fmmx;

namespace {

// Device-memory budget of a context (fmmx_config.device_budget_bytes): every
// engine buffer is charged to it, and the allocation that would take the
// context above it fails with FMMX_OVER_BUDGET, naming the buffer, the bytes
// it needs and the limit (the reference's GPU OverBudget error,
// crates/visual/src/gpufmm.rs:1653-1672, after which its callers fall back).
struct Budget {
    uint64_t limit = 0;  // bytes; 0: no limit
    uint64_t used = 0;
    bool over = false;   // the last refusal, until reported
    uint64_t asked = 0;
};
// the budget of the context whose API call runs on this thread
thread_local Budget* tl_budget = nullptr;

// Every device buffer of a context registers itself while the context is
// constructed, so that the context can drop all of them (a cache: the next
// call reallocates) after a call fails over its budget.
struct DBufBase {
    DBufBase();
    virtual ~DBufBase() = default;
    virtual void release() = 0;
};
thread_local std::vector<DBufBase*>* tl_registry = nullptr;
DBufBase::DBufBase() {
    if (tl_registry) tl_registry->push_back(this);
}

template <class T>
struct DBuf : DBufBase {
    T* p = nullptr;
    size_t cap = 0;
    Budget* bud = nullptr;  // charged for this buffer
    ~DBuf() override { release(); }
    void release() override {
        if (p) {
            cudaFree(p);
            if (bud) bud->used -= cap * sizeof(T);
        }
        p = nullptr;
        cap = 0;
        bud = nullptr;
    }
    // Grows by at least half of the current capacity, so a context that sees
    // slowly growing inputs (a serving loop's forests) reallocates -- and
    // cudaFree synchronises the device -- only a logarithmic number of times;
    // a first allocation carries 1/8 slack, so that sizes which drift up a
    // little between calls (a leapfrog's interaction lists) do not reallocate
    // at the first step (cudaMalloc of a large buffer took over a second at
    // times on a busy device).
    cudaError_t ensure(size_t n) {
        if (n <= cap && p) return cudaSuccess;
        const size_t grown = cap + cap / 2;
        size_t want = std::max<size_t>(std::max<size_t>(n + n / 8, grown), 1);
        Budget* b = tl_budget;
        if (b && b->limit) {
            const uint64_t base = b->used - (p && bud == b ? cap * sizeof(T) : 0);
            if (base + want * sizeof(T) > b->limit) want = std::max<size_t>(n, 1);  // no slack
            if (base + want * sizeof(T) > b->limit) {
                b->over = true;
                b->asked = want * sizeof(T);
                return cudaErrorMemoryAllocation;
            }
        }
        release();
        cudaError_t e = cudaMalloc((void**)&p, want * sizeof(T));
        if (e != cudaSuccess && want > n) {  // no room for the slack: exactly n
            cudaGetLastError();
            want = std::max<size_t>(n, 1);
            e = cudaMalloc((void**)&p, want * sizeof(T));
        }
        if (e != cudaSuccess) {
            p = nullptr;
            cudaGetLastError();
            return e;
        }
        cap = want;
        bud = b;
        if (bud) bud->used += cap * sizeof(T);
        return cudaSuccess;
    }
};

// charges the allocations of one API call to its context's budget
struct BudgetScope {
    Budget* prev;
    explicit BudgetScope(Budget* b) : prev(tl_budget) { tl_budget = b; }
    ~BudgetScope() { tl_budget = prev; }
};

int rot_moff_host(int k) { return 4 * (k * (k + 1) * (2 * k + 1) / 6); }

int bits_for(uint64_t v) {
    int b = 0;
    while (b < 64 && (v >> b) != 0) ++b;
    return std::max(b, 1);
}

struct Status {
    fmmx_status code = FMMX_OK;
    std::string msg;
};

}  // namespace

struct fmmx_ctx {
    Budget budget;  // first: outlives every buffer charged to it
    fmmx_config cfg;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string err;

    OrderTables tab;
    std::vector<double> swap_host;
    DBuf<double> swap_dev;

    // sizes of the current tree; a forest of nsys independent systems
    size_t n = 0;
    int nsys = 1;
    DBuf<uint64_t> sys_off;  // nsys + 1 offsets into the inputs
    std::vector<uint64_t> sys_off_host;
    int steps_since_build = 0;
    DBuf<double> c_h;        // box size of every cell
    int nc = 0, nleaves = 0, nlevels = 0;
    int lvl_start[FMMX_NLEVELS + 1] = {0}, lvl_count[FMMX_NLEVELS + 1] = {0};
    bool built = false, evaluated = false, lists_valid = false;
    // leapfrog steps on a reused tree, recorded once per tree as a CUDA graph
    cudaGraphExec_t step_graph = nullptr;
    const void* graph_key[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    double graph_dt = 0.0;
    int graph_scheme = -1;
    void drop_graph() {
        if (step_graph) cudaGraphExecDestroy(step_graph);
        step_graph = nullptr;
    }
    std::vector<DBufBase*> cache;  // every buffer but the constant tables
    int n_m2l = 0, n_p2p = 0;
    unsigned long long pops = 0, p2p_inter = 0;

    // inputs (host API copies) and outputs
    DBuf<double> pos_in, mass_in, acc_out, pot_out;
    const double* build_pos = nullptr;  // device pointers of the last build's inputs
    const double* build_mass = nullptr;

    DBuf<double> box, bbox_part;
    DBuf<int> flags;
    DBuf<uint64_t> keys, keys_sorted;
    DBuf<uint32_t> idx, order;
    DBuf<double> x, y, z, m, nax, nay, naz, npot;
    DBuf<char> cub_tmp;

    // nodes before renumbering
    DBuf<uint32_t> t_first, t_count;
    DBuf<int32_t> t_parent;
    DBuf<uint8_t> t_oct, t_level, t_leaf;
    uint32_t tcap = 0;
    DBuf<int> lvl;
    DBuf<uint64_t> dfs_key, dfs_key_alt;
    DBuf<uint32_t> dfs_val, dfs_val_alt;
    DBuf<int32_t> new_id;

    // cells (depth-first pre-order)
    DBuf<uint32_t> c_first, c_count;
    DBuf<int32_t> c_child, c_parent, level_cells, body_leaf;
    DBuf<uint8_t> c_leaf, c_level;
    DBuf<double> c_cx, c_cy, c_cz, c_mass, c_rho;
    DBuf<double4> c_geo;  // (cx, cy, cz, rho) per cell

    // expansions
    DBuf<zd> moments, locals;
    DBuf<double> pows, f, fmin;
    // mixed form: normalised FP32 half-layout expansions and the per-cell length
    DBuf<zf> mom_f, loc_f;
    DBuf<double> ell;
    DBuf<unsigned long long> rho_now;  // radii about the build's centres on a reused tree (FP64 bits)
    DBuf<float> ellf;

    // walk
    DBuf<uint2> front0, front1, m2l, p2p;
    DBuf<int> wcounts;
    DBuf<unsigned long long> wpops, inter;
    uint32_t cap_front = 0, cap_m2l = 0, cap_p2p = 0;
    uint64_t walk_cap0 = 0;  // FMMX_TEST_WALK_CAPACITY (tests of the overflow retry); 0: sized by the tree
    int walk_retries = 0;

    // directed lists
    // per destination cell c: sources src[off[c] .. off[c+1]), ascending
    DBuf<uint32_t> m2l_src_u, m2l_src, p2p_src_u, p2p_src;  // scattered, then sorted within segments
    DBuf<uint32_t> m2l_off, p2p_off, list_cnt;               // nc + 1 each
    DBuf<int> m2l_longs, p2p_longs;                         // long-segment lists, 2 nc + 128 each
    DBuf<uint32_t> long_bounds;
    DBuf<char> cub_tmp2;                // the M2L list's sort scratch (built beside the P2P)
    DBuf<uint32_t> list_cnt2, long_bounds2;
    // near-field work units of the mixed P2P (per leaf: units, scratch bodies)
    DBuf<uint32_t> p2p_units, p2p_scr, p2p_uoff, p2p_soff;
    DBuf<uint32_t> p2p_units_s, p2p_units_b, p2p_uoff_s, p2p_uoff_b;  // small-leaf units apart
    DBuf<double4> p2p_part;
    DBuf<float4> body_loc;  // mixed near field: bodies relative to their leaf's centre, FP32, with the mass
    DBuf<unsigned> p2p_next;

    DBuf<int> work;  // persistent-kernel work counter
    int nsm = 148;
    int walk_blocks[2] = {0, 0};  // resident blocks of k_walk_iter<theta, Dehnen> on the whole device
    uint64_t launches = 0, launches_build = 0;

    fmmx_stats st;
    cudaEvent_t ev[16];
    // second stream: the walk and the lists run beside the upward pass, the
    // P2P beside the M2L and L2L; fork/join events order the two
    cudaStream_t stream2 = nullptr;
    cudaEvent_t fork[3] = {nullptr, nullptr, nullptr};
    bool events = false;
};

namespace {

fmmx_status fail(fmmx_ctx* c, fmmx_status s, const std::string& msg) {
    c->err = msg;
    return s;
}

fmmx_status cuda_fail(fmmx_ctx* c, cudaError_t e, const char* where) {
    if (e == cudaErrorMemoryAllocation && c->budget.over) {
        c->budget.over = false;
        char buf[256];
        std::snprintf(buf, sizeof(buf), "%s needs %.1f MiB, device budget %.1f MiB (%.1f MiB in use)", where,
                      c->budget.asked / 1048576.0, c->budget.limit / 1048576.0, c->budget.used / 1048576.0);
        return fail(c, FMMX_OVER_BUDGET, buf);
    }
    std::string m = std::string(where) + ": " + cudaGetErrorString(e);
    cudaGetLastError();
    if (e == cudaErrorMemoryAllocation) return fail(c, FMMX_OUT_OF_MEMORY, m);
    return fail(c, FMMX_DEVICE_ERROR, m);
}

// A call that failed over the budget leaves the context with whatever its
// buffers had grown to: drop them all (the next call reallocates what it
// needs), so that a smaller system fits again.
fmmx_status finish(fmmx_ctx* ctx, fmmx_status st) {
    if (st != FMMX_OVER_BUDGET) return st;
    cudaStreamSynchronize(ctx->stream);
    if (ctx->stream2) cudaStreamSynchronize(ctx->stream2);
    cudaGetLastError();
    ctx->drop_graph();
    for (DBufBase* b : ctx->cache) b->release();
    ctx->built = ctx->evaluated = ctx->lists_valid = false;
    ctx->cap_front = ctx->cap_m2l = ctx->cap_p2p = 0;
    ctx->tcap = 0;
    return st;
}

#define CK(expr, where)                                   \
    do {                                                  \
        cudaError_t e__ = (expr);                         \
        if (e__ != cudaSuccess) return cuda_fail(ctx, e__, where); \
    } while (0)

#define CKL(where) CK(cudaGetLastError(), where)
// kernel launches of the current build/evaluate (reported in fmmx_stats)
#define LCOUNT(k) (ctx->launches += (k))

CellsView view(fmmx_ctx* c) {
    CellsView v;
    v.first = c->c_first.p;
    v.count = c->c_count.p;
    v.child = c->c_child.p;
    v.leaf = c->c_leaf.p;
    v.level = c->c_level.p;
    v.cx = c->c_cx.p;
    v.cy = c->c_cy.p;
    v.cz = c->c_cz.p;
    v.mass = c->c_mass.p;
    v.rho = c->c_rho.p;
    v.geo = c->c_geo.p;
    return v;
}

CellsMut view_mut(fmmx_ctx* c) {
    CellsMut v;
    v.first = c->c_first.p;
    v.count = c->c_count.p;
    v.child = c->c_child.p;
    v.parent = c->c_parent.p;
    v.leaf = c->c_leaf.p;
    v.level = c->c_level.p;
    v.cx = c->c_cx.p;
    v.cy = c->c_cy.p;
    v.cz = c->c_cz.p;
    v.mass = c->c_mass.p;
    v.rho = c->c_rho.p;
    return v;
}

// Swap matrices B_n in block layout, Dehnen 2014 eq 63 (rotation.rs:136-211).
void build_swap(int p, std::vector<double>& sw) {
    auto boff = [](int j) { return j == 0 ? 0 : j * (4 * j * j - 1) / 3; };
    const int bs = (p + 1) * (4 * p * p + 8 * p + 3) / 3;
    sw.assign(bs, 0.0);
    sw[0] = 1.0;
    for (int n = 1; n <= p; ++n) {
        const int nb = 2 * n + 1, off = boff(n), nbp = 2 * n - 1, offp = boff(n - 1);
        auto prev = [&](int row_base, int l) -> double {
            return (std::abs(l) <= n - 1) ? sw[row_base + l + (n - 1)] : 0.0;
        };
        for (int mr = 0; mr < nb; ++mr) {
            const int mm = mr - n;
            for (int lc = 0; lc < nb; ++lc) {
                const int l = lc - n;
                double v;
                if (std::abs(mm) <= n - 1) {
                    const int rp = offp + (mr - 1) * nbp;
                    v = (prev(rp, l - 1) - prev(rp, l + 1)) * 0.5;
                } else if (mm == n) {
                    const int src = offp + (2 * n - 2) * nbp;
                    v = (prev(src, l - 1) + prev(src, l + 1) + 2.0 * prev(src, l)) * 0.5;
                } else {
                    const int src = offp;
                    v = (prev(src, l - 1) + prev(src, l + 1) - 2.0 * prev(src, l)) * 0.5;
                }
                sw[off + mr * nb + lc] = v;
            }
        }
    }
}

}  // namespace

// Real half-basis forms of the swap matrices for the warp rotation M2L.
void fmmx::make_rotw_tables(RotwTables& t) {
    const int P = kRotwMaxP;
    std::vector<double> sw;
    build_swap(P, sw);
    auto boff = [](int j) { return j == 0 ? 0 : j * (4 * j * j - 1) / 3; };
    t.mats.assign(rot_moff_host(P + 1), 0.0);
    for (int k = 0; k <= P; ++k) {
        const int nb = 2 * k + 1, off = boff(k), kk = (k + 1) * (k + 1);
        auto B = [&](int r, int c) { return sw[off + (r + k) * nb + (c + k)]; };
        double* Pm = t.mats.data() + rot_moff_host(k);
        double* Qm = Pm + kk;
        double* PT = Qm + kk;
        double* QT = PT + kk;
        for (int r = 0; r <= k; ++r)
            for (int c = 0; c <= k; ++c) {
                const double sg = (c & 1) ? -1.0 : 1.0;
                if (c == 0) {
                    Pm[r * (k + 1)] = B(r, 0);
                    Qm[r * (k + 1)] = B(r, 0);
                    PT[r * (k + 1)] = B(0, r);
                    QT[r * (k + 1)] = B(0, r);
                } else {
                    Pm[r * (k + 1) + c] = B(r, c) + sg * B(r, -c);
                    Qm[r * (k + 1) + c] = B(r, c) - sg * B(r, -c);
                    PT[r * (k + 1) + c] = B(c, r) + sg * B(-c, r);
                    QT[r * (k + 1) + c] = B(c, r) - sg * B(-c, r);
                }
            }
    }
    std::vector<double> f(2 * P + 1, 1.0);
    for (int i = 1; i <= 2 * P; ++i) f[i] = f[i - 1] * (double)i;
    t.fact = f;
    const int nh = P * (P + 1) / 2 + P + 1;
    t.fm.assign(nh, 0.0);
    t.ifm.assign(nh, 0.0);
    for (int n = 0; n <= P; ++n)
        for (int m = 0; m <= n; ++m) {
            const int h = n * (n + 1) / 2 + m;
            t.fm[h] = f[n - m] * f[n + m];
            t.ifm[h] = 1.0 / t.fm[h];
        }
}

bool fmmx::rotw_tables_check(const RotwTables& t) {
    for (int k = 0; k <= kRotwMaxP; ++k) {
        const int n = k + 1;
        const double* m = t.mats.data() + rot_moff_host(k);  // P, Q, PT, QT
        for (int r = 0; r < n; ++r)
            for (int q = 0; q < n; ++q) {
                const bool p_nz = ((r + q + k) & 1) == 0;
                const bool q_nz = r >= 1 && q >= 1 && ((r + q + k) & 1) == 1;
                if (!p_nz && (m[r * n + q] != 0.0 || m[2 * n * n + r * n + q] != 0.0)) return false;
                if (q >= 1 && !q_nz && (m[n * n + r * n + q] != 0.0 || m[3 * n * n + r * n + q] != 0.0))
                    return false;
            }
    }
    return true;
}

namespace {

void make_tables(OrderTables& t) {
    const int P = FMMX_MAXP;
    std::memset(&t, 0, sizeof(t));
    t.fact[0] = 1.0;
    for (int i = 1; i <= 2 * P; ++i) t.fact[i] = t.fact[i - 1] * (double)i;  // moments.rs:11-17
    for (int p = 0; p <= P; ++p)
        for (int k = 0; k <= p; ++k) t.binom[p][k] = t.fact[p] / (t.fact[k] * t.fact[p - k]);  // :20-27
    for (int m = 1; m <= P; ++m) t.inv2m[m] = 1.0 / (double)(2 * m);
    for (int n = 0; n <= P; ++n)
        for (int m = 0; m < n; ++m) t.invc[n][m] = 1.0 / (double)(n * n - m * m);
}

enum M2lChoice { M2L_NAIVE_BLOCK, M2L_ROT_BLOCK, M2L_ROT_WARP };

// AUTO and ROTATION take the warp rotation kernel where its constant tables
// reach (p <= 16), else the block rotation kernel; NAIVE keeps the reference's
// O(p^4) convolution.
M2lChoice m2l_choice(const fmmx_config& c) {
    if (c.m2l_kernel == FMMX_M2L_NAIVE) return M2L_NAIVE_BLOCK;
    return c.p <= kRotwMaxP ? M2L_ROT_WARP : M2L_ROT_BLOCK;
}


// ---------------------------------------------------------------- build
// nsys > 1 builds a forest: system s is inputs [off[s], off[s+1]) (host
// offsets), each with its own bounding box, keys, key sort and root.
fmmx_status build_impl(fmmx_ctx* ctx, size_t n, const double* d_pos, const double* d_mass, int nsys = 1,
                       const uint64_t* h_off = nullptr) {
    cudaStream_t s = ctx->stream;
    if (n == 0) return fail(ctx, FMMX_INVALID_ARG, "empty input (the reference asserts !parts.is_empty(), tree.rs:95)");
    if (n >= (1ull << 31)) return fail(ctx, FMMX_INVALID_ARG, "n must be below 2^31");
    if (nsys < 1) return fail(ctx, FMMX_INVALID_ARG, "no systems");
    if (nsys > 1) {
        if (h_off[0] != 0 || h_off[nsys] != n) return fail(ctx, FMMX_INVALID_ARG, "offsets must run from 0 to n");
        for (int q = 0; q < nsys; ++q)
            if (h_off[q + 1] <= h_off[q]) return fail(ctx, FMMX_INVALID_ARG, "every system needs at least one body");
    }
    ctx->built = false;
    ctx->evaluated = false;
    ctx->lists_valid = false;
    ctx->drop_graph();  // its kernels address the buffers and sizes of the old tree
    ctx->n = n;
    ctx->nsys = nsys;
    if (ctx->events) CK(cudaEventRecord(ctx->ev[0], s), "event");
    CK(ctx->keys.ensure(n), "alloc keys");
    CK(ctx->keys_sorted.ensure(n), "alloc keys");
    CK(ctx->idx.ensure(n), "alloc idx");
    CK(ctx->order.ensure(n), "alloc order");
    for (DBuf<double>* b : {&ctx->x, &ctx->y, &ctx->z, &ctx->m, &ctx->nax, &ctx->nay, &ctx->naz, &ctx->npot})
        CK(b->ensure(n), "alloc bodies");
    CK(ctx->box.ensure(8 * (size_t)nsys), "alloc box");
    ctx->steps_since_build = 0;
    if (nsys > 1) {
        ctx->sys_off_host.assign(h_off, h_off + nsys + 1);
        CK(ctx->sys_off.ensure(nsys + 1), "alloc offsets");
        CK(cudaMemcpyAsync(ctx->sys_off.p, h_off, (nsys + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, s), "copy");
    }
    const unsigned gb = std::min<unsigned>(grid_for(n, 256), 1024u);
    CK(ctx->bbox_part.ensure(gb * 6), "alloc box");
    CK(ctx->flags.ensure(8), "alloc flags");
    CK(cudaMemsetAsync(ctx->flags.p, 0, 8 * sizeof(int), s), "memset");

    ctx->launches = 0;
    const int nbits = 3 * FMMX_BITS;
    size_t tb;
    LCOUNT(5);  // bbox (2), keys, key sort (onesweep passes counted as 1), gather
    if (nsys == 1) {
        k_bbox_partial<<<gb, 256, 0, s>>>(d_pos, n, ctx->bbox_part.p, ctx->flags.p + 2);
        k_bbox_final<<<1, 32, 0, s>>>(ctx->bbox_part.p, (int)gb, ctx->box.p);
        k_keys<<<grid_for(n, 256), 256, 0, s>>>(d_pos, n, ctx->box.p, ctx->keys.p, ctx->idx.p);
        CKL("keys");
        tb = sort_pairs_u64_u32_temp((int)n, nbits);
        CK(ctx->cub_tmp.ensure(tb), "alloc sort");
        CK(sort_pairs_u64_u32(ctx->cub_tmp.p, tb, ctx->keys.p, ctx->keys_sorted.p, ctx->idx.p, ctx->order.p, (int)n,
                              nbits, s),
           "key sort");
    } else {
        k_bbox_seg<<<nsys, 256, 0, s>>>(d_pos, ctx->sys_off.p, ctx->box.p, ctx->flags.p + 2);
        k_keys_seg<<<grid_for(n, 256), 256, 0, s>>>(d_pos, n, ctx->sys_off.p, nsys, ctx->box.p, ctx->keys.p,
                                                    ctx->idx.p);
        CKL("keys");
        tb = sort_pairs_seg_temp((int)n, nsys, ctx->sys_off.p, nbits);
        CK(ctx->cub_tmp.ensure(tb), "alloc sort");
        CK(sort_pairs_seg(ctx->cub_tmp.p, tb, ctx->keys.p, ctx->keys_sorted.p, ctx->idx.p, ctx->order.p, (int)n, nsys,
                          ctx->sys_off.p, nbits, s),
           "key sort");
    }
    k_gather<<<grid_for(n, 256), 256, 0, s>>>(d_pos, d_mass, ctx->order.p, n, ctx->x.p, ctx->y.p, ctx->z.p, ctx->m.p);
    CKL("gather");

    // level-by-level node creation, retried with more room on overflow
    CK(ctx->lvl.ensure(LV_SIZE), "alloc lvl");
    if (ctx->tcap == 0 || ctx->tcap < (uint32_t)nsys) {
        uint64_t est = 4ull * n / (uint64_t)std::max(ctx->cfg.n_leaf, 1) + 8ull * FMMX_NLEVELS * nsys + 64;
        ctx->tcap = (uint32_t)std::min<uint64_t>(est, 0x7fffffffull);
    }
    int hl[LV_SIZE];
    int hflags[8];
    for (int attempt = 0;; ++attempt) {
        const uint32_t cap = ctx->tcap;
        CK(ctx->t_first.ensure(cap), "alloc nodes");
        CK(ctx->t_count.ensure(cap), "alloc nodes");
        CK(ctx->t_parent.ensure(cap), "alloc nodes");
        CK(ctx->t_oct.ensure(cap), "alloc nodes");
        CK(ctx->t_level.ensure(cap), "alloc nodes");
        CK(ctx->t_leaf.ensure(cap), "alloc nodes");
        TmpNodes tn{ctx->t_first.p, ctx->t_count.p, ctx->t_parent.p, ctx->t_oct.p, ctx->t_level.p, ctx->t_leaf.p};
        CK(cudaMemsetAsync(ctx->lvl.p, 0, LV_SIZE * sizeof(int), s), "memset");
        CK(cudaMemsetAsync(ctx->flags.p, 0, 2 * sizeof(int), s), "memset");
        if (nsys == 1) k_tree_init<<<1, 32, 0, s>>>(tn, (uint32_t)n, ctx->lvl.p);
        else k_tree_init_forest<<<grid_for(nsys, 128), 128, 0, s>>>(tn, ctx->sys_off.p, nsys, ctx->lvl.p);
        LCOUNT(1 + FMMX_NLEVELS);
        const unsigned gl = std::min<unsigned>(grid_for(cap, 256), 8u * (unsigned)ctx->nsm);
        for (int L = 0; L < FMMX_NLEVELS; ++L)
            k_build_level<<<gl, 256, 0, s>>>(tn, ctx->keys_sorted.p, L, (long long)ctx->cfg.n_leaf, cap, ctx->lvl.p,
                                              ctx->flags.p);
        CKL("build levels");
        CK(cudaMemcpyAsync(hl, ctx->lvl.p, sizeof(hl), cudaMemcpyDeviceToHost, s), "copy");
        CK(cudaMemcpyAsync(hflags, ctx->flags.p, sizeof(hflags), cudaMemcpyDeviceToHost, s), "copy");
        CK(cudaStreamSynchronize(s), "tree build");
        if (hflags[2]) return fail(ctx, FMMX_INVALID_ARG, "non-finite position");
        if (!hflags[0]) break;
        uint64_t total = 0;
        for (int L = 0; L < FMMX_NLEVELS; ++L) total += (uint64_t)hl[LV_COUNT + L];
        uint64_t want = std::max<uint64_t>(2ull * cap, total + total / 2 + 64);
        if (want > 0x7fffffffull || attempt > 8) return fail(ctx, FMMX_OUT_OF_MEMORY, "node capacity");
        ctx->tcap = (uint32_t)want;
    }
    int nc = 0, nlev = 0;
    for (int L = 0; L < FMMX_NLEVELS; ++L) {
        ctx->lvl_start[L] = nc;
        ctx->lvl_count[L] = hl[LV_COUNT + L];
        nc += hl[LV_COUNT + L];
        if (hl[LV_COUNT + L] > 0) nlev = L + 1;
    }
    ctx->nc = nc;
    ctx->nlevels = nlev;
    ctx->nleaves = hflags[1];

    // depth-first renumbering: sort nodes by (first slot, level)
    TmpNodes tn{ctx->t_first.p, ctx->t_count.p, ctx->t_parent.p, ctx->t_oct.p, ctx->t_level.p, ctx->t_leaf.p};
    CK(ctx->dfs_key.ensure(nc), "alloc");
    CK(ctx->dfs_key_alt.ensure(nc), "alloc");
    CK(ctx->dfs_val.ensure(nc), "alloc");
    CK(ctx->dfs_val_alt.ensure(nc), "alloc");
    CK(ctx->new_id.ensure(nc), "alloc");
    k_dfs_keys<<<grid_for(nc, 256), 256, 0, s>>>(tn, nc, ctx->dfs_key.p, ctx->dfs_val.p);
    LCOUNT(5 + nlev);  // dfs keys, sort, finalize, link, body->leaf, geometry per level
    const int dbits = 5 + bits_for(n);
    tb = sort_pairs_u64_u32_temp(nc, dbits);
    CK(ctx->cub_tmp.ensure(tb), "alloc sort");
    CK(sort_pairs_u64_u32(ctx->cub_tmp.p, tb, ctx->dfs_key.p, ctx->dfs_key_alt.p, ctx->dfs_val.p, ctx->dfs_val_alt.p,
                          nc, dbits, s),
       "dfs sort");
    for (DBuf<uint32_t>* b : {&ctx->c_first, &ctx->c_count}) CK(b->ensure(nc), "alloc cells");
    CK(ctx->c_child.ensure(8 * (size_t)nc), "alloc cells");
    CK(ctx->c_parent.ensure(nc), "alloc cells");
    CK(ctx->level_cells.ensure(nc), "alloc cells");
    CK(ctx->body_leaf.ensure(n), "alloc cells");
    CK(ctx->c_leaf.ensure(nc), "alloc cells");
    CK(ctx->c_level.ensure(nc), "alloc cells");
    for (DBuf<double>* b : {&ctx->c_cx, &ctx->c_cy, &ctx->c_cz, &ctx->c_mass, &ctx->c_rho})
        CK(b->ensure(nc), "alloc cells");
    CK(cudaMemsetAsync(ctx->c_child.p, 0xff, 8 * (size_t)nc * sizeof(int32_t), s), "memset");
    k_finalize_cells<<<grid_for(nc, 256), 256, 0, s>>>(ctx->dfs_val_alt.p, nc, tn, ctx->new_id.p, view_mut(ctx));
    k_link_cells<<<grid_for(nc, 256), 256, 0, s>>>(nc, tn, ctx->new_id.p, view_mut(ctx), ctx->level_cells.p);
    k_body_leaf<<<grid_for((size_t)nc * 32, 256), 256, 0, s>>>(nc, ctx->c_first.p, ctx->c_count.p, ctx->c_leaf.p,
                                                               ctx->body_leaf.p);
    CKL("finalize cells");
    for (int L = nlev - 1; L >= 0; --L) {
        const int cnt = ctx->lvl_count[L];
        k_geometry_level<<<grid_for(cnt, 128), 128, 0, s>>>(ctx->level_cells.p, ctx->lvl_start[L], cnt,
                                                            view_mut(ctx), ctx->x.p, ctx->y.p, ctx->z.p, ctx->m.p,
                                                            ctx->cfg.center_mode);
    }
    CKL("geometry");
    CK(ctx->c_h.ensure(nc), "alloc cells");
    for (int L = 0; L < nlev; ++L) {
        const int cnt = ctx->lvl_count[L];
        k_cell_h<<<grid_for(cnt, 256), 256, 0, s>>>(ctx->level_cells.p, ctx->lvl_start[L], cnt, ctx->c_parent.p,
                                                    ctx->box.p, ctx->c_h.p);
    }
    CK(ctx->c_geo.ensure(nc), "alloc cells");
    k_pack_geo<<<grid_for(nc, 256), 256, 0, s>>>(nc, ctx->c_cx.p, ctx->c_cy.p, ctx->c_cz.p, ctx->c_rho.p, ctx->c_geo.p);
    LCOUNT(nlev + 1);
    CKL("cell sizes");
    if (ctx->events) CK(cudaEventRecord(ctx->ev[1], s), "event");
    CK(cudaStreamSynchronize(s), "build");
    if (ctx->events) {
        float ms = 0;
        cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
        ctx->st.ms_build = ms;
    }
    ctx->build_pos = d_pos;
    ctx->build_mass = d_mass;
    ctx->launches_build = ctx->launches;
    ctx->built = true;
    return FMMX_OK;
}

// ---------------------------------------------------------------- evaluate
fmmx_status walk_impl(fmmx_ctx* ctx, cudaStream_t s) {
    const int nc = ctx->nc;
    // capacities follow the current tree (a context may see trees of very
    // different sizes, e.g. the forests of a serving loop) and grow on overflow
    auto at_least = [](uint32_t c, uint64_t w) { return (uint32_t)std::min<uint64_t>(std::max<uint64_t>(c, w), 0x7fffffffull); };
    if (ctx->walk_cap0 > 0) {  // test knob: start from the given capacity (and grow on overflow)
        ctx->cap_front = at_least(ctx->cap_front, ctx->walk_cap0);
        ctx->cap_m2l = at_least(ctx->cap_m2l, ctx->walk_cap0);
        ctx->cap_p2p = at_least(ctx->cap_p2p, ctx->walk_cap0);
    } else {
        ctx->cap_front = at_least(ctx->cap_front, 64ull * nc + 1024);
        ctx->cap_m2l = at_least(ctx->cap_m2l, 64ull * nc + 1024);
        ctx->cap_p2p = at_least(ctx->cap_p2p, 32ull * nc + 1024);
    }
    ctx->walk_retries = 0;
    CK(ctx->wcounts.ensure(WC_SIZE), "alloc");
    CK(ctx->wpops.ensure(1), "alloc");
    MacParams mp;
    mp.mode = ctx->cfg.mac_mode;
    mp.p = ctx->cfg.p;
    mp.eps = ctx->cfg.mac_eps;
    mp.theta = ctx->cfg.theta;
    mp.gap = ctx->cfg.soft_gap * ctx->cfg.softening;
    const CellsView cv = view(ctx);
    for (int attempt = 0;; ++attempt) {
        CK(ctx->front0.ensure(ctx->cap_front), "alloc walk");
        CK(ctx->front1.ensure(ctx->cap_front), "alloc walk");
        CK(ctx->m2l.ensure(ctx->cap_m2l), "alloc walk");
        CK(ctx->p2p.ensure(ctx->cap_p2p), "alloc walk");
        WalkBufs w;
        w.front[0] = ctx->front0.p;
        w.front[1] = ctx->front1.p;
        w.m2l = ctx->m2l.p;
        w.p2p = ctx->p2p.p;
        w.counts = ctx->wcounts.p;
        w.pops_ptr = ctx->wpops.p;
        w.cap_front = ctx->cap_front;
        w.cap_m2l = ctx->cap_m2l;
        w.cap_p2p = ctx->cap_p2p;
        CK(cudaMemsetAsync(ctx->wcounts.p, 0, WC_SIZE * sizeof(int), s), "memset");
        CK(cudaMemsetAsync(ctx->wpops.p, 0, sizeof(unsigned long long), s), "memset");
        // seeds: the self pair of every root (one per system)
        k_walk_init<<<grid_for(ctx->nsys, 128), 128, 0, s>>>(ctx->level_cells.p, ctx->nsys, ctx->front0.p);
        LCOUNT(1);
        const int seeds = ctx->nsys;  // pageable source: staged before the call returns
        CK(cudaMemcpyAsync(ctx->wcounts.p + WC_FRONT0, &seeds, sizeof(int), cudaMemcpyHostToDevice, s), "copy");
        int cur = 0;
        int hc[WC_SIZE];
        bool done = false;
        const int max_iter = 8 * FMMX_NLEVELS + 16;
        // One kernel per MAC, so the theta form carries none of the Dehnen
        // estimate's registers (54 against 80: four resident blocks per SM
        // instead of three), launched with exactly the resident blocks: the
        // grid-stride loop then runs in one wave instead of a last, partly
        // filled one.
        const bool dehnen = mp.mode == FMMX_MAC_DEHNEN;
        int& wb = ctx->walk_blocks[dehnen ? 1 : 0];
        if (wb == 0) wb = walk_iter_blocks_per_sm(dehnen) * ctx->nsm;
        for (int it = 0; it < max_iter && !done;) {
            for (int b = 0; b < 6; ++b, ++it) {
                launch_walk_iter(dehnen, (unsigned)wb, s, cv, mp, ctx->pows.p, ctx->fmin.p, w, cur);
                LCOUNT(1);
                CK(cudaMemsetAsync(ctx->wcounts.p + cur, 0, sizeof(int), s), "memset");
                cur ^= 1;
            }
            CKL("walk");
            CK(cudaMemcpyAsync(hc, ctx->wcounts.p, sizeof(hc), cudaMemcpyDeviceToHost, s), "copy");
            CK(cudaStreamSynchronize(s), "walk");
            if (hc[WC_OVERFLOW] || hc[cur] == 0) done = true;
        }
        if (!done) return fail(ctx, FMMX_TIMEOUT, "dual walk did not terminate");
        if (hc[WC_OVERFLOW]) {
            if (attempt > 24) return fail(ctx, FMMX_OUT_OF_MEMORY, "walk capacity");
            ctx->walk_retries++;
            auto grow = [](uint32_t c, int used) {
                uint64_t w2 = std::max<uint64_t>(4ull * c, (uint64_t)used + (uint64_t)used / 2 + 1024);
                return (uint32_t)std::min<uint64_t>(w2, 0x7fffffffull);
            };
            if (hc[WC_OVERFLOW] & 1) ctx->cap_front = grow(ctx->cap_front, 0);
            if (hc[WC_OVERFLOW] & 2) ctx->cap_p2p = grow(ctx->cap_p2p, hc[WC_P2P]);
            if (hc[WC_OVERFLOW] & 4) ctx->cap_m2l = grow(ctx->cap_m2l, hc[WC_M2L]);
            continue;
        }
        ctx->n_m2l = hc[WC_M2L];
        ctx->n_p2p = hc[WC_P2P];
        CK(cudaMemcpy(&ctx->pops, ctx->wpops.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost), "copy");
        return FMMX_OK;
    }
}

// The directed lists of one kind (M2L or P2P) from the walk's mutual pairs:
// a counting sort on the destination, segment sorts, and -- after a host
// read-back of the number of long segments -- CUB's segmented sort of those.
// The two kinds run on different streams with their own scratch (tmp, cnt,
// bounds). list_launch queues a list's kernels without waiting on the device;
// list_finish reads back its long-segment count (waiting for that stream) and
// sorts the long segments. Both lists are launched before either is finished,
// so their builds -- bound by atomics and latency, not by the SMs' arithmetic
// -- run side by side.
fmmx_status list_launch(fmmx_ctx* ctx, bool near, cudaStream_t s, DBuf<char>& tmp, DBuf<uint32_t>& cnt) {
    const int nc = ctx->nc;
    const int npairs = near ? ctx->n_p2p : ctx->n_m2l;
    const size_t ndir = near ? (npairs > 0 ? 2 * (size_t)npairs - (size_t)ctx->nleaves : 0)  // one entry per self pair
                             : 2 * (size_t)npairs;
    if (ndir > 0x7fffffffull) return fail(ctx, FMMX_OUT_OF_MEMORY, "interaction lists above 2^31 entries");
    DBuf<uint32_t>& off = near ? ctx->p2p_off : ctx->m2l_off;
    DBuf<uint32_t>& src_u = near ? ctx->p2p_src_u : ctx->m2l_src_u;
    DBuf<uint32_t>& src = near ? ctx->p2p_src : ctx->m2l_src;
    DBuf<int>& longs = near ? ctx->p2p_longs : ctx->m2l_longs;
    CK(off.ensure(nc + 1), "alloc lists");
    CK(cnt.ensure(nc + 1), "alloc lists");
    // (P2P: room for 2 entries per pair -- the scatter writes inside the
    // counted segments whatever the number of self pairs)
    const size_t room = near ? 2 * (size_t)npairs : ndir;
    CK(src_u.ensure(std::max<size_t>(room, 1)), "alloc lists");
    CK(src.ensure(std::max<size_t>(room, 1)), "alloc lists");
    CK(longs.ensure(2 * (size_t)nc + 128), "alloc lists");
    if (near) {
        CK(ctx->inter.ensure(1), "alloc");
        CK(cudaMemsetAsync(ctx->inter.p, 0, sizeof(unsigned long long), s), "memset");
    }
    CK(tmp.ensure(directed_list_temp((int)ndir, nc)), "alloc sort");
    LCOUNT(6);  // count, scan (2), scatter, segment sorts (2)
    CK(build_directed_list(tmp.p, tmp.cap, near ? ctx->p2p.p : ctx->m2l.p, npairs, (int)ndir, nc,
                           near ? ctx->c_count.p : nullptr, near ? ctx->inter.p : nullptr, cnt.p, off.p, src_u.p,
                           src.p, longs.p, grid_for(npairs, 256), s),
       near ? "p2p lists" : "m2l lists");
    const bool units = near && ctx->cfg.precision == FMMX_MIXED;
    if (units) {
        // near-field work units: per leaf ceil(sources / P2P_UNIT_SRC), and the
        // scratch for the partial sums of leaves with several units
        for (DBuf<uint32_t>* b : {&ctx->p2p_units, &ctx->p2p_scr, &ctx->p2p_uoff, &ctx->p2p_soff, &ctx->p2p_units_s,
                                   &ctx->p2p_units_b, &ctx->p2p_uoff_s, &ctx->p2p_uoff_b})
            CK(b->ensure(nc + 1), "alloc lists");
        CK(ctx->p2p_next.ensure(2), "alloc lists");
        const DirList lp{nullptr, ctx->p2p_src.p, ctx->p2p_off.p, ctx->p2p_off.p + 1, 32};
        launch_p2p_plan(grid_for(nc + 1, 256), s, nc, lp, ctx->c_count.p, ctx->p2p_units.p, ctx->p2p_units_s.p,
                        ctx->p2p_units_b.p, ctx->p2p_scr.p);
        CK(scan_u32(tmp.p, tmp.cap, ctx->p2p_units.p, ctx->p2p_uoff.p, nc + 1, s), "p2p units");
        CK(scan_u32(tmp.p, tmp.cap, ctx->p2p_units_s.p, ctx->p2p_uoff_s.p, nc + 1, s), "p2p units");
        CK(scan_u32(tmp.p, tmp.cap, ctx->p2p_units_b.p, ctx->p2p_uoff_b.p, nc + 1, s), "p2p units");
        CK(scan_u32(tmp.p, tmp.cap, ctx->p2p_scr.p, ctx->p2p_soff.p, nc + 1, s), "p2p units");
        LCOUNT(9);
    }
    return FMMX_OK;
}

fmmx_status list_finish(fmmx_ctx* ctx, bool near, cudaStream_t s, DBuf<char>& tmp, DBuf<uint32_t>& bounds) {
    const int nc = ctx->nc;
    const int npairs = near ? ctx->n_p2p : ctx->n_m2l;
    const size_t ndir = near ? (npairs > 0 ? 2 * (size_t)npairs - (size_t)ctx->nleaves : 0) : 2 * (size_t)npairs;
    DBuf<uint32_t>& off = near ? ctx->p2p_off : ctx->m2l_off;
    DBuf<uint32_t>& src_u = near ? ctx->p2p_src_u : ctx->m2l_src_u;
    DBuf<uint32_t>& src = near ? ctx->p2p_src : ctx->m2l_src;
    DBuf<int>& longs = near ? ctx->p2p_longs : ctx->m2l_longs;
    const bool units = near && ctx->cfg.precision == FMMX_MIXED;
    // host read-back: the number of long segments (and the P2P scratch size)
    int nlong = 0;
    uint32_t nscr = 0;
    CK(cudaMemcpyAsync(&nlong, longs.p, sizeof(int), cudaMemcpyDeviceToHost, s), "copy");
    if (units) CK(cudaMemcpyAsync(&nscr, ctx->p2p_soff.p + nc, sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "copy");
    CK(cudaStreamSynchronize(s), "lists");
    if (units) CK(ctx->p2p_part.ensure(std::max<size_t>(nscr, 1)), "alloc p2p scratch");
    if (nlong > 0) {
        const int end_bit = bits_for((uint64_t)nc);
        CK(bounds.ensure(2 * (size_t)nlong), "alloc lists");
        CK(tmp.ensure(long_segments_temp((int)ndir, nlong, end_bit)), "alloc sort");
        LCOUNT(2);
        CK(sort_long_segments(tmp.p, tmp.cap, off.p, longs.p, nlong, src_u.p, src.p, (int)ndir, end_bit, bounds.p,
                              s),
           near ? "p2p lists" : "m2l lists");
    }
    return FMMX_OK;
}

// Mixed form, near field: FP32 + double-single P2P on the second stream.
fmmx_status near_mixed(fmmx_ctx* ctx, const DirList& lp, bool tm) {
    cudaStream_t s2 = ctx->cfg.overlap ? ctx->stream2 : ctx->stream;
    const int nc = ctx->nc;
    const size_t n = ctx->n;
    const CellsView cv = view(ctx);
    cudaEvent_t* ev = ctx->ev;
    if (tm) CK(cudaEventRecord(ev[12], s2), "event");
    const float soft2 = (float)(ctx->cfg.softening * ctx->cfg.softening);
    CK(cudaMemsetAsync(ctx->p2p_next.p, 0, 2 * sizeof(unsigned), s2), "memset");
    const P2pUnits units{ctx->p2p_uoff.p, ctx->p2p_uoff_s.p, ctx->p2p_uoff_b.p, ctx->p2p_soff.p, ctx->p2p_part.p,
                         ctx->p2p_next.p};
    launch_p2p_mixed(ctx->cfg.p2p_tile > 0 ? ctx->cfg.p2p_tile : 512, ctx->nsm, s2, lp, nc, cv, units, n,
                     ctx->body_leaf.p, ctx->x.p, ctx->y.p, ctx->z.p, ctx->m.p, ctx->body_loc.p, soft2, ctx->nax.p,
                     ctx->nay.p, ctx->naz.p, ctx->npot.p);
    CKL("p2p (mixed)");
    if (tm) CK(cudaEventRecord(ev[8], s2), "event");
    CK(cudaEventRecord(ctx->fork[2], s2), "event");
    return FMMX_OK;
}

// Mixed form, far field: FP32 M2L/L2L on normalised expansions, then the L2P,
// which adds the near field.
fmmx_status far_mixed(fmmx_ctx* ctx, const DirList& lm, double* d_acc, double* d_pot, bool tm) {
    cudaStream_t s = ctx->stream;
    const int p = ctx->cfg.p, nc = ctx->nc;
    const size_t n = ctx->n;
    const CellsView cv = view(ctx);
    cudaEvent_t* ev = ctx->ev;
    if (tm) CK(cudaEventRecord(ev[11], s), "event");  // far field from here
    CK(cudaMemsetAsync(ctx->loc_f.p, 0, (size_t)nc * half_stride(p) * sizeof(zf), s), "memset");
    if (ctx->n_m2l > 0) {
        if (p > kRotwMaxP) return fail(ctx, FMMX_INVALID_ARG, "mixed precision supports p <= 16");
        int* work = nullptr;  // preemptible: one block per destination cell
        if (!ctx->cfg.preemptible) {
            CK(ctx->work.ensure(1), "alloc");
            CK(cudaMemsetAsync(ctx->work.p, 0, sizeof(int), s), "memset");
            work = ctx->work.p;
        }
        CK(launch_rotw_f32(p, lm, nc, cv, ctx->ellf.p, ctx->mom_f.p, ctx->loc_f.p, work, ctx->nsm, s), "m2l");
    }
    if (tm) CK(cudaEventRecord(ev[6], s), "event");
    LCOUNT((ctx->n_m2l > 0 ? 1 : 0) + (ctx->nlevels - 1) + 5);  // m2l, l2l per level, coords + p2p (2) + combine, l2p
    for (int L = 1; L < ctx->nlevels; ++L) {
        const int cnt = ctx->lvl_count[L];
        const unsigned g = std::min<unsigned>(cnt, 16u * (unsigned)ctx->nsm);
        launch_l2l_mixed(L <= 3, g, s, ctx->level_cells.p, ctx->lvl_start[L], cnt, cv, ctx->c_parent.p, ctx->ell.p,
                         p, ctx->loc_f.p);
    }
    CKL("l2l (mixed)");
    if (tm) CK(cudaEventRecord(ev[7], s), "event");
    CK(cudaStreamWaitEvent(s, ctx->fork[2], 0), "join");  // L2P adds the near field
    if (tm) CK(cudaEventRecord(ev[13], s), "event");
    k_l2p_mixed<<<grid_for(n, 128), 128, 0, s>>>(n, ctx->body_leaf.p, ctx->order.p, cv, ctx->ell.p, p,
                                                 ctx->loc_f.p, ctx->x.p, ctx->y.p, ctx->z.p, ctx->nax.p,
                                                 ctx->nay.p, ctx->naz.p, ctx->npot.p, d_acc, d_pot);
    CKL("l2p (mixed)");
    return FMMX_OK;
}

// reuse: keep the interaction lists of the last evaluation of this tree (no
// f pre-pass, walk or list build); moments and locals are recomputed from the
// given positions about the cell centres of the last build. This is the
// tree reuse of the reference's GPU backend (crates/visual/src/gpufmm.rs:9-20).
// capture: the calls are being recorded into a CUDA graph (reuse only): no
// timing events and no read-back at the end.
fmmx_status evaluate_impl(fmmx_ctx* ctx, const double* d_pos, const double* d_mass, double* d_acc, double* d_pot,
                          bool reuse = false, bool capture = false) {
    cudaStream_t s = ctx->stream, s2 = ctx->cfg.overlap ? ctx->stream2 : ctx->stream;
    if (!ctx->built) return fail(ctx, FMMX_NOT_BUILT, "evaluate before build");
    const int p = ctx->cfg.p, dim = dimp(p), nc = ctx->nc;
    const size_t n = ctx->n;
    cudaEvent_t* ev = ctx->ev;
    const bool tm = ctx->events && !capture;
    if (tm) CK(cudaEventRecord(ev[2], s), "event");
    ctx->launches = ctx->launches_build;
    if (d_pos == nullptr) d_pos = ctx->build_pos;
    if (d_mass == nullptr) d_mass = ctx->build_mass;
    k_gather<<<grid_for(n, 256), 256, 0, s>>>(d_pos, d_mass, ctx->order.p, n, ctx->x.p, ctx->y.p, ctx->z.p, ctx->m.p);
    CKL("gather");
    LCOUNT(1 + ctx->nlevels + (ctx->cfg.mac_mode == FMMX_MAC_DEHNEN ? 1 : 0));  // gather, upward levels, f pre-pass
    CK(ctx->moments.ensure((size_t)nc * dim), "alloc expansions");
    CK(ctx->locals.ensure((size_t)nc * dim), "alloc expansions");
    CK(ctx->pows.ensure((size_t)nc * (p + 1)), "alloc expansions");
    CK(ctx->fmin.ensure(nc), "alloc expansions");
    CK(ctx->f.ensure(n), "alloc expansions");
    if (reuse && !ctx->lists_valid) reuse = false;
    const bool dehnen = ctx->cfg.mac_mode == FMMX_MAC_DEHNEN && !reuse;  // f pre-pass and power needed
    const bool mixed = ctx->cfg.precision == FMMX_MIXED;
    const int H = (p + 1) * (p + 2) / 2;
    const CellsView cv = view(ctx);
    if (mixed) {
        CK(ctx->body_loc.ensure(n), "alloc expansions");
        CK(ctx->mom_f.ensure((size_t)nc * half_stride(p)), "alloc expansions");
        CK(ctx->loc_f.ensure((size_t)nc * half_stride(p)), "alloc expansions");
        CK(ctx->ell.ensure(nc), "alloc expansions");
        CK(ctx->ellf.ensure(nc), "alloc expansions");
        const double* rho = ctx->c_rho.p;
        // sized on every mixed evaluation, so that a reuse step recorded into
        // a CUDA graph never allocates while capturing
        CK(ctx->rho_now.ensure(nc), "alloc expansions");
        if (reuse) {  // the bodies moved since the build: radii about the same centres
            CK(cudaMemsetAsync(ctx->rho_now.p, 0, (size_t)nc * sizeof(unsigned long long), s), "memset");
            k_rho_bodies<<<grid_for(n, 256), 256, 0, s>>>(n, ctx->body_leaf.p, cv, ctx->x.p, ctx->y.p, ctx->z.p,
                                                          ctx->rho_now.p);
            for (int L = ctx->nlevels - 1; L >= 0; --L) {
                const int cnt = ctx->lvl_count[L];
                k_rho_level<<<grid_for(cnt, 256), 256, 0, s>>>(ctx->level_cells.p, ctx->lvl_start[L], cnt, cv,
                                                               ctx->rho_now.p);
            }
            LCOUNT(1 + ctx->nlevels);
            rho = reinterpret_cast<const double*>(ctx->rho_now.p);
        }
        k_cell_scale<<<grid_for(nc, 256), 256, 0, s>>>(nc, rho, ctx->c_h.p, ctx->ell.p, ctx->ellf.p);
        LCOUNT(1);
    }
    // the second stream starts once the bodies are gathered (and, for the
    // Dehnen MAC, whose walk reads the multipole power and fmin, after the
    // upward pass)
    if (!dehnen) {
        CK(cudaEventRecord(ctx->fork[0], s), "event");
        CK(cudaStreamWaitEvent(s2, ctx->fork[0], 0), "fork");
    }
    if (dehnen) {
        CK(cudaMemsetAsync(ctx->flags.p + 3, 0, sizeof(int), s), "memset");
        k_fprepass<<<grid_for(n, 128), 128, 0, s>>>(cv, ctx->x.p, ctx->y.p, ctx->z.p, ctx->m.p, n, ctx->sys_off.p,
                                                    ctx->nsys, ctx->level_cells.p, ctx->f.p, ctx->flags.p + 3);
        CKL("f pre-pass");
    }
    if (mixed && !dehnen) {
        // normalised FP32 upward pass; FP64 accumulation on the top three levels
        for (int L = ctx->nlevels - 1; L >= 0; --L) {
            const int cnt = ctx->lvl_count[L];
            const unsigned g = std::min<unsigned>(cnt, 16u * (unsigned)ctx->nsm);
            launch_upward_mixed(L <= 2, g, 4, s, ctx->level_cells.p, ctx->lvl_start[L], cnt, cv, ctx->ell.p,
                                ctx->x.p, ctx->y.p, ctx->z.p, ctx->m.p, p, ctx->mom_f.p);
        }
        CKL("upward (mixed)");
    } else {
        const int warps = 2;  // the P2M tables take 35 KB of shared memory per warp at p = 10
        const size_t smem = (size_t)warps * upward_exact_smem_per_warp(p);
        if (smem > 48 * 1024)
            CK(cudaFuncSetAttribute(k_upward_exact, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "attr");
        const size_t smem_b = 16 * (size_t)dim * sizeof(zd);
        if (smem_b > 48 * 1024)
            CK(cudaFuncSetAttribute(k_m2m_exact_block, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_b),
               "attr");
        // per level: the leaves' P2M (a warp per leaf), then the internal
        // cells' M2M (a block per cell)
        for (int L = ctx->nlevels - 1; L >= 0; --L) {
            const int cnt = ctx->lvl_count[L];
            unsigned g = std::min<unsigned>((cnt + warps - 1) / warps, 16u * (unsigned)ctx->nsm);
            k_upward_exact<<<g, 32 * warps, smem, s>>>(ctx->level_cells.p, ctx->lvl_start[L], cnt, cv, ctx->x.p,
                                                       ctx->y.p, ctx->z.p, ctx->m.p, p, ctx->moments.p, ctx->pows.p,
                                                       dehnen ? ctx->f.p : nullptr, ctx->fmin.p, 1);
            if (L < ctx->nlevels - 1) {
                k_m2m_exact_block<<<std::min<unsigned>(cnt, 16u * (unsigned)ctx->nsm), 256, smem_b, s>>>(
                    ctx->level_cells.p, ctx->lvl_start[L], cnt, cv, p, ctx->moments.p, ctx->pows.p,
                    dehnen ? ctx->f.p : nullptr, ctx->fmin.p);
                LCOUNT(1);
            }
        }
        CKL("upward");
        if (mixed) {  // the MAC saw exact FP64 moments; the translations use FP32
            k_moments_to_mixed<<<grid_for((size_t)nc * H, 256), 256, 0, s>>>(nc, p, ctx->moments.p, ctx->ell.p,
                                                                            ctx->mom_f.p);
            LCOUNT(1);
            CKL("moments to mixed");
        }
    }
    if (tm) CK(cudaEventRecord(ev[3], s), "event");
    if (dehnen) {
        CK(cudaEventRecord(ctx->fork[0], s), "event");
        CK(cudaStreamWaitEvent(s2, ctx->fork[0], 0), "fork");
    }
    if (tm) CK(cudaEventRecord(ev[10], s2), "event");
    if (!reuse) {
        // a recorded leapfrog step addresses the list buffers and list sizes of
        // the last walk; this walk and its lists may reallocate or resize them
        ctx->drop_graph();
        ctx->lists_valid = false;
        fmmx_status st = walk_impl(ctx, s2);
        if (st != FMMX_OK) return st;
        if (dehnen) {
            int bad = 0;
            CK(cudaMemcpy(&bad, ctx->flags.p + 3, sizeof(int), cudaMemcpyDeviceToHost), "copy");
            if (bad) return fail(ctx, FMMX_DEVICE_ERROR, "f pre-pass stack overflow");
        }
    }
    if (tm) CK(cudaEventRecord(ev[4], s2), "event");
    if (!reuse) {
        CK(cudaEventRecord(ctx->fork[1], s2), "event");  // the walk's pairs are in place
        fmmx_status st = list_launch(ctx, true, s2, ctx->cub_tmp, ctx->list_cnt);
        if (st != FMMX_OK) return st;
        CK(cudaStreamWaitEvent(s, ctx->fork[1], 0), "join");  // the M2L list reads the walk's pairs
        if (tm) CK(cudaEventRecord(ev[14], s), "event");
        st = list_launch(ctx, false, s, ctx->cub_tmp2, ctx->list_cnt2);
        if (st != FMMX_OK) return st;
        st = list_finish(ctx, true, s2, ctx->cub_tmp, ctx->long_bounds);
        if (st != FMMX_OK) return st;
    }
    if (tm) CK(cudaEventRecord(ev[5], s2), "event");

    // (each list's pointers are taken after its build, which may reallocate it)
    const DirList lp{nullptr, ctx->p2p_src.p, ctx->p2p_off.p, ctx->p2p_off.p + 1, 32};
    // The near field starts on the second stream as soon as its list is
    // built; the far field's list, launched beside it, is finished on the
    // first stream after the near field is queued.
    if (mixed) {
        fmmx_status ms = near_mixed(ctx, lp, tm);
        if (ms != FMMX_OK) return ms;
    } else {
        if (tm) CK(cudaEventRecord(ev[12], s2), "event");
        const double soft2 = ctx->cfg.softening * ctx->cfg.softening;
        k_p2p_f64<<<(unsigned)nc, 128, 0, s2>>>(lp, nc, cv, ctx->x.p, ctx->y.p, ctx->z.p, ctx->m.p, soft2,
                                                ctx->nax.p, ctx->nay.p, ctx->naz.p, ctx->npot.p);
        CKL("p2p");
        if (tm) CK(cudaEventRecord(ev[8], s2), "event");
        CK(cudaEventRecord(ctx->fork[2], s2), "event");
    }
    if (!reuse) {
        fmmx_status st = list_finish(ctx, false, s, ctx->cub_tmp2, ctx->long_bounds2);
        if (st != FMMX_OK) return st;
        if (tm) CK(cudaEventRecord(ev[15], s), "event");
        ctx->lists_valid = true;
    }
    const DirList lm{nullptr, ctx->m2l_src.p, ctx->m2l_off.p, ctx->m2l_off.p + 1, 32};
    if (mixed) {
        fmmx_status ms = far_mixed(ctx, lm, d_acc, d_pot, tm);
        if (ms != FMMX_OK) return ms;
    } else {
    if (tm) CK(cudaEventRecord(ev[11], s), "event");  // far field from here
    CK(cudaMemsetAsync(ctx->locals.p, 0, (size_t)nc * dim * sizeof(zd), s), "memset");
    if (ctx->n_m2l > 0) {
        const unsigned g = std::min<unsigned>(nc, 16u * (unsigned)ctx->nsm);
        const M2lChoice ch = m2l_choice(ctx->cfg);
        if (ch == M2L_ROT_WARP) {
            int* work = nullptr;  // preemptible: one block per destination cell
            if (!ctx->cfg.preemptible) {
                CK(ctx->work.ensure(1), "alloc");
                CK(cudaMemsetAsync(ctx->work.p, 0, sizeof(int), s), "memset");
                work = ctx->work.p;
            }
            CK(launch_rotw_f64(p, lm, nc, cv, ctx->moments.p, ctx->locals.p, work, ctx->nsm, s), "m2l");
        } else if (ch == M2L_ROT_BLOCK) {
            const size_t smem = m2l_rot_smem_bytes(p);
            CK(cudaFuncSetAttribute(k_m2l_rot_f64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "attr");
            k_m2l_rot_f64<<<g, 128, smem, s>>>(lm, nc, cv, p, ctx->moments.p, ctx->locals.p, ctx->swap_dev.p);
        } else {
            const size_t smem = 2 * (size_t)dim * sizeof(zd);
            k_m2l_naive_f64<<<g, 128, smem, s>>>(lm, nc, cv, p, ctx->moments.p, ctx->locals.p);
        }
        CKL("m2l");
    }
    if (tm) CK(cudaEventRecord(ev[6], s), "event");
    LCOUNT((ctx->n_m2l > 0 ? 1 : 0) + (ctx->nlevels - 1) + 2);  // m2l, l2l per level, p2p, l2p
    {
        const size_t smem = 2 * (size_t)dim * sizeof(zd);
        for (int L = 1; L < ctx->nlevels; ++L) {
            const int cnt = ctx->lvl_count[L];
            k_l2l_f64<<<std::min<unsigned>(cnt, 16u * (unsigned)ctx->nsm), 128, smem, s>>>(ctx->level_cells.p, ctx->lvl_start[L],
                                                                            cnt, cv, ctx->c_parent.p, p,
                                                                            ctx->locals.p);
        }
        CKL("l2l");
    }
    if (tm) CK(cudaEventRecord(ev[7], s), "event");
    CK(cudaStreamWaitEvent(s, ctx->fork[2], 0), "join");  // L2P adds the near field
    if (tm) CK(cudaEventRecord(ev[13], s), "event");
    k_l2p_f64<<<grid_for(n, 128), 128, 0, s>>>(n, ctx->body_leaf.p, ctx->order.p, cv, p, ctx->locals.p, ctx->x.p,
                                               ctx->y.p, ctx->z.p, ctx->nax.p, ctx->nay.p, ctx->naz.p, ctx->npot.p,
                                               d_acc, d_pot);
    CKL("l2p");
    }
    if (tm) CK(cudaEventRecord(ev[9], s), "event");
    if (capture) return FMMX_OK;
    CK(cudaStreamSynchronize(s), "evaluate");
    CK(cudaMemcpy(&ctx->p2p_inter, ctx->inter.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost), "copy");
    if (tm) {
        auto el = [&](int a, int b) {
            float ms = 0;
            cudaEventElapsedTime(&ms, ev[a], ev[b]);
            return (double)ms;
        };
        // stages on the two streams overlap: each is timed on its own stream
        ctx->st.ms_upward = el(2, 3);
        ctx->st.ms_walk = el(10, 4);
        ctx->st.ms_lists = el(4, 5) + (reuse ? 0.0 : el(14, 15));
        ctx->st.ms_m2l = el(11, 6);
        ctx->st.ms_l2l = el(6, 7);
        ctx->st.ms_p2p = el(12, 8);
        ctx->st.ms_l2p = el(13, 9);
        ctx->st.ms_evaluate = el(2, 9);
    }
    ctx->evaluated = true;
    return FMMX_OK;
}

}  // namespace

// ================================================================== C ABI
extern "C" {

void fmmx_config_default(fmmx_config* c) {
    if (!c) return;
    c->p = 8;
    c->mac_mode = FMMX_MAC_DEHNEN;
    c->mac_eps = 1e-5;
    c->theta = 0.5;
    c->softening = 0.0;
    c->n_leaf = 16;
    c->center_mode = FMMX_CENTER_COM;
    c->precision = FMMX_PLAIN_FP64;
    c->m2l_kernel = FMMX_M2L_AUTO;
    c->device = 0;
    c->stream = nullptr;
    c->p2p_tile = 0;
    c->preemptible = 0;
    c->soft_gap = 0.0;
    c->use_graphs = 1;
    c->overlap = 1;
    c->device_budget_bytes = 0;
}

const char* fmmx_status_string(fmmx_status s) {
    switch (s) {
        case FMMX_OK: return "ok";
        case FMMX_INVALID_ARG: return "invalid argument";
        case FMMX_OUT_OF_MEMORY: return "out of memory";
        case FMMX_OVER_BUDGET: return "over budget";
        case FMMX_LEAF_OVERFLOW: return "leaf overflow";
        case FMMX_DEVICE_ERROR: return "device error";
        case FMMX_TIMEOUT: return "timeout";
        case FMMX_NOT_BUILT: return "not built";
        case FMMX_NO_DEVICE: return "no CUDA device";
    }
    return "unknown";
}

fmmx_status fmmx_create(const fmmx_config* cfg, fmmx_ctx** out) {
    if (!out) return FMMX_INVALID_ARG;
    *out = nullptr;
    fmmx_config c;
    if (cfg) c = *cfg;
    else fmmx_config_default(&c);
    if (c.p < 1 || c.p > FMMX_MAXP) return FMMX_INVALID_ARG;
    if (c.n_leaf < 0) return FMMX_INVALID_ARG;
    if (c.mac_mode != FMMX_MAC_DEHNEN && c.mac_mode != FMMX_MAC_THETA) return FMMX_INVALID_ARG;
    if (c.mac_mode == FMMX_MAC_THETA && !(c.theta > 0.0)) return FMMX_INVALID_ARG;
    if (!(c.softening >= 0.0)) return FMMX_INVALID_ARG;
    if (c.center_mode != FMMX_CENTER_COM && c.center_mode != FMMX_CENTER_SPHERE) return FMMX_INVALID_ARG;
    if (c.precision != FMMX_PLAIN_FP64 && c.precision != FMMX_MIXED) return FMMX_INVALID_ARG;
    if (c.p2p_tile < 0 || c.p2p_tile > 1024) return FMMX_INVALID_ARG;
    if (c.preemptible != 0 && c.preemptible != 1) return FMMX_INVALID_ARG;
    if (!(c.soft_gap >= 0.0) || !std::isfinite(c.soft_gap)) return FMMX_INVALID_ARG;
    if (c.use_graphs != 0 && c.use_graphs != 1) return FMMX_INVALID_ARG;
    if (c.overlap != 0 && c.overlap != 1) return FMMX_INVALID_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return FMMX_NO_DEVICE;
    }
    if (c.device < 0 || c.device >= ndev) return FMMX_INVALID_ARG;
    if (cudaSetDevice(c.device) != cudaSuccess) return FMMX_DEVICE_ERROR;
    std::vector<DBufBase*> reg;
    tl_registry = &reg;
    fmmx_ctx* ctx = new fmmx_ctx();
    tl_registry = nullptr;
    for (DBufBase* b : reg)
        if (b != &ctx->swap_dev) ctx->cache.push_back(b);
    ctx->cfg = c;
    ctx->budget.limit = c.device_budget_bytes;
    BudgetScope bscope(&ctx->budget);
    if (const char* wc = std::getenv("FMMX_TEST_WALK_CAPACITY")) ctx->walk_cap0 = std::strtoull(wc, nullptr, 10);
    std::memset(&ctx->st, 0, sizeof(ctx->st));
    if (c.stream) {
        ctx->stream = (cudaStream_t)c.stream;
    } else {
        if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete ctx;
            return FMMX_DEVICE_ERROR;
        }
        ctx->own_stream = true;
    }
    ctx->events = true;
    for (int i = 0; i < 16; ++i) cudaEventCreate(&ctx->ev[i]);
    {
        int prio = 0;
        cudaStreamGetPriority(ctx->stream, &prio);
        if (cudaStreamCreateWithPriority(&ctx->stream2, cudaStreamNonBlocking, prio) != cudaSuccess) {
            cudaGetLastError();
            fmmx_destroy(ctx);
            return FMMX_DEVICE_ERROR;
        }
        for (int i = 0; i < 3; ++i)
            if (cudaEventCreateWithFlags(&ctx->fork[i], cudaEventDisableTiming) != cudaSuccess) {
                cudaGetLastError();
                fmmx_destroy(ctx);
                return FMMX_DEVICE_ERROR;
            }
    }
    cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, c.device);
    if (ctx->nsm < 1) ctx->nsm = 1;
    g_nsm = ctx->nsm;
    make_tables(ctx->tab);
    {
        RotwTables rt;
        make_rotw_tables(rt);
        if (!rotw_tables_check(rt)) {  // cannot happen: the tables are fixed numbers
            fmmx_destroy(ctx);
            return FMMX_DEVICE_ERROR;
        }
        rotw_upload_f64(rt, ctx->stream);
        rotw_upload_f32(rt, ctx->stream);
    }
    upload_tables_exact(ctx->tab, ctx->stream);
    upload_tables_m2l(ctx->tab, ctx->stream);
    upload_tables_sweeps(ctx->tab, ctx->stream);
    upload_tables_mixed(ctx->tab, ctx->stream);
    build_swap(c.p, ctx->swap_host);
    if (ctx->swap_dev.ensure(ctx->swap_host.size()) != cudaSuccess ||
        cudaMemcpyAsync(ctx->swap_dev.p, ctx->swap_host.data(), ctx->swap_host.size() * sizeof(double),
                        cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        cudaGetLastError();
        fmmx_destroy(ctx);
        return FMMX_DEVICE_ERROR;
    }
    *out = ctx;
    return FMMX_OK;
}

void fmmx_destroy(fmmx_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->cfg.device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->stream2) cudaStreamSynchronize(ctx->stream2);
    ctx->drop_graph();
    for (int i = 0; i < 16; ++i)
        if (ctx->ev[i]) cudaEventDestroy(ctx->ev[i]);
    for (int i = 0; i < 3; ++i)
        if (ctx->fork[i]) cudaEventDestroy(ctx->fork[i]);
    if (ctx->stream2) cudaStreamDestroy(ctx->stream2);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char* fmmx_last_error(const fmmx_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

fmmx_status fmmx_build_device(fmmx_ctx* ctx, size_t n, const double* d_pos, const double* d_mass) {
    if (!ctx) return FMMX_INVALID_ARG;
    BudgetScope bscope(&ctx->budget);
    if (!d_pos || !d_mass) return fail(ctx, FMMX_INVALID_ARG, "null input");
    cudaSetDevice(ctx->cfg.device);
    return finish(ctx, build_impl(ctx, n, d_pos, d_mass));
}

fmmx_status fmmx_build(fmmx_ctx* ctx, size_t n, const double* pos, const double* mass) {
    if (!ctx) return FMMX_INVALID_ARG;
    BudgetScope bscope(&ctx->budget);
    if (!pos || !mass) return fail(ctx, FMMX_INVALID_ARG, "null input");
    if (n == 0) return fail(ctx, FMMX_INVALID_ARG, "empty input (the reference asserts !parts.is_empty(), tree.rs:95)");
    cudaSetDevice(ctx->cfg.device);
    if (ctx->pos_in.ensure(3 * n) != cudaSuccess || ctx->mass_in.ensure(n) != cudaSuccess)
        return fail(ctx, FMMX_OUT_OF_MEMORY, "input buffers");
    cudaStream_t s = ctx->stream;
    if (cudaMemcpyAsync(ctx->pos_in.p, pos, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(ctx->mass_in.p, mass, n * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess)
        return cuda_fail(ctx, cudaGetLastError(), "copy inputs");
    return finish(ctx, build_impl(ctx, n, ctx->pos_in.p, ctx->mass_in.p));
}

fmmx_status fmmx_build_ensemble_device(fmmx_ctx* ctx, size_t nsys, const uint64_t* offsets, const double* d_pos,
                                       const double* d_mass) {
    if (!ctx) return FMMX_INVALID_ARG;
    BudgetScope bscope(&ctx->budget);
    if (!d_pos || !d_mass || !offsets || nsys == 0 || nsys > (1u << 24)) return fail(ctx, FMMX_INVALID_ARG, "bad input");
    cudaSetDevice(ctx->cfg.device);
    return finish(ctx, build_impl(ctx, (size_t)offsets[nsys], d_pos, d_mass, (int)nsys, offsets));
}

fmmx_status fmmx_build_ensemble(fmmx_ctx* ctx, size_t nsys, const uint64_t* offsets, const double* pos,
                                const double* mass) {
    if (!ctx) return FMMX_INVALID_ARG;
    BudgetScope bscope(&ctx->budget);
    if (!pos || !mass || !offsets || nsys == 0 || nsys > (1u << 24)) return fail(ctx, FMMX_INVALID_ARG, "bad input");
    const size_t n = (size_t)offsets[nsys];
    if (n == 0) return fail(ctx, FMMX_INVALID_ARG, "empty input");
    cudaSetDevice(ctx->cfg.device);
    if (ctx->pos_in.ensure(3 * n) != cudaSuccess || ctx->mass_in.ensure(n) != cudaSuccess)
        return fail(ctx, FMMX_OUT_OF_MEMORY, "input buffers");
    cudaStream_t s = ctx->stream;
    if (cudaMemcpyAsync(ctx->pos_in.p, pos, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(ctx->mass_in.p, mass, n * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess)
        return cuda_fail(ctx, cudaGetLastError(), "copy inputs");
    return finish(ctx, build_impl(ctx, n, ctx->pos_in.p, ctx->mass_in.p, (int)nsys, offsets));
}

fmmx_status fmmx_evaluate_device(fmmx_ctx* ctx, const double* d_pos, const double* d_mass, double* d_acc,
                                 double* d_pot) {
    if (!ctx) return FMMX_INVALID_ARG;
    BudgetScope bscope(&ctx->budget);
    if (!d_acc) return fail(ctx, FMMX_INVALID_ARG, "null output");
    cudaSetDevice(ctx->cfg.device);
    if (!d_pot) {
        if (ctx->pot_out.ensure(ctx->n) != cudaSuccess) return fail(ctx, FMMX_OUT_OF_MEMORY, "pot buffer");
        d_pot = ctx->pot_out.p;
    }
    return finish(ctx, evaluate_impl(ctx, d_pos, d_mass, d_acc, d_pot));
}

static constexpr int kGraphMinUses = 2;

fmmx_status fmmx_leapfrog_device(fmmx_ctx* ctx, double* d_pos, double* d_vel, const double* d_mass, double* d_acc,
                                 double* d_pot, double dt, int nsteps, int scheme, int refresh_every) {
    if (!ctx) return FMMX_INVALID_ARG;
    BudgetScope bscope(&ctx->budget);
    if (!d_pos || !d_vel || !d_mass || !d_acc || nsteps < 0 || refresh_every < 1 || (scheme != 0 && scheme != 1))
        return fail(ctx, FMMX_INVALID_ARG, "bad leapfrog arguments");
    if (!ctx->built) return fail(ctx, FMMX_NOT_BUILT, "leapfrog needs a built tree (build + evaluate first)");
    cudaSetDevice(ctx->cfg.device);
    cudaStream_t s = ctx->stream;
    const size_t n = ctx->n;
    if (!d_pot) {
        if (ctx->pot_out.ensure(n) != cudaSuccess) return fail(ctx, FMMX_OUT_OF_MEMORY, "pot buffer");
        d_pot = ctx->pot_out.p;
    }
    const unsigned g = grid_for(3 * n, 256);
    const void* key[5] = {d_pos, d_vel, d_mass, d_acc, d_pot};
    for (int step = 0; step < nsteps; ++step) {
        const bool rebuild = (ctx->steps_since_build + 1) >= refresh_every;
        // A step on a reused tree is the same sequence of launches every time:
        // record it once as a CUDA graph and replay it (one launch instead of
        // about 30). Not on the legacy default stream, which cannot be captured.
        // A recording costs more than a launched step, so a tree is recorded
        // only when the refresh cadence will replay it at least
        // kGraphMinUses times (steps_since_build counts the reuse steps done).
        const bool same = ctx->step_graph && ctx->graph_dt == dt && ctx->graph_scheme == scheme &&
                          std::equal(key, key + 5, ctx->graph_key);
        const int reuse_left = refresh_every - 1 - ctx->steps_since_build;
        if (!rebuild && ctx->cfg.use_graphs && s != nullptr && ctx->lists_valid &&
            (same || reuse_left >= kGraphMinUses)) {
            if (!same) {
                ctx->drop_graph();
                const bool ev_saved = ctx->events;
                ctx->events = false;
                cudaGraph_t graph = nullptr;
                fmmx_status st = FMMX_OK;
                if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
                    st = cuda_fail(ctx, cudaGetLastError(), "graph capture");
                if (st == FMMX_OK) {
                    if (scheme == 0) {
                        k_kick<<<g, 256, 0, s>>>(3 * n, d_vel, d_acc, 0.5 * dt);
                        k_drift<<<g, 256, 0, s>>>(3 * n, d_pos, d_vel, dt);
                    } else {
                        k_drift<<<g, 256, 0, s>>>(3 * n, d_pos, d_vel, 0.5 * dt);
                    }
                    st = evaluate_impl(ctx, d_pos, d_mass, d_acc, d_pot, true, true);
                    if (scheme == 0) {
                        k_kick<<<g, 256, 0, s>>>(3 * n, d_vel, d_acc, 0.5 * dt);
                    } else {
                        k_kick<<<g, 256, 0, s>>>(3 * n, d_vel, d_acc, dt);
                        k_drift<<<g, 256, 0, s>>>(3 * n, d_pos, d_vel, 0.5 * dt);
                    }
                    const cudaError_t ec = cudaStreamEndCapture(s, &graph);
                    if (st == FMMX_OK && ec != cudaSuccess) st = cuda_fail(ctx, ec, "graph capture");
                }
                ctx->events = ev_saved;
                if (st == FMMX_OK && cudaGraphInstantiate(&ctx->step_graph, graph, 0) != cudaSuccess) {
                    ctx->step_graph = nullptr;
                    st = cuda_fail(ctx, cudaGetLastError(), "graph instantiate");
                }
                if (graph) cudaGraphDestroy(graph);
                if (st != FMMX_OK) return st;
                std::copy(key, key + 5, ctx->graph_key);
                ctx->graph_dt = dt;
                ctx->graph_scheme = scheme;
            }
            if (cudaGraphLaunch(ctx->step_graph, s) != cudaSuccess) return cuda_fail(ctx, cudaGetLastError(), "graph");
            ctx->steps_since_build++;
            continue;
        }
        if (scheme == 0) {  // kick-drift-kick; d_acc holds the forces at d_pos
            k_kick<<<g, 256, 0, s>>>(3 * n, d_vel, d_acc, 0.5 * dt);
            k_drift<<<g, 256, 0, s>>>(3 * n, d_pos, d_vel, dt);
        } else {  // drift-kick-drift (crates/fmm/tests/energy_gate.rs:156-177)
            k_drift<<<g, 256, 0, s>>>(3 * n, d_pos, d_vel, 0.5 * dt);
        }
        if (cudaGetLastError() != cudaSuccess) return fail(ctx, FMMX_DEVICE_ERROR, "leapfrog update");
        fmmx_status st;
        if (rebuild) {
            if (ctx->nsys == 1) {
                st = build_impl(ctx, n, d_pos, d_mass);
            } else {
                std::vector<uint64_t> off(ctx->sys_off_host);
                st = build_impl(ctx, n, d_pos, d_mass, ctx->nsys, off.data());
            }
            if (st != FMMX_OK) return finish(ctx, st);
            ctx->steps_since_build = 0;
            st = evaluate_impl(ctx, d_pos, d_mass, d_acc, d_pot, false);
        } else {
            ctx->steps_since_build++;
            st = evaluate_impl(ctx, d_pos, d_mass, d_acc, d_pot, true);
        }
        if (st != FMMX_OK) return finish(ctx, st);
        if (scheme == 0) {
            k_kick<<<g, 256, 0, s>>>(3 * n, d_vel, d_acc, 0.5 * dt);
        } else {
            k_kick<<<g, 256, 0, s>>>(3 * n, d_vel, d_acc, dt);
            k_drift<<<g, 256, 0, s>>>(3 * n, d_pos, d_vel, 0.5 * dt);
        }
        if (cudaGetLastError() != cudaSuccess) return fail(ctx, FMMX_DEVICE_ERROR, "leapfrog update");
    }
    if (cudaStreamSynchronize(s) != cudaSuccess) return cuda_fail(ctx, cudaGetLastError(), "leapfrog");
    return FMMX_OK;
}

fmmx_status fmmx_kdk_step_device(fmmx_ctx* ctx, double* d_pos, double* d_vel, const double* d_mass, double* d_acc,
                                 double* d_pot, const double* d_dt, size_t nsys, const uint64_t* offsets,
                                 int rebuild) {
    if (!ctx) return FMMX_INVALID_ARG;
    BudgetScope bscope(&ctx->budget);
    if (!d_pos || !d_vel || !d_mass || !d_acc || !d_dt) return fail(ctx, FMMX_INVALID_ARG, "null pointer");
    if (!offsets && !ctx->built) return fail(ctx, FMMX_NOT_BUILT, "no tree to step on: give offsets");
    if (offsets && (nsys == 0 || nsys > (1u << 24))) return fail(ctx, FMMX_INVALID_ARG, "bad system count");
    cudaSetDevice(ctx->cfg.device);
    cudaStream_t s = ctx->stream;
    const size_t n = offsets ? (size_t)offsets[nsys] : ctx->n;
    if (n == 0) return fail(ctx, FMMX_INVALID_ARG, "empty input");
    if (!d_pot) {
        if (ctx->pot_out.ensure(n) != cudaSuccess) return fail(ctx, FMMX_OUT_OF_MEMORY, "pot buffer");
        d_pot = ctx->pot_out.p;
    }
    const unsigned g = grid_for(3 * n, 256);
    k_kick_rows<<<g, 256, 0, s>>>(3 * n, d_vel, d_acc, d_dt, 0.5);
    k_drift_rows<<<g, 256, 0, s>>>(3 * n, d_pos, d_vel, d_dt);
    if (cudaGetLastError() != cudaSuccess) return fail(ctx, FMMX_DEVICE_ERROR, "kick/drift");
    fmmx_status st = FMMX_OK;
    const bool build = offsets != nullptr || rebuild || !ctx->lists_valid;
    if (build) {
        if (offsets) {
            st = nsys == 1 ? build_impl(ctx, n, d_pos, d_mass) : build_impl(ctx, n, d_pos, d_mass, (int)nsys, offsets);
        } else if (ctx->nsys == 1) {
            st = build_impl(ctx, n, d_pos, d_mass);
        } else {
            std::vector<uint64_t> off(ctx->sys_off_host);
            st = build_impl(ctx, n, d_pos, d_mass, ctx->nsys, off.data());
        }
        if (st != FMMX_OK) return finish(ctx, st);
        ctx->steps_since_build = 0;
        st = evaluate_impl(ctx, d_pos, d_mass, d_acc, d_pot, false);
    } else {
        ctx->steps_since_build++;
        st = evaluate_impl(ctx, d_pos, d_mass, d_acc, d_pot, true);
    }
    if (st != FMMX_OK) return finish(ctx, st);
    k_kick_rows<<<g, 256, 0, s>>>(3 * n, d_vel, d_acc, d_dt, 0.5);
    if (cudaGetLastError() != cudaSuccess) return fail(ctx, FMMX_DEVICE_ERROR, "kick");
    return FMMX_OK;
}

fmmx_status fmmx_evaluate(fmmx_ctx* ctx, const double* pos, const double* mass, double* acc, double* pot) {
    if (!ctx) return FMMX_INVALID_ARG;
    BudgetScope bscope(&ctx->budget);
    if (!acc) return fail(ctx, FMMX_INVALID_ARG, "null output");
    if (!ctx->built) return fail(ctx, FMMX_NOT_BUILT, "evaluate before build");
    cudaSetDevice(ctx->cfg.device);
    const size_t n = ctx->n;
    cudaStream_t s = ctx->stream;
    const double* dp = nullptr;
    const double* dm = nullptr;
    if (pos || mass) {
        if (ctx->pos_in.ensure(3 * n) != cudaSuccess || ctx->mass_in.ensure(n) != cudaSuccess)
            return fail(ctx, FMMX_OUT_OF_MEMORY, "input buffers");
        if (pos) {
            if (cudaMemcpyAsync(ctx->pos_in.p, pos, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess)
                return cuda_fail(ctx, cudaGetLastError(), "copy inputs");
            dp = ctx->pos_in.p;
        }
        if (mass) {
            if (cudaMemcpyAsync(ctx->mass_in.p, mass, n * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess)
                return cuda_fail(ctx, cudaGetLastError(), "copy inputs");
            dm = ctx->mass_in.p;
        }
    }
    if (ctx->acc_out.ensure(3 * n) != cudaSuccess || ctx->pot_out.ensure(n) != cudaSuccess)
        return fail(ctx, FMMX_OUT_OF_MEMORY, "output buffers");
    fmmx_status st = evaluate_impl(ctx, dp, dm, ctx->acc_out.p, ctx->pot_out.p);
    if (st != FMMX_OK) return finish(ctx, st);
    if (cudaMemcpyAsync(acc, ctx->acc_out.p, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return cuda_fail(ctx, cudaGetLastError(), "copy outputs");
    if (pot && cudaMemcpyAsync(pot, ctx->pot_out.p, n * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return cuda_fail(ctx, cudaGetLastError(), "copy outputs");
    if (cudaStreamSynchronize(s) != cudaSuccess) return cuda_fail(ctx, cudaGetLastError(), "evaluate");
    return FMMX_OK;
}

fmmx_status fmmx_synchronize(fmmx_ctx* ctx) {
    if (!ctx) return FMMX_INVALID_ARG;
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "synchronize");
    return FMMX_OK;
}

fmmx_status fmmx_get_stats(const fmmx_ctx* ctx, fmmx_stats* out) {
    if (!ctx || !out) return FMMX_INVALID_ARG;
    *out = ctx->st;
    out->n = ctx->n;
    out->n_cells = ctx->nc;
    out->n_leaves = ctx->nleaves;
    out->n_levels = ctx->nlevels;
    out->n_m2l = ctx->n_m2l;
    out->n_p2p = ctx->n_p2p;
    out->walk_pops = ctx->pops;
    out->p2p_interactions = ctx->p2p_inter;
    out->m2l_directed = 2ull * (uint64_t)ctx->n_m2l;
    out->kernel_launches = ctx->launches;
    out->walk_retries = (uint64_t)ctx->walk_retries;
    out->device_bytes = ctx->budget.used;
    return FMMX_OK;
}

fmmx_status fmmx_export_tree(const fmmx_ctx* cctx, uint32_t* order, uint64_t* keys_sorted, uint32_t* cell_info,
                             int32_t* children, double* cen, double* mass, double* rho) {
    fmmx_ctx* ctx = const_cast<fmmx_ctx*>(cctx);
    if (!ctx) return FMMX_INVALID_ARG;
    if (!ctx->built) return fail(ctx, FMMX_NOT_BUILT, "export before build");
    cudaSetDevice(ctx->cfg.device);
    CK(cudaStreamSynchronize(ctx->stream), "sync");
    const size_t n = ctx->n, nc = ctx->nc;
    if (order) CK(cudaMemcpy(order, ctx->order.p, n * 4, cudaMemcpyDeviceToHost), "copy");
    if (keys_sorted) CK(cudaMemcpy(keys_sorted, ctx->keys_sorted.p, n * 8, cudaMemcpyDeviceToHost), "copy");
    if (cell_info) {
        std::vector<uint32_t> f(nc), c(nc);
        std::vector<uint8_t> lv(nc), lf(nc);
        CK(cudaMemcpy(f.data(), ctx->c_first.p, nc * 4, cudaMemcpyDeviceToHost), "copy");
        CK(cudaMemcpy(c.data(), ctx->c_count.p, nc * 4, cudaMemcpyDeviceToHost), "copy");
        CK(cudaMemcpy(lv.data(), ctx->c_level.p, nc, cudaMemcpyDeviceToHost), "copy");
        CK(cudaMemcpy(lf.data(), ctx->c_leaf.p, nc, cudaMemcpyDeviceToHost), "copy");
        for (size_t i = 0; i < nc; ++i) {
            cell_info[4 * i] = f[i];
            cell_info[4 * i + 1] = c[i];
            cell_info[4 * i + 2] = lv[i];
            cell_info[4 * i + 3] = lf[i];
        }
    }
    if (children) CK(cudaMemcpy(children, ctx->c_child.p, nc * 8 * 4, cudaMemcpyDeviceToHost), "copy");
    if (cen) {
        std::vector<double> a(nc), b(nc), c(nc);
        CK(cudaMemcpy(a.data(), ctx->c_cx.p, nc * 8, cudaMemcpyDeviceToHost), "copy");
        CK(cudaMemcpy(b.data(), ctx->c_cy.p, nc * 8, cudaMemcpyDeviceToHost), "copy");
        CK(cudaMemcpy(c.data(), ctx->c_cz.p, nc * 8, cudaMemcpyDeviceToHost), "copy");
        for (size_t i = 0; i < nc; ++i) {
            cen[3 * i] = a[i];
            cen[3 * i + 1] = b[i];
            cen[3 * i + 2] = c[i];
        }
    }
    if (mass) CK(cudaMemcpy(mass, ctx->c_mass.p, nc * 8, cudaMemcpyDeviceToHost), "copy");
    if (rho) CK(cudaMemcpy(rho, ctx->c_rho.p, nc * 8, cudaMemcpyDeviceToHost), "copy");
    return FMMX_OK;
}

fmmx_status fmmx_export_lists(const fmmx_ctx* cctx, uint32_t* m2l, uint32_t* p2p) {
    fmmx_ctx* ctx = const_cast<fmmx_ctx*>(cctx);
    if (!ctx) return FMMX_INVALID_ARG;
    if (!ctx->evaluated) return fail(ctx, FMMX_NOT_BUILT, "export before evaluate");
    cudaSetDevice(ctx->cfg.device);
    CK(cudaStreamSynchronize(ctx->stream), "sync");
    if (m2l && ctx->n_m2l) CK(cudaMemcpy(m2l, ctx->m2l.p, (size_t)ctx->n_m2l * 8, cudaMemcpyDeviceToHost), "copy");
    if (p2p && ctx->n_p2p) CK(cudaMemcpy(p2p, ctx->p2p.p, (size_t)ctx->n_p2p * 8, cudaMemcpyDeviceToHost), "copy");
    return FMMX_OK;
}

fmmx_status fmmx_export_expansions(const fmmx_ctx* cctx, double* moments, double* locals, double* pows, double* f,
                                   double* fmin) {
    fmmx_ctx* ctx = const_cast<fmmx_ctx*>(cctx);
    if (!ctx) return FMMX_INVALID_ARG;
    if (!ctx->evaluated) return fail(ctx, FMMX_NOT_BUILT, "export before evaluate");
    cudaSetDevice(ctx->cfg.device);
    CK(cudaStreamSynchronize(ctx->stream), "sync");
    const size_t nc = ctx->nc, dim = dimp(ctx->cfg.p);
    if (moments) CK(cudaMemcpy(moments, ctx->moments.p, nc * dim * 16, cudaMemcpyDeviceToHost), "copy");
    if (locals) CK(cudaMemcpy(locals, ctx->locals.p, nc * dim * 16, cudaMemcpyDeviceToHost), "copy");
    if (pows) CK(cudaMemcpy(pows, ctx->pows.p, nc * (ctx->cfg.p + 1) * 8, cudaMemcpyDeviceToHost), "copy");
    if (f && ctx->cfg.mac_mode == FMMX_MAC_DEHNEN) CK(cudaMemcpy(f, ctx->f.p, ctx->n * 8, cudaMemcpyDeviceToHost), "copy");
    if (fmin && ctx->cfg.mac_mode == FMMX_MAC_DEHNEN)
        CK(cudaMemcpy(fmin, ctx->fmin.p, nc * 8, cudaMemcpyDeviceToHost), "copy");
    return FMMX_OK;
}

fmmx_status fmmx_direct_targets(int device, size_t n, const double* pos, const double* mass, double softening,
                                size_t nt, const uint32_t* targets, double* acc, double* pot, double* fscale) {
    if (!pos || !mass || !targets || !acc || n == 0) return FMMX_INVALID_ARG;
    if (nt == 0) return FMMX_OK;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return FMMX_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) return FMMX_INVALID_ARG;
    for (size_t q = 0; q < nt; ++q)
        if (targets[q] >= n) return FMMX_INVALID_ARG;
    cudaSetDevice(device);
    const int nsplit = 32;
    double *dpos = nullptr, *dmass = nullptr, *part = nullptr, *dacc = nullptr, *dpot = nullptr, *df = nullptr;
    uint32_t* dt = nullptr;
    fmmx_status st = FMMX_OK;
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&dpos, 3 * n * 8) != cudaSuccess || cudaMalloc(&dmass, n * 8) != cudaSuccess ||
        cudaMalloc(&dt, nt * 4) != cudaSuccess || cudaMalloc(&part, nsplit * nt * 5 * 8) != cudaSuccess ||
        cudaMalloc(&dacc, nt * 3 * 8) != cudaSuccess || cudaMalloc(&dpot, nt * 8) != cudaSuccess ||
        cudaMalloc(&df, nt * 8) != cudaSuccess) {
        st = FMMX_OUT_OF_MEMORY;
    } else {
        cudaMemcpyAsync(dpos, pos, 3 * n * 8, cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(dmass, mass, n * 8, cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(dt, targets, nt * 4, cudaMemcpyHostToDevice, s);
        dim3 g((unsigned)((nt + 127) / 128), nsplit);
        k_direct_targets<<<g, 128, 0, s>>>(dpos, dmass, n, dt, nt, softening * softening, part);
        k_direct_reduce<<<grid_for(nt, 128), 128, 0, s>>>(part, nsplit, nt, dacc, dpot, df);
        cudaMemcpyAsync(acc, dacc, nt * 3 * 8, cudaMemcpyDeviceToHost, s);
        if (pot) cudaMemcpyAsync(pot, dpot, nt * 8, cudaMemcpyDeviceToHost, s);
        if (fscale) cudaMemcpyAsync(fscale, df, nt * 8, cudaMemcpyDeviceToHost, s);
        if (cudaStreamSynchronize(s) != cudaSuccess || cudaGetLastError() != cudaSuccess) st = FMMX_DEVICE_ERROR;
    }
    for (void* q : {(void*)dpos, (void*)dmass, (void*)dt, (void*)part, (void*)dacc, (void*)dpot, (void*)df})
        if (q) cudaFree(q);
    if (s) cudaStreamDestroy(s);
    return st;
}

}  // extern "C"
