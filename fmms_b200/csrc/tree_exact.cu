// Bit-exact stages of the engine: bounding box, Morton keys, octree topology,
// cell geometry, P2M/M2M, multipole power, the f pre-pass and the dual tree
// walk with its MAC.
//
// Everything here feeds the multipole acceptance decisions, so it reproduces
// the reference's FP64 operation order exactly and this file is compiled with
// --fmad=false (the reference never contracts a*b+c into an FMA). sqrt and
// division are IEEE round-to-nearest in CUDA double precision, as in the
// reference. Citations are file:line in crates/fmm/src.
#include <float.h>

#include "common.cuh"
#include "kernels.h"

namespace fmmx {

// The order tables in global memory: the kernels read them with lane-
// dependent indices (a lane per order m or per degree), which the constant
// cache would serialise over the distinct addresses; global loads are served
// from L1 in parallel.
static __device__ OrderTables g_tab;

void upload_tables_exact(const OrderTables& t, cudaStream_t s) {
    cudaMemcpyToSymbolAsync(g_tab, &t, sizeof(t), 0, cudaMemcpyHostToDevice, s);
}

// ------------------------------------------------------------ bounding box
// tree.rs:98-111. min/max are exact, so any reduction order gives the same box.
__global__ void k_bbox_partial(const double* __restrict__ pos, size_t n, double* __restrict__ part,
                               int* __restrict__ bad) {
    double lo[3] = {INFINITY, INFINITY, INFINITY};
    double hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    int nonfinite = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            double v = pos[3 * i + d];
            nonfinite |= !isfinite(v);
            lo[d] = fmin(lo[d], v);
            hi[d] = fmax(hi[d], v);
        }
    }
    __shared__ double s[6][256];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        s[d][threadIdx.x] = lo[d];
        s[3 + d][threadIdx.x] = hi[d];
    }
    if (nonfinite) atomicOr(bad, 1);
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                s[d][threadIdx.x] = fmin(s[d][threadIdx.x], s[d][threadIdx.x + w]);
                s[3 + d][threadIdx.x] = fmax(s[3 + d][threadIdx.x], s[3 + d][threadIdx.x + w]);
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int d = 0; d < 6; ++d) part[blockIdx.x * 6 + d] = s[d][0];
}

// box = {lo[3], hi[3], side, inv_side}; side as tree.rs:107-111.
// One warp: lanes reduce strided partials, then a shuffle reduction (min and
// max are exact, so the order does not matter).
__global__ void k_bbox_final(const double* __restrict__ part, int nparts, double* __restrict__ box) {
    if (blockIdx.x != 0 || threadIdx.x >= 32) return;
    const int lane = threadIdx.x;
    double lo[3] = {INFINITY, INFINITY, INFINITY};
    double hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int b = lane; b < nparts; b += 32)
        for (int d = 0; d < 3; ++d) {
            lo[d] = fmin(lo[d], part[b * 6 + d]);
            hi[d] = fmax(hi[d], part[b * 6 + 3 + d]);
        }
    for (int o = 16; o > 0; o >>= 1)
        for (int d = 0; d < 3; ++d) {
            lo[d] = fmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
            hi[d] = fmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
        }
    if (lane != 0) return;
    double side = fmax(fmax(fmax(hi[0] - lo[0], hi[1] - lo[1]), hi[2] - lo[2]), DBL_MIN);
    for (int d = 0; d < 3; ++d) {
        box[d] = lo[d];
        box[3 + d] = hi[d];
    }
    box[6] = side;
    box[7] = 1.0 / side;
}

// Forest of independent systems (segments [off[s], off[s+1]) of the input):
// one block per system reduces its own box.
__global__ void k_bbox_seg(const double* __restrict__ pos, const uint64_t* __restrict__ off,
                           double* __restrict__ box, int* __restrict__ bad) {
    const int sys = blockIdx.x;
    const uint64_t b = off[sys], e = off[sys + 1];
    double lo[3] = {INFINITY, INFINITY, INFINITY};
    double hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    int nonfinite = 0;
    for (uint64_t i = b + threadIdx.x; i < e; i += blockDim.x) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            double v = pos[3 * i + d];
            nonfinite |= !isfinite(v);
            lo[d] = fmin(lo[d], v);
            hi[d] = fmax(hi[d], v);
        }
    }
    __shared__ double sh[6][256];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        sh[d][threadIdx.x] = lo[d];
        sh[3 + d][threadIdx.x] = hi[d];
    }
    if (nonfinite) atomicOr(bad, 1);
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                sh[d][threadIdx.x] = fmin(sh[d][threadIdx.x], sh[d][threadIdx.x + w]);
                sh[3 + d][threadIdx.x] = fmax(sh[3 + d][threadIdx.x], sh[3 + d][threadIdx.x + w]);
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double* bx = box + 8 * sys;
        for (int d = 0; d < 3; ++d) {
            bx[d] = sh[d][0];
            bx[3 + d] = sh[3 + d][0];
        }
        const double side = fmax(fmax(fmax(bx[3] - bx[0], bx[4] - bx[1]), bx[5] - bx[2]), DBL_MIN);
        bx[6] = side;
        bx[7] = 1.0 / side;
    }
}

// ------------------------------------------------------------ Morton keys
// dilate, tree.rs:28-35
__device__ __forceinline__ uint64_t dilate21(uint64_t x) {
    x &= (1ULL << FMMX_BITS) - 1;
    x = (x | (x << 32)) & 0x001f00000000ffffULL;
    x = (x | (x << 16)) & 0x001f0000ff0000ffULL;
    x = (x | (x << 8)) & 0x100f00f00f00f00fULL;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ULL;
    return (x | (x << 2)) & 0x1249249249249249ULL;
}

// morton_key, tree.rs:37-46: every axis is quantised against lo[0].
__device__ __forceinline__ uint64_t quant(double c, double lo0, double inv_side) {
    double v = (c - lo0) * inv_side;
    if (v != v) return 0;
    v = v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v);
    return (uint64_t)(v * (double)((1ULL << FMMX_BITS) - 1));
}

__global__ void k_keys(const double* __restrict__ pos, size_t n, const double* __restrict__ box,
                       uint64_t* __restrict__ keys, uint32_t* __restrict__ idx) {
    const double lo0 = box[0], inv = box[7];
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        uint64_t k = dilate21(quant(pos[3 * i + 2], lo0, inv));
        k |= dilate21(quant(pos[3 * i + 1], lo0, inv)) << 1;
        k |= dilate21(quant(pos[3 * i + 0], lo0, inv)) << 2;
        keys[i] = k;
        idx[i] = (uint32_t)i;
    }
}

// Keys of a forest: each body is quantised in its own system's box.
__global__ void k_keys_seg(const double* __restrict__ pos, size_t n, const uint64_t* __restrict__ off, int nsys,
                           const double* __restrict__ box, uint64_t* __restrict__ keys, uint32_t* __restrict__ idx) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        int lo = 0, hi = nsys;  // last system with off[sys] <= i
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (off[mid] <= i) lo = mid;
            else hi = mid;
        }
        const double lo0 = box[8 * lo], inv = box[8 * lo + 7];
        uint64_t k = dilate21(quant(pos[3 * i + 2], lo0, inv));
        k |= dilate21(quant(pos[3 * i + 1], lo0, inv)) << 1;
        k |= dilate21(quant(pos[3 * i + 0], lo0, inv)) << 2;
        keys[i] = k;
        idx[i] = (uint32_t)i;
    }
}

// Bodies::from_parts / gather_into, bodies.rs:27-60: slot k <- particle order[k].
__global__ void k_gather(const double* __restrict__ pos, const double* __restrict__ mass,
                         const uint32_t* __restrict__ order, size_t n, double* __restrict__ x, double* __restrict__ y,
                         double* __restrict__ z, double* __restrict__ m) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        uint32_t id = order[k];
        x[k] = pos[3 * (size_t)id];
        y[k] = pos[3 * (size_t)id + 1];
        z[k] = pos[3 * (size_t)id + 2];
        m[k] = mass[id];
    }
}

// ------------------------------------------------------------ topology
// The reference builds cells by depth-first recursion (build_rec,
// tree.rs:404-445). Here nodes are created level by level from the sorted
// keys (every node of a level in parallel, its octant ranges by binary search
// on the key digit), then renumbered into depth-first pre-order: with ranges
// nested or disjoint, pre-order is the order of (first slot, level).
__global__ void k_tree_init(TmpNodes t, uint32_t n, int* __restrict__ lvl) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        t.first[0] = 0;
        t.count[0] = n;
        t.parent[0] = -1;
        t.oct[0] = 0;
        t.level[0] = 0;
        lvl[LV_START + 0] = 0;
        lvl[LV_COUNT + 0] = 1;
    }
}

// One root per system.
__global__ void k_tree_init_forest(TmpNodes t, const uint64_t* __restrict__ off, int nsys, int* __restrict__ lvl) {
    for (int sys = blockIdx.x * blockDim.x + threadIdx.x; sys < nsys; sys += gridDim.x * blockDim.x) {
        t.first[sys] = (uint32_t)off[sys];
        t.count[sys] = (uint32_t)(off[sys + 1] - off[sys]);
        t.parent[sys] = -1;
        t.oct[sys] = 0;
        t.level[sys] = 0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        lvl[LV_START + 0] = 0;
        lvl[LV_COUNT + 0] = nsys;
    }
}

// Box size of every cell: a root gets its system's box side, a child half its
// parent's. Level 0 lists the roots in system order.
__global__ void k_cell_h(const int32_t* __restrict__ level_cells, int lstart, int lcnt, const int32_t* __restrict__ parent,
                         const double* __restrict__ box, double* __restrict__ h) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < lcnt; j += gridDim.x * blockDim.x) {
        const int c = level_cells[lstart + j];
        const int par = parent[c];
        h[c] = par < 0 ? box[8 * j + 6] : 0.5 * h[par];
    }
}

// Walk seeds: the self pair of every root.
__global__ void k_walk_init(const int32_t* __restrict__ level_cells, int nroots, uint2* __restrict__ front) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nroots; j += gridDim.x * blockDim.x) {
        const int r = level_cells[j];
        front[j] = make_uint2(r, r);
    }
}

__global__ void k_build_level(TmpNodes t, const uint64_t* __restrict__ keys, int L, long long n_leaf, uint32_t cap,
                              int* __restrict__ lvl, int* __restrict__ flags) {
    const int start = lvl[LV_START + L];
    const int cnt = lvl[LV_COUNT + L];
    const int next_start = start + cnt;
    if (blockIdx.x == 0 && threadIdx.x == 0) lvl[LV_START + L + 1] = next_start;
    if (flags[0]) return;  // capacity exceeded earlier: the host retries larger
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < cnt; j += gridDim.x * blockDim.x) {
        const int tt = start + j;
        if ((uint32_t)tt >= cap) break;
        const uint32_t f = t.first[tt], c = t.count[tt];
        const bool leaf = (long long)c <= n_leaf || L >= FMMX_MAXLEVEL;
        t.leaf[tt] = leaf ? 1 : 0;
        if (leaf) {
            atomicAdd(&flags[1], 1);  // leaf count
            continue;
        }
        const int shift = 3 * (FMMX_MAXLEVEL - (L + 1));
        const uint32_t end = f + c;
        uint32_t lo = f;
        for (uint32_t oct = 0; oct < 8; ++oct) {
            uint32_t a = lo, b = end;
            while (a < b) {  // first slot whose octant digit exceeds oct
                uint32_t mid = a + ((b - a) >> 1);
                uint32_t d = (uint32_t)((keys[mid] >> shift) & 7ULL);
                if (d <= oct) a = mid + 1;
                else b = mid;
            }
            const uint32_t hi = a;
            if (hi > lo) {
                int slot = atomicAdd(&lvl[LV_COUNT + L + 1], 1);
                uint32_t ct = (uint32_t)(next_start + slot);
                if (ct < cap) {
                    t.first[ct] = lo;
                    t.count[ct] = hi - lo;
                    t.parent[ct] = tt;
                    t.oct[ct] = (uint8_t)oct;
                    t.level[ct] = (uint8_t)(L + 1);
                } else {
                    atomicOr(&flags[0], 1);  // node capacity exceeded
                }
            }
            lo = hi;
        }
    }
}

__global__ void k_dfs_keys(TmpNodes t, int nc, uint64_t* __restrict__ key, uint32_t* __restrict__ val) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nc; i += gridDim.x * blockDim.x) {
        key[i] = ((uint64_t)t.first[i] << 5) | (uint64_t)t.level[i];
        val[i] = (uint32_t)i;
    }
}

__global__ void k_finalize_cells(const uint32_t* __restrict__ sorted_t, int nc, TmpNodes t,
                                 int32_t* __restrict__ new_id, CellsMut cells) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nc; i += gridDim.x * blockDim.x) {
        uint32_t tt = sorted_t[i];
        new_id[tt] = i;
        cells.first[i] = t.first[tt];
        cells.count[i] = t.count[tt];
        cells.level[i] = t.level[tt];
        cells.leaf[i] = t.leaf[tt];
    }
}

__global__ void k_link_cells(int nc, TmpNodes t, const int32_t* __restrict__ new_id, CellsMut cells,
                             int32_t* __restrict__ level_cells) {
    for (int tt = blockIdx.x * blockDim.x + threadIdx.x; tt < nc; tt += gridDim.x * blockDim.x) {
        int c = new_id[tt];
        level_cells[tt] = c;
        int par = t.parent[tt];
        if (par >= 0) {
            int pc = new_id[par];
            cells.child[8 * pc + t.oct[tt]] = c;
            cells.parent[c] = pc;
        } else {
            cells.parent[c] = -1;
        }
    }
}

// slot -> leaf cell, for the L2P stage
__global__ void k_body_leaf(int nc, const uint32_t* __restrict__ first, const uint32_t* __restrict__ count,
                            const uint8_t* __restrict__ leaf, int32_t* __restrict__ body_leaf) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int c = warp; c < nc; c += nwarps) {
        if (!leaf[c]) continue;
        uint32_t f = first[c], e = first[c] + count[c];
        for (uint32_t k = f + lane; k < e; k += 32) body_leaf[k] = c;
    }
}

// ------------------------------------------------------------ geometry
__device__ __forceinline__ double dist3(double ax, double ay, double az, double bx, double by, double bz) {
    double dx = ax - bx, dy = ay - by, dz = az - bz;
    return sqrt(dx * dx + dy * dy + dz * dz);
}
__device__ __forceinline__ double dist2_3(double ax, double ay, double az, double bx, double by, double bz) {
    double dx = ax - bx, dy = ay - by, dz = az - bz;
    return dx * dx + dy * dy + dz * dz;
}

// Item accessors for the Ritter sphere: leaf bodies (radius 0) or child cells.
struct LeafItems {
    const double *x, *y, *z;
    uint32_t first, count;
    __device__ int size() const { return (int)count; }
    __device__ void get(int i, double& cx, double& cy, double& cz, double& r) const {
        cx = x[first + i];
        cy = y[first + i];
        cz = z[first + i];
        r = 0.0;
    }
};
struct ChildItems {
    int ids[8];
    int nitems;
    const double *cx, *cy, *cz, *rho;
    __device__ int size() const { return nitems; }
    __device__ void get(int i, double& x, double& y, double& z, double& r) const {
        int c = ids[i];
        x = cx[c];
        y = cy[c];
        z = cz[c];
        r = rho[c];
    }
};

// Ritter grow/enclose sphere, tree.rs:290-389 (operation order kept).
template <class Items>
__device__ void ritter(const Items& it, double cen[3]) {
    int n = it.size();
    int a = 0, b = 0;
    double best = -1.0;
    double ax, ay, az, ar, qx, qy, qz, qr;
    it.get(a, ax, ay, az, ar);
    for (int i = 0; i < n; ++i) {
        it.get(i, qx, qy, qz, qr);
        double d2 = dist2_3(qx, qy, qz, ax, ay, az);
        if (d2 > best) { best = d2; b = i; }
    }
    a = b;
    best = -1.0;
    it.get(a, ax, ay, az, ar);
    for (int i = 0; i < n; ++i) {
        it.get(i, qx, qy, qz, qr);
        double d2 = dist2_3(qx, qy, qz, ax, ay, az);
        if (d2 > best) { best = d2; b = i; }
    }
    double pa[3], pb[3], ra, rb_;
    it.get(a, pa[0], pa[1], pa[2], ra);
    it.get(b, pb[0], pb[1], pb[2], rb_);
    double dir[3];
    {
        double dx = pb[0] - pa[0], dy = pb[1] - pa[1], dz = pb[2] - pa[2];
        double d = fmax(sqrt(dx * dx + dy * dy + dz * dz), DBL_MIN);
        dir[0] = dx / d; dir[1] = dy / d; dir[2] = dz / d;
    }
    double fa[3] = {pa[0] + ra * dir[0], pa[1] + ra * dir[1], pa[2] + ra * dir[2]};
    double fb[3] = {pb[0] - rb_ * dir[0], pb[1] - rb_ * dir[1], pb[2] - rb_ * dir[2]};
    double c[3] = {(fa[0] + fb[0]) * 0.5, (fa[1] + fb[1]) * 0.5, (fa[2] + fb[2]) * 0.5};
    double r = dist3(fa[0], fa[1], fa[2], fb[0], fb[1], fb[2]) * 0.5;
    for (int pass = 0; pass < 2; ++pass) {
        for (int i = 0; i < n; ++i) {
            it.get(i, qx, qy, qz, qr);
            double d = dist3(qx, qy, qz, c[0], c[1], c[2]);
            if (d + qr > r) {
                double dd = fmax(d, DBL_MIN);
                double dv[3] = {(qx - c[0]) / dd, (qy - c[1]) / dd, (qz - c[2]) / dd};
                double pp[3] = {qx + qr * dv[0], qy + qr * dv[1], qz + qr * dv[2]};
                double d_far = d + qr;
                double t = (d_far - r) / (2.0 * d_far);
                for (int k = 0; k < 3; ++k) c[k] += t * (pp[k] - c[k]);
                r = (d_far + r) * 0.5;
            }
        }
    }
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = 0; i < n; ++i) {
        it.get(i, qx, qy, qz, qr);
        double q[3] = {qx, qy, qz};
        for (int d = 0; d < 3; ++d) {
            lo[d] = fmin(lo[d], q[d] - qr);
            hi[d] = fmax(hi[d], q[d] + qr);
        }
    }
    double cb[3] = {(lo[0] + hi[0]) * 0.5, (lo[1] + hi[1]) * 0.5, (lo[2] + hi[2]) * 0.5};
    double rbb = 0.0;
    for (int i = 0; i < n; ++i) {
        it.get(i, qx, qy, qz, qr);
        rbb = fmax(rbb, dist3(qx, qy, qz, cb[0], cb[1], cb[2]) + qr);
    }
    if (rbb < r) {
        cen[0] = cb[0]; cen[1] = cb[1]; cen[2] = cb[2];
    } else {
        cen[0] = c[0]; cen[1] = c[1]; cen[2] = c[2];
    }
}

// Octree::geometry, tree.rs:152-227, one level at a time from the deepest.
__global__ void k_geometry_level(const int32_t* __restrict__ level_cells, int lstart, int lcnt, CellsMut cells,
                                 const double* __restrict__ x, const double* __restrict__ y,
                                 const double* __restrict__ z, const double* __restrict__ m, int center_mode) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < lcnt; j += gridDim.x * blockDim.x) {
        const int c = level_cells[lstart + j];
        double mass = 0.0, cen[3], rho = 0.0;
        if (cells.leaf[c]) {
            const uint32_t f = cells.first[c], e = f + cells.count[c];
            for (uint32_t k = f; k < e; ++k) mass += m[k];
            if (center_mode == FMMX_CENTER_COM) {
                double com[3] = {0.0, 0.0, 0.0};
                for (uint32_t k = f; k < e; ++k) {
                    com[0] += m[k] * x[k];
                    com[1] += m[k] * y[k];
                    com[2] += m[k] * z[k];
                }
                cen[0] = com[0] / mass;
                cen[1] = com[1] / mass;
                cen[2] = com[2] / mass;
            } else {
                LeafItems it{x, y, z, f, e - f};
                ritter(it, cen);
            }
            for (uint32_t k = f; k < e; ++k) rho = fmax(rho, dist3(x[k], y[k], z[k], cen[0], cen[1], cen[2]));
        } else {
            const int32_t* ch = cells.child + 8 * c;
            for (int o = 0; o < 8; ++o)
                if (ch[o] >= 0) mass += cells.mass[ch[o]];
            if (center_mode == FMMX_CENTER_COM) {
                double com[3] = {0.0, 0.0, 0.0};
                for (int o = 0; o < 8; ++o) {
                    int q = ch[o];
                    if (q < 0) continue;
                    com[0] += cells.mass[q] * cells.cx[q];
                    com[1] += cells.mass[q] * cells.cy[q];
                    com[2] += cells.mass[q] * cells.cz[q];
                }
                cen[0] = com[0] / mass;
                cen[1] = com[1] / mass;
                cen[2] = com[2] / mass;
            } else {
                ChildItems it;
                it.nitems = 0;
                for (int o = 0; o < 8; ++o)
                    if (ch[o] >= 0) it.ids[it.nitems++] = ch[o];
                it.cx = cells.cx;
                it.cy = cells.cy;
                it.cz = cells.cz;
                it.rho = cells.rho;
                ritter(it, cen);
            }
            for (int o = 0; o < 8; ++o) {
                int q = ch[o];
                if (q < 0) continue;
                rho = fmax(rho, cells.rho[q] + dist3(cells.cx[q], cells.cy[q], cells.cz[q], cen[0], cen[1], cen[2]));
            }
        }
        cells.mass[c] = mass;
        cells.cx[c] = cen[0];
        cells.cy[c] = cen[1];
        cells.cz[c] = cen[2];
        cells.rho[c] = rho;
    }
}

// ------------------------------------------------------------ upward pass
__device__ __forceinline__ void split_nm(int e, int& n, int& m) {
    int q = (int)sqrt((double)e);
    while (q * q > e) --q;
    while ((q + 1) * (q + 1) <= e) ++q;
    n = q;
    m = e - q * (q + 1);
}

// Υ column m for r = (dx,dy,dz), into u (full table when mirror is set):
// upsilon_table_into, harmonic.rs:141-173, operation order kept.
__device__ __forceinline__ void upsilon_column(double dx, double dy, double dz, double r2, int p, int m, zd* u) {
    zd d = mk(1.0, 0.0);
    for (int j = 1; j <= m; ++j) d = zmul(zscale(mk(dx, dy), g_tab.inv2m[j]), d);
    u[cidx(m, m)] = d;
    zd u1 = d, u2 = mk(0.0, 0.0);
    for (int n = m + 1; n <= p; ++n) {
        double a = (double)(2 * n - 1) * dz;
        zd t = zscale(u1, a);
        if (n >= m + 2) t = zsub(t, zscale(u2, r2));
        zd un = zscale(t, g_tab.invc[n][m]);
        u[cidx(n, m)] = un;
        u2 = u1;
        u1 = un;
    }
    if (m > 0) {
        double sgn = (m % 2 == 0) ? 1.0 : -1.0;
        for (int n = m; n <= p; ++n) u[cidx(n, -m)] = zscale(zconj(u[cidx(n, m)]), sgn);
    }
}

// Shared memory of k_upward_exact per warp: the cell's accumulator (dim
// complex), then either the Υ table of an M2M child offset (dim complex) or,
// for a leaf's P2M, the m >= 0 Υ tables of a round of B bodies, entry-major
// in separate real and imaginary arrays of stride B + 1 (conflict-free both
// when a lane writes its body's table and when lanes read one body's
// entries).
__host__ __device__ size_t upward_exact_smem_per_warp(int p) {
    const int B = p2m_round(p), H = (p + 1) * (p + 2) / 2;
    const size_t u = (size_t)dimp(p) * sizeof(zd), tab = 2 * (size_t)H * (B + 1) * sizeof(double);
    return (size_t)dimp(p) * sizeof(zd) + (u > tab ? u : tab);
}

// One warp per cell of a level, deepest level first (compute_moments,
// moments.rs:96-108): P2M for leaves (p2m_cell :30-53), M2M for internal
// cells (m2m_cell :56-90), then the multipole power (:150-168) and, when f is
// given, fmin (mac.rs:151-173). With skip_internal (the engine's choice), the
// internal cells of the level are left to k_m2m_exact_block.
//
// P2M: the lanes build the Υ tables of B bodies at once (a lane per body, the
// recursion of upsilon_table_into, harmonic.rs:141-173); then each lane owns
// the m >= 0 coefficients e = lane, lane + 32, ... and adds m_k Υ_k[e] over
// the round's bodies in slot order, so every coefficient is the reference's
// sum in the reference's order.
__global__ void k_upward_exact(const int32_t* __restrict__ level_cells, int lstart, int lcnt, CellsView cells,
                               const double* __restrict__ x, const double* __restrict__ y,
                               const double* __restrict__ z, const double* __restrict__ m, int p,
                               zd* __restrict__ moments, double* __restrict__ pows, const double* __restrict__ f,
                               double* __restrict__ fmin_out, int skip_internal) {
    extern __shared__ unsigned char smem_raw[];
    const int dim = dimp(p);
    const int H = (p + 1) * (p + 2) / 2;
    const int B = p2m_round(p), S = B + 1;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    unsigned char* wbase = smem_raw + (size_t)wib * upward_exact_smem_per_warp(p);
    zd* acc = reinterpret_cast<zd*>(wbase);
    zd* u = acc + dim;                                   // M2M: Υ of the child offset
    double* tre = reinterpret_cast<double*>(acc + dim);  // P2M: Υ tables, real parts
    double* tim = tre + (size_t)H * S;                   //      imaginary parts
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int j = warp; j < lcnt; j += nwarps) {
        const int c = level_cells[lstart + j];
        if (skip_internal && !cells.leaf[c]) continue;
        const double zx = cells.cx[c], zy = cells.cy[c], zz = cells.cz[c];
        for (int e = lane; e < dim; e += 32) acc[e] = mk(0.0, 0.0);
        __syncwarp();
        if (cells.leaf[c]) {
            const uint32_t fst = cells.first[c], end = fst + cells.count[c];
            double ar[8], ai[8];  // this lane's coefficients e = lane + 32 t (m >= 0 half, H <= 231)
#pragma unroll
            for (int t = 0; t < 8; ++t) ar[t] = ai[t] = 0.0;
            for (uint32_t k0 = fst; k0 < end; k0 += B) {
                const int nb = (int)min((uint32_t)B, end - k0);
                if (lane < nb) {
                    const uint32_t k = k0 + lane;
                    const double dx = x[k] - zx, dy = y[k] - zy, dz = z[k] - zz;
                    const double r2 = dx * dx + dy * dy + dz * dz;
                    zd d = mk(1.0, 0.0);
                    for (int mm = 0; mm <= p; ++mm) {
                        if (mm > 0) d = zmul(zscale(mk(dx, dy), g_tab.inv2m[mm]), d);
                        int h = mm * (mm + 1) / 2 + mm;  // half index of (mm, mm)
                        tre[h * S + lane] = d.re;
                        tim[h * S + lane] = d.im;
                        zd u1 = d, u2 = mk(0.0, 0.0);
                        for (int n = mm + 1; n <= p; ++n) {
                            const double a = (double)(2 * n - 1) * dz;
                            zd t = zscale(u1, a);
                            if (n >= mm + 2) t = zsub(t, zscale(u2, r2));
                            const zd un = zscale(t, g_tab.invc[n][mm]);
                            h += n;  // half index of (n, mm)
                            tre[h * S + lane] = un.re;
                            tim[h * S + lane] = un.im;
                            u2 = u1;
                            u1 = un;
                        }
                    }
                }
                __syncwarp();
#pragma unroll
                for (int t = 0; t < 8; ++t) {
                    const int e = lane + 32 * t;
                    if (e < H) {
                        for (int b = 0; b < nb; ++b) {
                            const double mk_ = m[k0 + b];
                            ar[t] += tre[e * S + b] * mk_;
                            ai[t] += tim[e * S + b] * mk_;
                        }
                    }
                }
                __syncwarp();
            }
            // the m >= 0 sums into the full layout; negative orders mirror
            // exactly (every increment of M_n^{-m} is (-1)^m conj of the
            // M_n^m increment)
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                const int e = lane + 32 * t;
                if (e < H) {
                    int n = 0;
                    while ((n + 1) * (n + 2) / 2 <= e) ++n;
                    const int mm = e - n * (n + 1) / 2;
                    acc[cidx(n, mm)] = mk(ar[t], ai[t]);
                }
            }
            __syncwarp();
            for (int e = lane; e < dim; e += 32) {
                int n, mm;
                split_nm(e, n, mm);
                if (mm < 0) {
                    double sgn = ((-mm) % 2 == 0) ? 1.0 : -1.0;
                    acc[e] = zscale(zconj(acc[cidx(n, -mm)]), sgn);
                }
            }
            __syncwarp();
        } else {
            for (int o = 0; o < 8; ++o) {
                const int ch = cells.child[8 * c + o];
                if (ch < 0) continue;
                const double dx = cells.cx[ch] - zx, dy = cells.cy[ch] - zy, dz = cells.cz[ch] - zz;
                const double r2 = dx * dx + dy * dy + dz * dz;
                for (int mm = lane; mm <= p; mm += 32) upsilon_column(dx, dy, dz, r2, p, mm, u);
                __syncwarp();
                const zd* mc = moments + (size_t)ch * dim;
                for (int e = lane; e < dim; e += 32) {
                    int n, mm;
                    split_nm(e, n, mm);
                    zd s = mk(0.0, 0.0);
                    for (int k = 0; k <= n; ++k) {
                        const int nk = n - k;
                        const int lo = max(-k, mm - nk), hi = min(k, mm + nk);
                        for (int l = lo; l <= hi; ++l) s = zadd(s, zmul(u[cidx(k, l)], mc[cidx(nk, mm - l)]));
                    }
                    acc[e] = zadd(acc[e], s);
                }
                __syncwarp();
            }
        }
        zd* out = moments + (size_t)c * dim;
        for (int e = lane; e < dim; e += 32) out[e] = acc[e];
        for (int n = lane; n <= p; n += 32) {
            double s = 0.0;
            for (int mm = -n; mm <= n; ++mm) {
                int am = mm < 0 ? -mm : mm;
                zd v = acc[cidx(n, mm)];
                double w = g_tab.fact[n - am] * g_tab.fact[n + am];
                s += w * (v.re * v.re + v.im * v.im);
            }
            pows[(size_t)c * (p + 1) + n] = sqrt(s);
        }
        if (f != nullptr && lane == 0) {
            double mn = INFINITY;
            if (cells.leaf[c]) {
                const uint32_t fst = cells.first[c], end = fst + cells.count[c];
                for (uint32_t k = fst; k < end; ++k) mn = fmin(mn, f[k]);
            } else {
                for (int o = 0; o < 8; ++o) {
                    int ch = cells.child[8 * c + o];
                    if (ch >= 0) mn = fmin(mn, fmin_out[ch]);
                }
            }
            fmin_out[c] = mn;
        }
        __syncwarp();
    }
}

// M2M of the internal cells of a level, one block per cell:
// the Υ tables of the (up to 8) child offsets and each child's convolution
// sums s_o[e] (8 dim independent chains) are computed side by side; then
// every coefficient adds its children's sums in octant order, as m2m_cell
// (moments.rs:56-90) does one child after the other. Power and fmin as in
// k_upward_exact. Shared memory: 16 dim complex.
__global__ void __launch_bounds__(256) k_m2m_exact_block(const int32_t* __restrict__ level_cells, int lstart,
                                                         int lcnt, CellsView cells, int p, zd* __restrict__ moments,
                                                         double* __restrict__ pows, const double* __restrict__ f,
                                                         double* __restrict__ fmin_out) {
    extern __shared__ unsigned char smem_raw[];
    const int dim = dimp(p);
    zd* ut = reinterpret_cast<zd*>(smem_raw);  // 8 Υ tables
    zd* st = ut + 8 * dim;                      // 8 child sums
    __shared__ int ch[8];
    const int tid = threadIdx.x;
    for (int j = blockIdx.x; j < lcnt; j += gridDim.x) {
        const int c = level_cells[lstart + j];
        if (cells.leaf[c]) continue;  // uniform: the whole block skips
        if (tid < 8) ch[tid] = cells.child[8 * c + tid];
        __syncthreads();
        const double zx = cells.cx[c], zy = cells.cy[c], zz = cells.cz[c];
        for (int t = tid; t < 8 * (p + 1); t += blockDim.x) {
            const int o = t / (p + 1), mm = t % (p + 1);
            const int cc = ch[o];
            if (cc < 0) continue;
            const double dx = cells.cx[cc] - zx, dy = cells.cy[cc] - zy, dz = cells.cz[cc] - zz;
            const double r2 = dx * dx + dy * dy + dz * dz;
            upsilon_column(dx, dy, dz, r2, p, mm, ut + o * dim);
        }
        __syncthreads();
        for (int t = tid; t < 8 * dim; t += blockDim.x) {
            const int o = t / dim, e = t % dim;
            const int cc = ch[o];
            if (cc < 0) continue;
            int n, mm;
            split_nm(e, n, mm);
            const zd* u = ut + o * dim;
            const zd* mc = moments + (size_t)cc * dim;
            zd s = mk(0.0, 0.0);
            for (int k = 0; k <= n; ++k) {
                const int nk = n - k;
                const int lo = max(-k, mm - nk), hi = min(k, mm + nk);
                for (int l = lo; l <= hi; ++l) s = zadd(s, zmul(u[cidx(k, l)], mc[cidx(nk, mm - l)]));
            }
            st[o * dim + e] = s;
        }
        __syncthreads();
        zd* out = moments + (size_t)c * dim;
        zd* acc = ut;  // the tables are no longer needed: the sums land in slot 0
        for (int e = tid; e < dim; e += blockDim.x) {
            zd a = mk(0.0, 0.0);
            for (int o = 0; o < 8; ++o)
                if (ch[o] >= 0) a = zadd(a, st[o * dim + e]);
            out[e] = a;
            acc[e] = a;
        }
        __syncthreads();
        for (int n = tid; n <= p; n += blockDim.x) {
            double s = 0.0;
            for (int mm = -n; mm <= n; ++mm) {
                int am = mm < 0 ? -mm : mm;
                zd v = acc[cidx(n, mm)];
                double w = g_tab.fact[n - am] * g_tab.fact[n + am];
                s += w * (v.re * v.re + v.im * v.im);
            }
            pows[(size_t)c * (p + 1) + n] = sqrt(s);
        }
        if (f != nullptr && tid == 0) {
            double mn = INFINITY;
            for (int o = 0; o < 8; ++o)
                if (ch[o] >= 0) mn = fmin(mn, fmin_out[ch[o]]);
            fmin_out[c] = mn;
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------ f pre-pass
// f_walk, mac.rs:99-147: monopole treecode estimate of f_b = sum m/r^2 with a
// LIFO stack (children pushed in octant order, so popped in reverse).
// In a forest the walk starts at the root of the body's own system (roots
// are level 0, in system order; slots of system s are [off[s], off[s+1])).
__global__ void k_fprepass(CellsView cells, const double* __restrict__ x, const double* __restrict__ y,
                           const double* __restrict__ z, const double* __restrict__ m, size_t n,
                           const uint64_t* __restrict__ off, int nsys, const int32_t* __restrict__ roots,
                           double* __restrict__ f, int* __restrict__ err) {
    constexpr int STACK = 8 * FMMX_NLEVELS;
    int stack[STACK];
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double px = x[i], py = y[i], pz = z[i];
        int root = 0;
        if (nsys > 1) {
            int lo = 0, hi = nsys;
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (off[mid] <= i) lo = mid;
                else hi = mid;
            }
            root = roots[lo];
        }
        int sp = 0;
        stack[sp++] = root;
        double fi = 0.0;
        while (sp > 0) {
            const int c = stack[--sp];
            if (cells.leaf[c]) {
                const uint32_t fst = cells.first[c], end = fst + cells.count[c];
                for (uint32_t k = fst; k < end; ++k) {
                    if (k == i) continue;
                    double dx = px - x[k], dy = py - y[k], dz = pz - z[k];
                    double r2 = dx * dx + dy * dy + dz * dz;
                    if (r2 > 0.0) fi += m[k] / r2;
                }
            } else {
                double dx = px - cells.cx[c], dy = py - cells.cy[c], dz = pz - cells.cz[c];
                double d2 = dx * dx + dy * dy + dz * dz;
                double rh = cells.rho[c];
                if (d2 > rh * rh) {
                    fi += cells.mass[c] / d2;
                } else {
                    if (sp + 8 > STACK) {
                        atomicOr(err, 1);
                        sp = 0;
                        break;
                    }
                    const int32_t* ch = cells.child + 8 * c;
                    for (int o = 0; o < 8; ++o)
                        if (ch[o] >= 0) stack[sp++] = ch[o];
                }
            }
        }
        f[i] = fi;
    }
}

// cx, cy, cz, rho of every cell in one 32-byte record, for the walk
__global__ void k_pack_geo(int nc, const double* __restrict__ cx, const double* __restrict__ cy,
                           const double* __restrict__ cz, const double* __restrict__ rho, double4* __restrict__ geo) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x)
        geo[c] = make_double4(cx[c], cy[c], cz[c], rho[c]);
}

// ------------------------------------------------------------ MAC
// error_estimate + accept, mac.rs:23-95 (operation order kept, including the
// inner r*r of error_estimate).
__device__ __forceinline__ bool accept_dehnen(const CellsView& cv, const MacParams& mp, const double* __restrict__ pows,
                                              const double* __restrict__ fminv, int a, int b, const double4 ga,
                                              const double4 gb) {
    const double ax = ga.x, ay = ga.y, az = ga.z;
    const double dx = gb.x - ax, dy = gb.y - ay, dz = gb.z - az;
    const double r2 = dx * dx + dy * dy + dz * dz;
    const double ra = ga.w, rb = gb.w;
    const double sum_rho = ra + rb;
    if (r2 <= sum_rho * sum_rho) return false;
    const double r = sqrt(r2);
    if (r == 0.0) return false;
    const int p = mp.p;
    const double rr2 = r * r;
    double rp = 1.0;
    for (int i = 0; i < p / 2; ++i) rp *= rr2;
    if (p % 2 == 1) rp *= r;
    double rpows[FMMX_MAXP + 1];
    rpows[0] = 1.0;
    for (int j = 1; j <= p; ++j) rpows[j] = rpows[j - 1] * rb;
    const double* pw = pows + (size_t)a * (p + 1);
    double s = 0.0;
    for (int k = 0; k <= p; ++k) s += g_tab.binom[p][k] * pw[k] * rpows[p - k];
    const double ma = cv.mass[a];
    const double e = s / (ma * rp);
    const double denom = ra + rb;
    double est;
    if (denom == 0.0) est = 0.0;
    else est = 8.0 * fmax(ra, rb) / denom * e;
    if (est == 0.0) return true;
    return est * ma / r2 < mp.eps * fminv[b];
}

// Separation condition (extension, with softening): the bodies of the two
// cells are at least mp.gap apart, r - rho_A - rho_B >= gap.
__device__ __forceinline__ bool gap_ok(const MacParams& mp, const double4 ga, const double4 gb) {
    if (!(mp.gap > 0.0)) return true;
    const double dx = gb.x - ga.x, dy = gb.y - ga.y, dz = gb.z - ga.z;
    const double r2 = dx * dx + dy * dy + dz * dz;
    return sqrt(r2) - (ga.w + gb.w) >= mp.gap;
}

// The geometric MAC (extension): accept when (rho_A + rho_B) < theta r, both
// ways round as the reference's walk applies its MAC (walk.rs:138-139), and
// gap_ok. The
// two directions and gap_ok evaluate the same r2 (the squares of b - a and
// a - b are equal bit for bit) and the same rho sum (addition commutes), so
// one square root decides all three.
__device__ __forceinline__ bool accept_theta_pair(const MacParams& mp, const double4 ga, const double4 gb) {
    const double dx = gb.x - ga.x, dy = gb.y - ga.y, dz = gb.z - ga.z;
    const double r2 = dx * dx + dy * dy + dz * dz;
    const double sum_rho = ga.w + gb.w;
    const double r = sqrt(r2);
    if (!(sum_rho < mp.theta * r)) return false;
    return !(mp.gap > 0.0) || r - sum_rho >= mp.gap;
}

// ------------------------------------------------------------ dual walk
// process_pair, walk.rs:94-190, applied to a whole frontier of cell pairs at
// once. Every decision depends only on the pair, so the emitted M2L and P2P
// pair sets equal those of the reference's depth-first stack walk. Appends are
// warp-aggregated: one atomic per warp and list (a ballot for the M2L and P2P
// lists, a prefix sum of the child-pair counts for the next frontier); the
// order within a list is arbitrary, the directed lists are sorted afterwards.
enum { WK_NONE = 0, WK_M2L = 1, WK_P2P = 2, WK_SPLIT_SELF = 3, WK_SPLIT = 4 };

// children of a cell: 8 ids (-1 absent), 32-byte aligned, read as two int4
__device__ __forceinline__ void load_children(const CellsView& cv, int c, int (&ch)[8]) {
    const int4* p = reinterpret_cast<const int4*>(cv.child + 8 * (size_t)c);
    const int4 u = p[0], v = p[1];
    ch[0] = u.x; ch[1] = u.y; ch[2] = u.z; ch[3] = u.w;
    ch[4] = v.x; ch[5] = v.y; ch[6] = v.z; ch[7] = v.w;
}
__device__ __forceinline__ int n_children(const CellsView& cv, int c) {
    int ch[8];
    load_children(cv, c, ch);
    int n = 0;
#pragma unroll
    for (int o = 0; o < 8; ++o) n += ch[o] >= 0;
    return n;
}

__device__ __forceinline__ int warp_append(int* counter, bool mine, int lane) {
    const unsigned mask = __ballot_sync(0xffffffffu, mine);
    if (!mask) return -1;
    const int leader = __ffs(mask) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(counter, __popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    return mine ? base + __popc(mask & ((1u << lane) - 1u)) : -1;
}

// Latency: a walk iteration is a chain of dependent L2 round trips (the
// frontier entry, then the cells, then the appends), so every read a pair can
// need -- both cells' leaf flags, geometry and children -- is issued at once
// after the entry, and the three appends (M2L, P2P, next frontier) are one
// atomic instruction from three lanes.
template <bool DEHNEN>
__global__ void k_walk_iter(CellsView cv, MacParams mp, const double* __restrict__ pows,
                            const double* __restrict__ fminv, WalkBufs w, int cur) {
    // After an overflow the frontier holds unwritten entries: stop, the host
    // retries with larger buffers.
    if (w.counts[WC_OVERFLOW]) return;
    const int nin = min(w.counts[cur], (int)w.cap_front);
    const int nxt = cur ^ 1;
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(w.pops_ptr, (unsigned long long)nin);
    const uint2* __restrict__ fin = w.front[cur];
    uint2* fout = w.front[nxt];
    const int lane = threadIdx.x & 31;
    const int stride = gridDim.x * blockDim.x;
    // whole warps step through the frontier together (the ballots need every lane)
    for (int q0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31); q0 < nin; q0 += stride) {
        const int q = q0 + lane;
        int kind = WK_NONE, a = 0, b = 0, npush = 0;
        bool split_a = false;
        int cha[8], chb[8];
        if (q < nin) {
            const uint2 pr = fin[q];
            a = (int)pr.x;
            b = (int)pr.y;
            const bool la = cv.leaf[a], lb = cv.leaf[b];
            const double4 ga = cv.geo[a], gb = cv.geo[b];
            load_children(cv, a, cha);
            load_children(cv, b, chb);
            if (a == b) {
                if (la) {
                    kind = WK_P2P;
                } else {
                    kind = WK_SPLIT_SELF;
                    int nch = 0;
#pragma unroll
                    for (int o = 0; o < 8; ++o) nch += cha[o] >= 0;
                    npush = nch * (nch + 1) / 2;
                }
            } else {
                bool acc;
                if (DEHNEN)
                    acc = accept_dehnen(cv, mp, pows, fminv, a, b, ga, gb) &&
                          accept_dehnen(cv, mp, pows, fminv, b, a, gb, ga) && gap_ok(mp, ga, gb);
                else
                    acc = accept_theta_pair(mp, ga, gb);
                if (acc) {
                    kind = WK_M2L;
                } else if (la && lb) {
                    kind = WK_P2P;
                } else {
                    // split b when a is a leaf or b is the larger cell, else split a
                    kind = WK_SPLIT;
                    split_a = lb || (!la && ga.w >= gb.w);
                    int nch = 0;
                    // chb takes the children of the cell that splits (element by
                    // element, so both arrays stay in registers)
#pragma unroll
                    for (int o = 0; o < 8; ++o) {
                        chb[o] = split_a ? cha[o] : chb[o];
                        nch += chb[o] >= 0;
                    }
                    npush = nch;
                }
            }
        }
        const unsigned mm = __ballot_sync(0xffffffffu, kind == WK_M2L);
        const unsigned mq = __ballot_sync(0xffffffffu, kind == WK_P2P);
        // next frontier: inclusive prefix sum of the pushes across the warp
        int incl = npush;
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        // lanes 0, 1, 2 reserve the warp's M2L, P2P and frontier entries
        int got = 0;
        {
            const int v = lane == 0 ? __popc(mm) : lane == 1 ? __popc(mq) : lane == 2 ? total : 0;
            int* ctr = w.counts + (lane == 0 ? WC_M2L : lane == 1 ? WC_P2P : nxt);
            if (v > 0) got = atomicAdd(ctr, v);
        }
        const int bm = __shfl_sync(0xffffffffu, got, 0);
        const int bp = __shfl_sync(0xffffffffu, got, 1);
        const int bf = __shfl_sync(0xffffffffu, got, 2);
        const unsigned below = (1u << lane) - 1u;
        if (kind == WK_M2L) {
            const int sm = bm + __popc(mm & below);
            if ((uint32_t)sm < w.cap_m2l) w.m2l[sm] = make_uint2(a, b);
            else atomicOr(&w.counts[WC_OVERFLOW], 4);
        } else if (kind == WK_P2P) {
            const int sp = bp + __popc(mq & below);
            if ((uint32_t)sp < w.cap_p2p) w.p2p[sp] = make_uint2(a, b);
            else atomicOr(&w.counts[WC_OVERFLOW], 2);
        }
        if (total == 0) continue;
        if ((uint32_t)(bf + total) > w.cap_front) {
            if (lane == 0) atomicOr(&w.counts[WC_OVERFLOW], 1);
            continue;
        }
        int pos = bf + incl - npush;
        if (kind == WK_SPLIT_SELF) {
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                if (cha[i] < 0) continue;
#pragma unroll
                for (int j = i; j < 8; ++j)
                    if (cha[j] >= 0) fout[pos++] = make_uint2(cha[i], cha[j]);
            }
        } else if (kind == WK_SPLIT) {
#pragma unroll
            for (int o = 0; o < 8; ++o) {
                const int c = chb[o];
                if (c < 0) continue;
                fout[pos++] = split_a ? make_uint2(c, b) : make_uint2(a, c);
            }
        }
    }
}

void launch_walk_iter(bool dehnen, unsigned grid, cudaStream_t s, CellsView cv, MacParams mp, const double* pows,
                      const double* fmin, WalkBufs w, int cur) {
    if (dehnen) k_walk_iter<true><<<grid, 256, 0, s>>>(cv, mp, pows, fmin, w, cur);
    else k_walk_iter<false><<<grid, 256, 0, s>>>(cv, mp, pows, fmin, w, cur);
}

int walk_iter_blocks_per_sm(bool dehnen) {
    int per_sm = 0;
    const cudaError_t e = dehnen ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_walk_iter<true>, 256, 0)
                                 : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_walk_iter<false>, 256, 0);
    return e == cudaSuccess && per_sm > 0 ? per_sm : 1;
}

}  // namespace fmmx
