// Kernel declarations and the device-side structures shared between the
// kernel files and the host orchestration (engine.cu).
#pragma once

#include "common.cuh"

namespace fmmx {

// Level bookkeeping array: start and count of each level's nodes.
enum { LV_START = 0, LV_COUNT = FMMX_NLEVELS + 1, LV_SIZE = 2 * (FMMX_NLEVELS + 1) };

// Nodes as created level by level, before depth-first renumbering.
struct TmpNodes {
    uint32_t* first;
    uint32_t* count;
    int32_t* parent;
    uint8_t* oct;
    uint8_t* level;
    uint8_t* leaf;
};

struct CellsMut {
    uint32_t* first;
    uint32_t* count;
    int32_t* child;
    int32_t* parent;
    uint8_t* leaf;
    uint8_t* level;
    double* cx;
    double* cy;
    double* cz;
    double* mass;
    double* rho;
};

struct MacParams {
    int mode;  // fmmx_mac_mode
    int p;
    double eps;
    double theta;
    double gap;  // minimum separation of the bodies of an M2L pair (soft_gap * softening); 0: none
};

enum { WC_FRONT0 = 0, WC_FRONT1 = 1, WC_M2L = 2, WC_P2P = 3, WC_OVERFLOW = 4, WC_SIZE = 8 };

struct WalkBufs {
    uint2* front[2];
    uint2* m2l;
    uint2* p2p;
    int* counts;           // WC_* slots
    unsigned long long* pops_ptr;
    uint32_t cap_front, cap_m2l, cap_p2p;
};

// Segmented directed interaction list: for destination cell c, sources
// src(key(i)) for i in [seg_begin[c], seg_end[c]), in ascending order.
struct DirList {
    const uint64_t* keys;    // entries (dst << shift) | src, or null
    const uint32_t* keys32;  // 32-bit entries (then keys is null); with shift = 32 the entries are the sources
    const uint32_t* seg_begin;
    const uint32_t* seg_end;
    int shift;
    __host__ __device__ uint64_t key(size_t i) const { return keys32 ? (uint64_t)keys32[i] : keys[i]; }
    __host__ __device__ uint32_t src(uint64_t key) const { return (uint32_t)(key & ((1ull << shift) - 1)); }
};

// tree_exact.cu
void upload_tables_exact(const OrderTables& t, cudaStream_t s);
__global__ void k_bbox_partial(const double* pos, size_t n, double* part, int* bad);
__global__ void k_bbox_final(const double* part, int nparts, double* box);
__global__ void k_keys(const double* pos, size_t n, const double* box, uint64_t* keys, uint32_t* idx);
__global__ void k_gather(const double* pos, const double* mass, const uint32_t* order, size_t n, double* x,
                         double* y, double* z, double* m);
__global__ void k_tree_init(TmpNodes t, uint32_t n, int* lvl);
__global__ void k_bbox_seg(const double* pos, const uint64_t* off, double* box, int* bad);
__global__ void k_keys_seg(const double* pos, size_t n, const uint64_t* off, int nsys, const double* box,
                           uint64_t* keys, uint32_t* idx);
__global__ void k_tree_init_forest(TmpNodes t, const uint64_t* off, int nsys, int* lvl);
__global__ void k_cell_h(const int32_t* level_cells, int lstart, int lcnt, const int32_t* parent, const double* box,
                         double* h);
__global__ void k_walk_init(const int32_t* level_cells, int nroots, uint2* front);
__global__ void k_build_level(TmpNodes t, const uint64_t* keys, int L, long long n_leaf, uint32_t cap, int* lvl,
                              int* flags);
__global__ void k_dfs_keys(TmpNodes t, int nc, uint64_t* key, uint32_t* val);
__global__ void k_finalize_cells(const uint32_t* sorted_t, int nc, TmpNodes t, int32_t* new_id, CellsMut cells);
__global__ void k_link_cells(int nc, TmpNodes t, const int32_t* new_id, CellsMut cells, int32_t* level_cells);
__global__ void k_body_leaf(int nc, const uint32_t* first, const uint32_t* count, const uint8_t* leaf,
                            int32_t* body_leaf);
__global__ void k_geometry_level(const int32_t* level_cells, int lstart, int lcnt, CellsMut cells, const double* x,
                                 const double* y, const double* z, const double* m, int center_mode);
// bodies per round of the exact P2M (the lanes of a warp build that many Υ tables at once)
__host__ __device__ inline int p2m_round(int p) { return p <= 12 ? 32 : (p <= 16 ? 16 : 8); }
__host__ __device__ size_t upward_exact_smem_per_warp(int p);
__global__ void k_upward_exact(const int32_t* level_cells, int lstart, int lcnt, CellsView cells, const double* x,
                               const double* y, const double* z, const double* m, int p, zd* moments, double* pows,
                               const double* f, double* fmin, int skip_internal);
__global__ void k_m2m_exact_block(const int32_t* level_cells, int lstart, int lcnt, CellsView cells, int p,
                                  zd* moments, double* pows, const double* f, double* fmin);
__global__ void k_fprepass(CellsView cells, const double* x, const double* y, const double* z, const double* m,
                           size_t n, const uint64_t* off, int nsys, const int32_t* roots, double* f, int* err);
// one dual-walk iteration over frontier `cur` (k_walk_iter<DEHNEN>: Dehnen's error-estimate MAC, else
// theta and soft_gap), 256-thread blocks; and its resident blocks per SM
void launch_walk_iter(bool dehnen, unsigned grid, cudaStream_t s, CellsView cv, MacParams mp, const double* pows,
                      const double* fmin, WalkBufs w, int cur);
int walk_iter_blocks_per_sm(bool dehnen);
__global__ void k_pack_geo(int nc, const double* cx, const double* cy, const double* cz, const double* rho,
                           double4* geo);

// lists.cu
// Directed list of `np` walk pairs with `nitems` directed entries: per
// destination c its sources src[off[c] .. off[c+1]) in ascending order
// (off has ncells + 1 entries; cnt is ncells + 1 scratch counters). With
// body_count, also adds the directed body-body interactions (P2P). Segments
// longer than 4096 entries are left for sort_long_segments: `longs`
// (2 ncells + 128 ints) receives their count at [0] and ids from [128].
size_t directed_list_temp(int nitems, int ncells);
cudaError_t build_directed_list(void* tmp, size_t tmp_bytes, const uint2* pairs, int np, int nitems, int ncells,
                                const uint32_t* body_count, unsigned long long* interactions, uint32_t* cnt,
                                uint32_t* off, uint32_t* src_unsorted, uint32_t* src, int* longs, unsigned grid,
                                cudaStream_t s);
size_t long_segments_temp(int nitems, int nlong, int end_bit);
// the nlong long segments (count read back from longs[0]); bounds: 2 nlong scratch
cudaError_t sort_long_segments(void* tmp, size_t tmp_bytes, const uint32_t* off, const int* longs, int nlong,
                               const uint32_t* src_unsorted, uint32_t* src, int nitems, int end_bit, uint32_t* bounds,
                               cudaStream_t s);
// exclusive prefix sum of n values (temp storage as for directed_list_temp)
cudaError_t scan_u32(void* tmp, size_t tmp_bytes, const uint32_t* in, uint32_t* out, int n, cudaStream_t s);

// m2l.cu
void upload_tables_m2l(const OrderTables& t, cudaStream_t s);
size_t m2l_rot_smem_bytes(int p);
__global__ void k_m2l_naive_f64(DirList L, int ncells, CellsView cv, int p, const zd* moments, zd* locals);
__global__ void k_m2l_rot_f64(DirList L, int ncells, CellsView cv, int p, const zd* moments, zd* locals,
                              const double* swap_g);

// sweeps.cu
void upload_tables_sweeps(const OrderTables& t, cudaStream_t s);
__global__ void k_l2l_f64(const int32_t* level_cells, int lstart, int lcnt, CellsView cv, const int32_t* parent,
                          int p, zd* locals);
__global__ void k_l2p_f64(size_t n, const int32_t* body_leaf, const uint32_t* order, CellsView cv, int p,
                          const zd* locals, const double* x, const double* y, const double* z, const double* nax,
                          const double* nay, const double* naz, const double* npot, double* acc, double* pot);

// mixed.cu
void upload_tables_mixed(const OrderTables& t, cudaStream_t s);
__global__ void k_cell_scale(int nc, const double* rho, const double* h, double* ell, float* ellf);
__global__ void k_rho_bodies(size_t n, const int32_t* body_leaf, CellsView cv, const double* x, const double* y,
                             const double* z, unsigned long long* rho_bits);
__global__ void k_rho_level(const int32_t* level_cells, int lstart, int lcnt, CellsView cv,
                            unsigned long long* rho_bits);
__global__ void k_moments_to_mixed(int nc, int p, const zd* full, const double* ell, zf* half);
void launch_upward_mixed(bool fp64, unsigned grid, int warps, cudaStream_t s, const int32_t* level_cells,
                         int lstart, int lcnt, CellsView cv, const double* ell, const double* x, const double* y,
                         const double* z, const double* m, int p, zf* mom);
void launch_l2l_mixed(bool fp64, unsigned grid, cudaStream_t s, const int32_t* level_cells, int lstart, int lcnt,
                      CellsView cv, const int32_t* parent, const double* ell, int p, zf* loc);
__global__ void k_l2p_mixed(size_t n, const int32_t* body_leaf, const uint32_t* order, CellsView cv,
                            const double* ell, int p, const zf* loc, const double* x, const double* y,
                            const double* z, const double* nax, const double* nay, const double* naz,
                            const double* npot, double* acc, double* pot);
// Near-field work units: the sources of a leaf in units of P2P_UNIT_SRC
// source leaves (uoff: units of cell c at uoff[c] .. uoff[c+1]; soff: the
// partial sums of a leaf with several units at part[soff[c] + k * count + i]).
// The units of leaves of at most P2P_SMALL_NT bodies are numbered apart
// (uoff_s) and run a warp each; the others (uoff_b) a block each.
#define P2P_UNIT_SRC 1024
#define P2P_SMALL_NT 32
struct P2pUnits {
    const uint32_t* uoff;    // ncells + 1, all units
    const uint32_t* uoff_s;  // ncells + 1, units of small leaves
    const uint32_t* uoff_b;  // ncells + 1, units of the other leaves
    const uint32_t* soff;    // ncells + 1
    double4* part;
    unsigned* next;  // two work counters (small, other), zero at launch
};
void launch_p2p_plan(unsigned grid, cudaStream_t s, int ncells, DirList L, const uint32_t* count, uint32_t* units,
                     uint32_t* units_s, uint32_t* units_b, uint32_t* scratch);
// loc: n float4 of scratch (bodies relative to their leaf's centre, with the mass)
void launch_p2p_mixed(int tile, int nsm, cudaStream_t s, DirList L, int ncells, CellsView cv, P2pUnits U, size_t n,
                      const int32_t* body_leaf, const double* x, const double* y, const double* z, const double* m,
                      float4* loc, float soft2, double* ax, double* ay, double* az, double* pot);

// p2p.cu
__global__ void k_p2p_f64(DirList L, int ncells, CellsView cv, const double* x, const double* y, const double* z,
                          const double* m, double soft2, double* ax, double* ay, double* az, double* pot);

// integrate.cu
__global__ void k_kick(size_t n3, double* v, const double* a, double h);
__global__ void k_drift(size_t n3, double* x, const double* v, double h);
__global__ void k_kick_rows(size_t n3, double* v, const double* a, const double* dt, double c);
__global__ void k_drift_rows(size_t n3, double* x, const double* v, const double* dt);

// direct.cu
__global__ void k_direct_targets(const double* pos, const double* mass, size_t n, const uint32_t* tgt, size_t nt,
                                 double soft2, double* part);
__global__ void k_direct_reduce(const double* part, int nsplit, size_t nt, double* acc, double* pot, double* fsc);

}  // namespace fmmx
