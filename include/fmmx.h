/*
 * fmmx.h — C ABI of the B200-native FMM force engine (libfmmx.so).
 *
 * This is the drop-in boundary for the force evaluation of the reference FMM
 * (Vedant9500/FMMS, crates/fmm). Every entry point names the reference
 * interface it replaces as file:line inside crates/fmm/src (or the crate
 * given). Plain pointers and sizes only: no CUDA or torch types.
 *
 * Conventions
 *  - Positions are n x 3 interleaved FP64 (Particle.pos, models.rs:7-10),
 *    masses n FP64; results come back in particle-id order (fmm.rs:17-21):
 *    acc n x 3 FP64, pot n FP64 with the positive convention pot_i = sum m_j/r_ij.
 *  - The caller owns every buffer it passes; the context owns device memory.
 *  - Every call returns an fmmx_status and never aborts; fmmx_last_error()
 *    gives the message of the last failure on a context.
 *  - One context is not thread-safe; separate contexts are independent.
 *  - G = 1.
 */
#ifndef FMMX_H
#define FMMX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. FMMX_OVER_BUDGET is the reference GPU backend's OverBudget
 * (crates/visual/src/gpufmm.rs:1653-1672): an engine buffer would take the
 * context above its device_budget_bytes; the message names the buffer, the
 * bytes and the limit; the context then drops its cached device buffers
 * and stays usable (the caller can retry smaller or fall back). FMMX_LEAF_OVERFLOW mirrors the reference's
 * OverfullLeaf (gpufmm.rs:1377-1379, a leaf above its 64-lane kernels); no
 * kernel here bounds the bodies of a leaf, so it is never returned. */
typedef enum fmmx_status {
    FMMX_OK = 0,
    FMMX_INVALID_ARG = 1,
    FMMX_OUT_OF_MEMORY = 2,
    FMMX_OVER_BUDGET = 3,
    FMMX_LEAF_OVERFLOW = 4,
    FMMX_DEVICE_ERROR = 5,
    FMMX_TIMEOUT = 6,
    FMMX_NOT_BUILT = 7,
    FMMX_NO_DEVICE = 8
} fmmx_status;

/* Multipole acceptance criterion. DEHNEN is the reference's error-controlled
 * criterion with accuracy parameter mac_eps (mac.rs:23-95, the `eps` of
 * Fmm::new). THETA accepts a cell pair when (rho_A + rho_B) / r < theta
 * (an extension; the reference has no opening-angle parameter). */
typedef enum fmmx_mac_mode { FMMX_MAC_DEHNEN = 0, FMMX_MAC_THETA = 1 } fmmx_mac_mode;

/* Expansion centres (tree.rs:18-25). */
typedef enum fmmx_center_mode { FMMX_CENTER_COM = 0, FMMX_CENTER_SPHERE = 1 } fmmx_center_mode;

/* PLAIN_FP64: FP64 end to end, keys/tree/lists bit-exact to the reference.
 * MIXED: FP32 P2P with compensated accumulation, FP32 M2L/L2L/L2P; FP64 only
 * for centre-relative subtraction, the MAC, and M2M/L2L on the top 3 levels. */
typedef enum fmmx_precision { FMMX_PLAIN_FP64 = 0, FMMX_MIXED = 1 } fmmx_precision;

/* M2L kernel. NAIVE is the reference's O(p^4) convolution (translate.rs:47-136);
 * ROTATION the O(p^3) rotate / translate-along-z / rotate-back kernel
 * (rotation.rs:262-435). AUTO picks the faster on the device, which is the
 * rotation kernel at every p (the reference switches to rotation only from
 * p = 20, rotation.rs:45, because on its CPU the naive form wins below). */
typedef enum fmmx_m2l_kernel { FMMX_M2L_AUTO = 0, FMMX_M2L_NAIVE = 1, FMMX_M2L_ROTATION = 2 } fmmx_m2l_kernel;

typedef struct fmmx_config {
    int p;             /* expansion order, 1..20 (Fmm::new `p`, fmm.rs:26) */
    int mac_mode;      /* fmmx_mac_mode */
    double mac_eps;    /* DEHNEN accuracy parameter (Fmm::new `eps`) */
    double theta;      /* THETA opening angle */
    double softening;  /* Plummer softening length (0 reproduces the reference) */
    int n_leaf;        /* leaf capacity (Fmm::new `n_leaf`) */
    int center_mode;   /* fmmx_center_mode */
    int precision;     /* fmmx_precision */
    int m2l_kernel;    /* fmmx_m2l_kernel */
    int device;        /* CUDA device ordinal */
    void* stream;      /* cudaStream_t to run on, or NULL for a private stream */
    int p2p_tile;      /* source bodies per shared-memory tile of the mixed P2P (128, 256, 512, 1024; 0 = 512) */
    int preemptible;   /* 1: the M2L runs one short block per destination cell instead of persistent warps,
                          so kernels on higher-priority streams start between its blocks (serving lanes);
                          0 (default): persistent warps, the faster form for one evaluation at a time */
    double soft_gap;   /* extension, with softening > 0: a cell pair is accepted for M2L only if its bodies are
                          at least soft_gap * softening apart (r - rho_A - rho_B), on top of the MAC. The far
                          field uses the unsoftened kernel, which errs by about softening^2 / (2 d^2) relative
                          at distance d; this bounds that error. 0 (default): no such condition */
    int use_graphs;    /* 1 (default): fmmx_leapfrog_device records a step on a reused tree (refresh_every > 1)
                          as a CUDA graph once per tree and replays it; 0: plain launches */
    int overlap;       /* 1 (default): an evaluation runs on two streams (walk and lists beside the upward pass,
                          P2P beside M2L and L2L; the per-stage times then overlap); 0: one stream, every
                          stage alone on the device (for timing single kernels) */
    uint64_t device_budget_bytes; /* device memory the context may hold, in bytes (0, the default: no limit);
                          an allocation above it fails with FMMX_OVER_BUDGET */
} fmmx_config;

typedef struct fmmx_stats {
    uint64_t n;
    uint64_t n_cells;
    uint64_t n_leaves;
    uint64_t n_levels;
    uint64_t n_m2l;            /* mutual M2L cell pairs */
    uint64_t n_p2p;            /* P2P leaf pairs, self pairs included */
    uint64_t walk_pops;        /* cell pairs examined by the dual walk */
    uint64_t p2p_interactions; /* directed body-body interactions */
    uint64_t m2l_directed;     /* directed M2L translations */
    double ms_build;           /* last build: keys, sort, cells, geometry */
    double ms_upward;          /* last evaluate: gather, P2M/M2M, power, f pre-pass */
    double ms_walk;            /* dual walk */
    double ms_lists;           /* directed list construction */
    double ms_m2l;
    double ms_p2p;
    double ms_l2l;
    double ms_l2p;
    double ms_evaluate;        /* whole evaluate, device time */
    uint64_t kernel_launches;  /* engine kernels launched by the last build + evaluate */
    uint64_t walk_retries;     /* walks of the last evaluate redone with larger buffers after an overflow */
    uint64_t device_bytes;     /* device memory held by the context */
} fmmx_stats;

typedef struct fmmx_ctx fmmx_ctx;

/* Defaults: p = 8, DEHNEN with mac_eps = 1e-5, softening 0, n_leaf = 16,
 * centre of mass, PLAIN_FP64, AUTO M2L, device 0, private stream. */
void fmmx_config_default(fmmx_config* cfg);

/* Context with its device memory pool. Replaces the state held by fmm::Fmm
 * (fmm.rs:10-15). */
fmmx_status fmmx_create(const fmmx_config* cfg, fmmx_ctx** out);
void fmmx_destroy(fmmx_ctx* ctx);
const char* fmmx_last_error(const fmmx_ctx* ctx);
const char* fmmx_status_string(fmmx_status s);

/* Build the octree from host buffers: Fmm::new / Fmm::with_center (fmm.rs:26,36)
 * and Fmm::refresh (fmm.rs:54, Octree::refresh_with_mode tree.rs:94-148). */
fmmx_status fmmx_build(fmmx_ctx* ctx, size_t n, const double* pos_xyz, const double* mass);

/* One force evaluation with host buffers: Fmm::run / Fmm::run_threaded
 * (fmm.rs:60-65, run_impl :69-142). pos_xyz/mass may be NULL to evaluate the
 * bodies given to the last build; pot may be NULL. */
fmmx_status fmmx_evaluate(fmmx_ctx* ctx, const double* pos_xyz, const double* mass, double* acc_xyz, double* pot);

/* Device-resident forms of the two calls above (pointers in device memory of
 * the context's device). */
fmmx_status fmmx_build_device(fmmx_ctx* ctx, size_t n, const double* d_pos_xyz, const double* d_mass);
fmmx_status fmmx_evaluate_device(fmmx_ctx* ctx, const double* d_pos_xyz, const double* d_mass, double* d_acc_xyz,
                                 double* d_pot);

/* Batched ensemble (no reference counterpart): build one forest over nsys
 * independent systems held back to back in the inputs; system s is bodies
 * [offsets[s], offsets[s+1]) (host array of nsys + 1 entries, offsets[0] = 0,
 * every system non-empty). Each system gets its own bounding box, keys, sort
 * and root, and no interaction crosses systems; one fmmx_evaluate then covers
 * all of them in the same launches, and every system's result is the one it
 * gets alone (same arithmetic in the same order). */
fmmx_status fmmx_build_ensemble(fmmx_ctx* ctx, size_t nsys, const uint64_t* offsets, const double* pos_xyz,
                                const double* mass);
fmmx_status fmmx_build_ensemble_device(fmmx_ctx* ctx, size_t nsys, const uint64_t* offsets, const double* d_pos_xyz,
                                       const double* d_mass);

/* Device-resident leapfrog (the integration loop of
 * crates/fmm/tests/energy_gate.rs:133-219, which drifts and kicks on the host
 * around Fmm::refresh + run). scheme 0 is kick-drift-kick: on entry d_acc must
 * hold the accelerations at d_pos (a build + evaluate, or a previous call);
 * scheme 1 is the reference test's drift-kick-drift. Positions and
 * velocities (n x 3) are updated in place, d_acc/d_pot (nullable) hold the
 * last evaluation. The tree is rebuilt every `refresh_every` steps (1 = every
 * step); in between, the tree and interaction lists are reused and only the
 * moments and locals are recomputed (tree reuse, gpufmm.rs:9-20). Works on a
 * forest too. No reference counterpart as a library call. */
fmmx_status fmmx_leapfrog_device(fmmx_ctx* ctx, double* d_pos_xyz, double* d_vel_xyz, const double* d_mass,
                                 double* d_acc_xyz, double* d_pot, double dt, int nsteps, int scheme,
                                 int refresh_every);

/* One kick-drift-kick step with a time step per body (d_dt[n]; a body with
 * dt = 0 does not move: its forces are evaluated, as for a session joining a
 * serving batch). On entry d_acc holds the forces at d_pos of the bodies with
 * dt > 0. With offsets (host, nsys + 1 entries, as fmmx_build_ensemble) the
 * tree is rebuilt over those systems from the drifted positions; without,
 * over the systems of the last build when rebuild != 0 (or when there are no
 * lists yet), else the tree and interaction lists of the last evaluation are
 * reused and only moments and locals are recomputed (tree reuse,
 * crates/visual/src/gpufmm.rs:9-20). Runs on the context's stream: returns
 * once the evaluation has finished on the device (the evaluation reads its
 * status back), with the closing half kick still queued behind it; a rebuild
 * also waits for the tree's level counts. No reference counterpart as a
 * library call (the
 * reference's loops step on the host, crates/fmm/tests/energy_gate.rs:156-177). */
fmmx_status fmmx_kdk_step_device(fmmx_ctx* ctx, double* d_pos_xyz, double* d_vel_xyz, const double* d_mass,
                                 double* d_acc_xyz, double* d_pot, const double* d_dt, size_t nsys,
                                 const uint64_t* offsets, int rebuild);

/* Wait for the context's stream. */
fmmx_status fmmx_synchronize(fmmx_ctx* ctx);

/* Counters and per-stage device times of the last build/evaluate (the walk
 * counters of walk.rs:27-86 and the bench profile mode,
 * crates/bench/src/main.rs:554-641). */
fmmx_status fmmx_get_stats(const fmmx_ctx* ctx, fmmx_stats* out);

/* ------------------------------------------------------------ parity exports
 * Copy the tree of the last build to host buffers, in the layout of
 * Octree/Cell (tree.rs:49-70): order[n], keys_sorted[n]; per cell
 * info[4] = {first, count, level, leaf}, children[8], cen[3], mass, rho.
 * Any pointer may be NULL. */
fmmx_status fmmx_export_tree(const fmmx_ctx* ctx, uint32_t* order, uint64_t* keys_sorted, uint32_t* cell_info,
                             int32_t* children, double* cen, double* mass, double* rho);

/* Interaction lists of the last evaluate, as the walk emits them
 * (walk.rs:94-190; record_pairs_par :342-488): m2l[2*n_m2l] mutual cell pairs
 * (a, b), p2p[2*n_p2p] leaf pairs (a, b) with self pairs (a, a). The order of
 * pairs is unspecified; the sets are those of the reference. */
fmmx_status fmmx_export_lists(const fmmx_ctx* ctx, uint32_t* m2l, uint32_t* p2p);

/* Expansions of the last evaluate (complex values as re, im pairs):
 * moments[ncells*dim] (moments.rs:96-108), locals[ncells*dim] after L2L
 * (translate.rs:209-218), pows[ncells*(p+1)] (moments.rs:150-168),
 * f[n] in slot order and fmin[ncells] (mac.rs:177-186; DEHNEN only).
 * PLAIN_FP64 only. Any pointer may be NULL. */
fmmx_status fmmx_export_expansions(const fmmx_ctx* ctx, double* moments, double* locals, double* pows, double* f,
                                   double* fmin);

/* --------------------------------------------------------------- error harness
 * FP64 direct sum at selected targets on the device: acc[nt*3], pot[nt]
 * (nullable), fscale[nt] = sum m/r^2 (nullable). Replaces the O(N^2) check of
 * direct.rs:6-31 and the sampled error of crates/bench/src/main.rs:34-78.
 * Host buffers. */
fmmx_status fmmx_direct_targets(int device, size_t n, const double* pos_xyz, const double* mass, double softening,
                                size_t nt, const uint32_t* targets, double* acc_xyz, double* pot, double* fscale);

/* Allocation-free form of fmmx_direct_targets, with no counterpart in the
 * reference: for callers that cannot allocate device memory, such as a physics
 * step in a fixed-latency frame loop (cudaMalloc/cudaFree can block and
 * synchronise the device) or a host whose device memory is owned by its own
 * pool allocator. All pointers are device memory of `device`; work is queued on
 * `stream` (a cudaStream_t, NULL for the default stream) and the call returns
 * without waiting. The per-split partial sums live in a static device array
 * sized for nt <= FMMX_DIRECT_NOALLOC_MAX_TARGETS (about 5 MB, held by every
 * GPU that loads the library until exit); larger nt returns FMMX_INVALID_ARG.
 * The first call on a device looks up that array's address, so make it before
 * any stream capture. Calls share the array: calls that overlap on the GPU
 * race. A target id >= n yields NaN for that target. */
#define FMMX_DIRECT_NOALLOC_MAX_TARGETS 4096
fmmx_status fmmx_direct_targets_noalloc(int device, void* stream, size_t n, const double* d_pos_xyz,
                                        const double* d_mass, double softening, size_t nt,
                                        const uint32_t* d_targets, double* d_acc_xyz, double* d_pot,
                                        double* d_fscale);

/* Diagnostics: measured FMA throughput of this device in TFLOP/s (an FMA
 * counts 2 flops) for FP64 (fp64 != 0) or FP32, from a register-resident FMA
 * loop over every SM. The roofline denominator of the CUDA-core kernels. No
 * reference counterpart. */
fmmx_status fmmx_probe_fma_peak(int device, int fp64, double* tflops);

/* ------------------------------------------------------------------ generators
 * Seeded inputs, host side. fmmx_gen_plummer reproduces models::plummer
 * (models.rs:35-58) bit for bit; fmmx_gen_hernquist models::hernquist
 * (models.rs:61-82). */
void fmmx_gen_plummer(size_t n, double cx, double cy, double cz, uint64_t seed, double* mass, double* pos_xyz);
void fmmx_gen_hernquist(size_t n, double cx, double cy, double cz, uint64_t seed, double* mass, double* pos_xyz);

/* Benchmark workloads (extensions, no reference counterpart).
 * fmmx_gen_plummer_ic: Plummer sphere (mass mtot, scale a) truncated at
 *   r <= rmax*a, isotropic velocities from the Plummer distribution function
 *   (vel n x 3, nullable).
 * fmmx_gen_uniform_lognormal: uniform in the unit cube, masses exp(N(0,sigma^2))
 *   normalised to sum 1.
 * fmmx_gen_clusters: nclust Plummer spheres, scale radii log-uniform in
 *   [amin, amax], centres uniform in the unit cube, sizes a Dirichlet(1) split
 *   of n, equal masses summing to 1. */
void fmmx_gen_plummer_ic(size_t n, double mtot, double a, double rmax, uint64_t seed, double* mass, double* pos_xyz,
                         double* vel_xyz);
void fmmx_gen_uniform_lognormal(size_t n, double sigma, uint64_t seed, double* mass, double* pos_xyz);
void fmmx_gen_clusters(size_t n, int nclust, double amin, double amax, uint64_t seed, double* mass, double* pos_xyz,
                       double* vel_xyz);

#ifdef __cplusplus
}
#endif

#endif /* FMMX_H */
