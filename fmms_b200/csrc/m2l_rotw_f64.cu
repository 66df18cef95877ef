// FP64 instantiation of the warp-per-destination rotation M2L (plain form:
// unscaled expansions in the full (n, m) layout of the reference).
#define ROTW_T double
#include "m2l_warp.cuh"
#include "rotw.h"

namespace fmmx {

void rotw_upload_f64(const RotwTables& t, cudaStream_t s) {
    cudaMemcpyToSymbolAsync(c_rot, t.mats.data(), sizeof(double) * ROTW_MATS, 0, cudaMemcpyHostToDevice, s);
    cudaMemcpyToSymbolAsync(c_fm, t.fm.data(), sizeof(double) * ROTW_NH, 0, cudaMemcpyHostToDevice, s);
    cudaMemcpyToSymbolAsync(c_ifm, t.ifm.data(), sizeof(double) * ROTW_NH, 0, cudaMemcpyHostToDevice, s);
    cudaMemcpyToSymbolAsync(c_fact, t.fact.data(), sizeof(double) * (2 * ROTW_MAXP + 1), 0, cudaMemcpyHostToDevice,
                            s);
}

template <int P>
static cudaError_t launch_p(DirList L, int nc, CellsView cv, const zd* mom, zd* loc, int* work, int nsm,
                            cudaStream_t s) {
    constexpr size_t smem = rotw_smem_per_warp<double, P>();
    auto kern = k_m2l_rotw<double, P, false, true>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = (int)std::min<size_t>(32, (220 * 1024) / smem);
    if (per_sm < 1) per_sm = 1;
    kern<<<work ? nsm * per_sm : (unsigned)nc, 32, smem, s>>>(L, nc, cv, nullptr, mom, loc, work);
    return cudaGetLastError();
}

cudaError_t launch_rotw_f64(int p, DirList L, int nc, CellsView cv, const zd* mom, zd* loc, int* work, int nsm,
                            cudaStream_t s) {
    switch (p) {
#define CASE(P) \
    case P: return launch_p<P>(L, nc, cv, mom, loc, work, nsm, s);
        CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7) CASE(8) CASE(9) CASE(10) CASE(11) CASE(12)
        CASE(13) CASE(14) CASE(15) CASE(16)
#undef CASE
    }
    return cudaErrorInvalidValue;
}

}  // namespace fmmx
