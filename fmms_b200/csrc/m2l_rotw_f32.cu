// FP32 instantiation of the warp-per-destination rotation M2L (mixed form:
// size-normalised expansions, m >= 0 half layout).
#define ROTW_T float
#include "m2l_warp.cuh"
#include "rotw.h"

namespace fmmx {

void rotw_upload_f32(const RotwTables& t, cudaStream_t s) {
    std::vector<float> mats(t.mats.begin(), t.mats.end()), fm(t.fm.begin(), t.fm.end()),
        ifm(t.ifm.begin(), t.ifm.end()), fact(t.fact.begin(), t.fact.end());
    cudaMemcpyToSymbolAsync(c_rot, mats.data(), sizeof(float) * ROTW_MATS, 0, cudaMemcpyHostToDevice, s);
    cudaMemcpyToSymbolAsync(c_fm, fm.data(), sizeof(float) * ROTW_NH, 0, cudaMemcpyHostToDevice, s);
    cudaMemcpyToSymbolAsync(c_ifm, ifm.data(), sizeof(float) * ROTW_NH, 0, cudaMemcpyHostToDevice, s);
    cudaMemcpyToSymbolAsync(c_fact, fact.data(), sizeof(float) * (2 * ROTW_MAXP + 1), 0, cudaMemcpyHostToDevice, s);
    cudaStreamSynchronize(s);  // the staging vectors die here
}

template <int P>
static cudaError_t launch_p(DirList L, int nc, CellsView cv, const float* scale, const zf* mom, zf* loc, int* work,
                            int nsm, cudaStream_t s) {
    constexpr size_t smem = rotw_smem_per_warp<float, P>();
    auto kern = k_m2l_rotw<float, P, true, false>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = (int)std::min<size_t>(32, (220 * 1024) / smem);
    if (per_sm < 1) per_sm = 1;
    kern<<<work ? nsm * per_sm : (unsigned)nc, 32, smem, s>>>(L, nc, cv, scale, mom, loc, work);
    return cudaGetLastError();
}

cudaError_t launch_rotw_f32(int p, DirList L, int nc, CellsView cv, const float* scale, const zf* mom, zf* loc,
                            int* work, int nsm, cudaStream_t s) {
    switch (p) {
#define CASE(P) \
    case P: return launch_p<P>(L, nc, cv, scale, mom, loc, work, nsm, s);
        CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7) CASE(8) CASE(9) CASE(10) CASE(11) CASE(12)
        CASE(13) CASE(14) CASE(15) CASE(16)
#undef CASE
    }
    return cudaErrorInvalidValue;
}

}  // namespace fmmx
