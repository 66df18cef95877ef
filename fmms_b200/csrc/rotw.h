// Host side of the warp rotation M2L: constant tables and launchers.
#pragma once
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "kernels.h"

namespace fmmx {

// Tables for degrees 0..16 (independent of the context's p): per degree k the
// real (k+1)^2 matrices P_k, Q_k of B_k and of B_k^T on the m >= 0 half, the
// factorial products (n-m)!(n+m)! on the half index, and j! for j <= 32.
struct RotwTables {
    std::vector<double> mats, fm, ifm, fact;
};
void make_rotw_tables(RotwTables& t);
// true if the tables have the zero pattern the warp kernel relies on
bool rotw_tables_check(const RotwTables& t);
void rotw_upload_f64(const RotwTables& t, cudaStream_t s);
void rotw_upload_f32(const RotwTables& t, cudaStream_t s);
cudaError_t launch_rotw_f64(int p, DirList L, int nc, CellsView cv, const zd* mom, zd* loc, int* work, int nsm,
                            cudaStream_t s);
cudaError_t launch_rotw_f32(int p, DirList L, int nc, CellsView cv, const float* scale, const zf* mom, zf* loc,
                            int* work, int nsm, cudaStream_t s);
constexpr int kRotwMaxP = 16;

}  // namespace fmmx
