// Register-resident line solves along x (kernel in sweep_reg.cuh).
#include "sweep_reg.cuh"

namespace mc3d {
template int launch_sweep_reg<0, float>(const Grid3 &, const LineOpDev<float> &, const SweepBatch<float> &, int,
                                         const RhsFinalArgs<float> &, int, int, int, cudaStream_t);
template int launch_sweep_reg<0, double>(const Grid3 &, const LineOpDev<double> &, const SweepBatch<double> &, int,
                                          const RhsFinalArgs<double> &, int, int, int, cudaStream_t);
}  // namespace mc3d
