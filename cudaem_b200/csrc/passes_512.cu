// Slice-pass kernels for transforms of 512 points.
#include "passes.cuh"

namespace msb {

template void row_dispatch<512>(int op, const PassArgs& a, int nwaves, int ny, cudaStream_t st);
template void col_dispatch<512>(int op, const PassArgs& a, int nwaves, int nx, cudaStream_t st);
template bool engine_dispatch<512>(int rowop, const PassArgs& a, const EngineArgs& e, int nwaves, cudaStream_t st);

}  // namespace msb
