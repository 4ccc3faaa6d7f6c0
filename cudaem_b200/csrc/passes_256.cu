// Slice-pass kernels for transforms of 256 points.
#include "passes.cuh"

namespace msb {

template void row_dispatch<256>(int op, const PassArgs& a, int nwaves, int ny, cudaStream_t st);
template void col_dispatch<256>(int op, const PassArgs& a, int nwaves, int nx, cudaStream_t st);
template bool engine_dispatch<256>(int rowop, const PassArgs& a, const EngineArgs& e, int nwaves, cudaStream_t st);

}  // namespace msb
