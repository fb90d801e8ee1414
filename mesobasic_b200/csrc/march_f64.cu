// Instantiations of the FP64 march step kernel (ch_march.cuh): row widths
// 64, 128, 192 and 256, ring depths 3, 4 and 6.
#include "ch_march.cuh"
#include "engine.h"

namespace mg {

template <int NXC>
static StepKernel march_f64_nbuf(int nbuf)
{
    switch (nbuf) {
    case 3: return ch_march_kernel<double, NXC, 3, false>;
    case 4: return ch_march_kernel<double, NXC, 4, false>;
    case 6: return ch_march_kernel<double, NXC, 6, false>;
    default: return nullptr;
    }
}

StepKernel march_kernel_f64(int nx, int nbuf, int ty)
{
    // the tile of the 256^3 benchmark shape, specialised
    if (nx == 256 && ty == 7 && nbuf == 6) return ch_march_kernel<double, 256, 6, false, 7>;
    if (nx == 256 && ty == 7 && nbuf == 3) return ch_march_kernel<double, 256, 3, false, 7>;
    switch (nx) {
    case 64: return march_f64_nbuf<64>(nbuf);
    case 128: return march_f64_nbuf<128>(nbuf);
    case 192: return march_f64_nbuf<192>(nbuf);
    case 256: return march_f64_nbuf<256>(nbuf);
    default: return nullptr;
    }
}

}  // namespace mg
