// Instantiations of the FP32 march step kernel (ch_march.cuh): every row
// width the tiled path takes up to 256, ring depths 3, 4 and 6, with and
// without the FP64 mass feedback.
#include "ch_march.cuh"
#include "engine.h"

namespace mg {

template <int NXC, bool MASS>
static StepKernel march_f32_nbuf(int nbuf)
{
    switch (nbuf) {
    case 3: return ch_march_kernel<float, NXC, 3, MASS>;
    case 4: return ch_march_kernel<float, NXC, 4, MASS>;
    case 6: return ch_march_kernel<float, NXC, 6, MASS>;
    default: return nullptr;
    }
}

template <bool MASS>
static StepKernel march_f32_width(int nx, int nbuf)
{
    switch (nx) {
    case 64: return march_f32_nbuf<64, MASS>(nbuf);
    case 96: return march_f32_nbuf<96, MASS>(nbuf);
    case 128: return march_f32_nbuf<128, MASS>(nbuf);
    case 160: return march_f32_nbuf<160, MASS>(nbuf);
    case 192: return march_f32_nbuf<192, MASS>(nbuf);
    case 224: return march_f32_nbuf<224, MASS>(nbuf);
    case 256: return march_f32_nbuf<256, MASS>(nbuf);
    default: return nullptr;
    }
}

StepKernel march_kernel_f32(int nx, int nbuf, bool mass, int ty)
{
    // the tile of the 256^3 benchmark shape, specialised
    if (nx == 256 && nbuf == 3 && ty == 8)
        return mass ? ch_march_kernel<float, 256, 3, true, 8> : ch_march_kernel<float, 256, 3, false, 8>;
    return mass ? march_f32_width<true>(nx, nbuf) : march_f32_width<false>(nx, nbuf);
}

}  // namespace mg
