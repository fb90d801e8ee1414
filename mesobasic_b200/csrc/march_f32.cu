// Instantiations of the FP32 march step kernels (ch_march.cuh): every row
// width the tiled path takes up to 256, ring depths 3, 4 and 6, with and
// without the FP64 mass feedback; the all-widths batch kernel at ring
// depths 3 and 6.
#include "ch_march.cuh"
#include "engine.h"

namespace mg {

template <int NXC, bool MASS>
static StepKernel march_f32_nbuf(int nbuf, int order)
{
    if (order == 0) {
        if constexpr (NXC == 256) {
            switch (nbuf) {
            case 3: return ch_march_kernel<float, 256, 3, MASS, 0>;
            case 4: return ch_march_kernel<float, 256, 4, MASS, 0>;
            case 6: return ch_march_kernel<float, 256, 6, MASS, 0>;
            default: return nullptr;
            }
        }
        return nullptr;
    }
    switch (nbuf) {
    case 3: return ch_march_kernel<float, NXC, 3, MASS, 1>;
    case 4: return ch_march_kernel<float, NXC, 4, MASS, 1>;
    case 6: return ch_march_kernel<float, NXC, 6, MASS, 1>;
    default: return nullptr;
    }
}

template <bool MASS>
static StepKernel march_f32_width(int nx, int nbuf, int order)
{
    switch (nx) {
    case 64: return march_f32_nbuf<64, MASS>(nbuf, order);
    case 96: return march_f32_nbuf<96, MASS>(nbuf, order);
    case 128: return march_f32_nbuf<128, MASS>(nbuf, order);
    case 160: return march_f32_nbuf<160, MASS>(nbuf, order);
    case 192: return march_f32_nbuf<192, MASS>(nbuf, order);
    case 224: return march_f32_nbuf<224, MASS>(nbuf, order);
    case 256: return march_f32_nbuf<256, MASS>(nbuf, order);
    default: return nullptr;
    }
}

StepKernel march_kernel_f32(int nx, int nbuf, bool mass, int order)
{
    return mass ? march_f32_width<true>(nx, nbuf, order) : march_f32_width<false>(nx, nbuf, order);
}

StepKernel march_batch_kernel_f32(int nbuf, bool mass, bool inlined)
{
    switch (nbuf) {
    case 3:
        if (inlined) return mass ? ch_march_batch_inline_kernel<float, 3, true> : ch_march_batch_inline_kernel<float, 3, false>;
        return mass ? ch_march_batch_kernel<float, 3, true> : ch_march_batch_kernel<float, 3, false>;
    case 6:
        if (inlined) return mass ? ch_march_batch_inline_kernel<float, 6, true> : ch_march_batch_inline_kernel<float, 6, false>;
        return mass ? ch_march_batch_kernel<float, 6, true> : ch_march_batch_kernel<float, 6, false>;
    default: return nullptr;
    }
}

}  // namespace mg
