// Instantiations of the FP64 march step kernels (ch_march.cuh): row widths
// 64, 128, 192 and 256, ring depths 3, 4 and 6; the all-widths batch kernel
// at ring depths 3 and 6.
#include "ch_march.cuh"
#include "engine.h"

namespace mg {

template <int NXC>
static StepKernel march_f64_nbuf(int nbuf, int order)
{
    if (order == 0) {
        if constexpr (NXC == 256) {
            switch (nbuf) {
            case 3: return ch_march_kernel<double, 256, 3, false, 0>;
            case 4: return ch_march_kernel<double, 256, 4, false, 0>;
            case 6: return ch_march_kernel<double, 256, 6, false, 0>;
            default: return nullptr;
            }
        }
        return nullptr;
    }
    switch (nbuf) {
    case 3: return ch_march_kernel<double, NXC, 3, false, 1>;
    case 4: return ch_march_kernel<double, NXC, 4, false, 1>;
    case 6: return ch_march_kernel<double, NXC, 6, false, 1>;
    default: return nullptr;
    }
}

StepKernel march_batch_kernel_f64(int nbuf, bool inlined)
{
    switch (nbuf) {
    case 3: return inlined ? ch_march_batch_inline_kernel<double, 3, false> : ch_march_batch_kernel<double, 3, false>;
    case 6: return inlined ? ch_march_batch_inline_kernel<double, 6, false> : ch_march_batch_kernel<double, 6, false>;
    default: return nullptr;
    }
}

StepKernel march_kernel_f64(int nx, int nbuf, int order)
{
    switch (nx) {
    case 64: return march_f64_nbuf<64>(nbuf, order);
    case 128: return march_f64_nbuf<128>(nbuf, order);
    case 192: return march_f64_nbuf<192>(nbuf, order);
    case 256: return march_f64_nbuf<256>(nbuf, order);
    default: return nullptr;
    }
}

}  // namespace mg
