// Instantiations of the FP32 march step kernel (ch_march.cuh): every row
// width the tiled path takes up to 256, ring depths 3, 4 and 6, with and
// without the FP64 mass feedback.
#include "ch_march.cuh"
#include "ch_march2.cuh"
#include "engine.h"

#include <cstdlib>

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

// The FP32 march kernels of ch_march2.cuh (C++ shared-memory accesses and
// float2 f32x2 builtins; measured 1-4 % faster, bit-identical) take every
// march width at ring depth 3; MG_MARCH2=0 keeps ch_march_kernel.
bool march2_enabled()
{
    static const bool v = [] {
        const char* e = std::getenv("MG_MARCH2");
        return !(e && e[0] == '0');
    }();
    return v;
}

StepKernel march_kernel_f32(int nx, int nbuf, bool mass, int ty)
{
    // the tile of the 256^3 benchmark shape, specialised
    if (nx == 256 && nbuf == 3 && ty == 8) {
        if (march2_enabled())
            return mass ? ch_march2_kernel<256, 3, true, 8> : ch_march2_kernel<256, 3, false, 8>;
        return mass ? ch_march_kernel<float, 256, 3, true, 8> : ch_march_kernel<float, 256, 3, false, 8>;
    }
    if (march2_enabled() && nbuf == 3) {
        // the tiles a batch of cubes 64..192 gets at its default targets
        // (CTAs of ~320 threads, batch_tiling_for), specialised
        if (mass) {
            if (nx == 64 && ty == 32) return ch_march2_kernel<64, 3, true, 32>;
            if (nx == 96 && ty == 24) return ch_march2_kernel<96, 3, true, 24>;
            if (nx == 128 && ty == 16) return ch_march2_kernel<128, 3, true, 16>;
            if (nx == 160 && ty == 14) return ch_march2_kernel<160, 3, true, 14>;
            if (nx == 192 && ty == 11) return ch_march2_kernel<192, 3, true, 11>;
        }
        switch (nx) {
        case 64: return mass ? ch_march2_kernel<64, 3, true, 0> : ch_march2_kernel<64, 3, false, 0>;
        case 96: return mass ? ch_march2_kernel<96, 3, true, 0> : ch_march2_kernel<96, 3, false, 0>;
        case 128: return mass ? ch_march2_kernel<128, 3, true, 0> : ch_march2_kernel<128, 3, false, 0>;
        case 160: return mass ? ch_march2_kernel<160, 3, true, 0> : ch_march2_kernel<160, 3, false, 0>;
        case 192: return mass ? ch_march2_kernel<192, 3, true, 0> : ch_march2_kernel<192, 3, false, 0>;
        case 224: return mass ? ch_march2_kernel<224, 3, true, 0> : ch_march2_kernel<224, 3, false, 0>;
        case 256: return mass ? ch_march2_kernel<256, 3, true, 0> : ch_march2_kernel<256, 3, false, 0>;
        default: break;
        }
    }
    return mass ? march_f32_width<true>(nx, nbuf) : march_f32_width<false>(nx, nbuf);
}

}  // namespace mg
