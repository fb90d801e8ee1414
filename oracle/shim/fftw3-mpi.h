// Test infrastructure for the oracle build only.
//
// The reference links FFTW-MPI for one call: fftw_mpi_local_size_3d, which
// gives each rank its x-slab (PFApp.cpp:46-52).  No transform is executed.
// This header answers that call with FFTW's documented default block
// distribution of the first dimension: block = ceil(n0 / np); rank r owns
// rows [r*block, min(n0, (r+1)*block)).
#pragma once

#include <cstddef>
#include "mpi.h"

inline void fftw_mpi_init() {}

inline ptrdiff_t fftw_mpi_local_size_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, MPI_Comm,
                                        ptrdiff_t* local_n0, ptrdiff_t* local_0_start)
{
    const ptrdiff_t np = MPI::COMM_WORLD.Get_size();
    const ptrdiff_t rank = MPI::COMM_WORLD.Get_rank();
    const ptrdiff_t block = (n0 + np - 1) / np;
    ptrdiff_t start = rank * block;
    if (start > n0) start = n0;
    ptrdiff_t count = n0 - start;
    if (count > block) count = block;
    *local_n0 = count;
    *local_0_start = start;
    return count * n1 * n2;
}
