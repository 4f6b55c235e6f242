// sketch.h - the minimizer k-mer hash shared by the host seeding (-S) and the
// device feature kernel of the band proposer.
//
// The hash is Thomas Wang's 64-bit integer hash as minimap2 (MIT, Heng Li)
// and minipoa (src/minimizer.cpp:11-21; MIT, Copyright (c) 2025 Haodong Liu)
// use it; identical minimizers need the identical function.
#pragma once
#include <stdint.h>

#ifndef PB_SKETCH_HD
#ifdef __CUDACC__
#define PB_SKETCH_HD __host__ __device__ __forceinline__
#else
#define PB_SKETCH_HD inline
#endif
#endif

namespace pb {

// Thomas Wang's 64-bit integer hash as the sketch uses it (src/minimizer.cpp:11-21):
// invertible on the masked 2k-bit k-mer code, so distinct k-mers never tie.
PB_SKETCH_HD uint64_t hash64(uint64_t key, uint64_t mask) {
    key = (~key + (key << 21)) & mask;
    key = key ^ key >> 24;
    key = ((key + (key << 3)) + (key << 8)) & mask;
    key = key ^ key >> 14;
    key = ((key + (key << 2)) + (key << 4)) & mask;
    key = key ^ key >> 28;
    key = (key + (key << 31)) & mask;
    return key;
}

}  // namespace pb
