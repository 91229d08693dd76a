// Device helpers shared by the colouring kernels: the Jones-Plassmann priority, the
// colouring control block and a bounded grid-wide barrier for cooperative launches.
#pragma once

#include "avbd_math.cuh"

namespace avbd
{

AVBD_DEV unsigned colour_priority(unsigned b)
{
    unsigned h = b * 0x9E3779B1u + 0x7F4A7C15u;
    h ^= h >> 16;
    h *= 0x85EBCA6Bu;
    h ^= h >> 13;
    h *= 0xC2B2AE35u;
    h ^= h >> 16;
    return h;
}

// Bounded grid-wide barrier for cooperative launches. Every wait has an iteration limit
// (BARRIER_SPIN_LIMIT unless the caller passes one); on expiry the kernel records an error
// and all blocks leave (the caller checks `error`).
constexpr int MAX_COLOUR_ROUNDS = 4096;
constexpr unsigned BARRIER_SPIN_LIMIT = 1u << 24;

struct ColourControl
{
    unsigned arrive; // barrier arrivals so far in this launch
    unsigned unused; // keeps the layout that readers of the block index by word
    int error;
    int vertices;
    int rounds;
    int maxColour;
    int coloured[MAX_COLOUR_ROUNDS];
};

// Arrivals count up through the launch (the control block starts zeroed): barrier k
// releases every block once k x gridDim.x blocks have arrived, so the last block's arrival
// alone opens it. `target` is the calling block's count of barriers passed x gridDim.x.
AVBD_DEV bool grid_barrier(ColourControl *ctl, unsigned &target, unsigned spinLimit = BARRIER_SPIN_LIMIT)
{
    __syncthreads();
    __shared__ int ok;
    target += gridDim.x;
    if (threadIdx.x == 0)
    {
        __threadfence();
        atomicAdd(&ctl->arrive, 1u);
        volatile unsigned *arrive = &ctl->arrive;
        unsigned spins = 0;
        while (*arrive < target && ++spins < spinLimit)
            if (spins > 256)
                __nanosleep(64);
        ok = spins < spinLimit;
        if (!ok)
            atomicExch(&ctl->error, 1);
        __threadfence();
    }
    __syncthreads();
    return ok && ((volatile int *)&ctl->error)[0] == 0;
}

AVBD_DEV int block_sum(int v)
{
    __shared__ int part[32];
    v = __reduce_add_sync(0xFFFFFFFFu, v);
    if ((threadIdx.x & 31) == 0)
        part[threadIdx.x >> 5] = v;
    __syncthreads();
    int s = 0;
    if (threadIdx.x < 32)
    {
        s = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0;
        s = __reduce_add_sync(0xFFFFFFFFu, s);
    }
    __syncthreads();
    return s; // valid in thread 0
}


} // namespace avbd
