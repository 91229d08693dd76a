// Constraint-graph colouring for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc at all: code running inside another framework's
// memory pool or allocator (which forbids raw device allocations), real-time loops that
// must not allocate after start-up, and hosts that pre-reserve every byte of the GPU.
// avbd_colour_graph_noalloc gives them the same Jones-Plassmann colouring that avbd_step
// computes for its primal sweep (k_colour_all), with all scratch memory in a fixed-size
// file-scope __device__ array of the library, so the call itself allocates nothing. Every
// GPU that loads the library holds this array (about 4 MiB) until the process exits.
// Under CUDA 12's default lazy module loading the driver loads this file's module onto a
// device, and places the array there, at the first call on that device (its
// cudaGetSymbolAddress); that first call is the one that needs the memory free, which is
// why callers make it at start-up. Later calls allocate nothing.
#include "../../include/avbd_cuda.h"
#include "avbd_colour.cuh"

#include <cuda_runtime.h>

#include <mutex>

using namespace avbd;

namespace
{

constexpr int NOALLOC_MAX_BODIES = AVBD_NOALLOC_MAX_BODIES;
constexpr size_t CONTROL_BYTES = (sizeof(ColourControl) + 255) / 256 * 256;
constexpr size_t SCRATCH_BYTES = CONTROL_BYTES + sizeof(int) * (size_t)NOALLOC_MAX_BODIES;

// Scratch of every call: the colouring control block, then one state word per body.
// In host code this name is only a host-side stand-in for the device symbol; kernels get
// the device address obtained with cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_setup_mutex;
void *g_scratch_address[MAX_DEVICES] = {};
int g_coop_blocks[MAX_DEVICES] = {};

// Same rounds as k_colour_all, over a caller-given neighbour CSR. A vertex is a body with
// vertex[b] != 0; neighbours outside [0, n) and non-vertices are ignored.
__global__ void k_colour_csr_noalloc(int n, const int *vertex, const int *adjStart, const int *adjOther, int mode,
                                     unsigned char *scratch, int *colourOut)
{
    ColourControl *ctl = (ColourControl *)scratch;
    int *state = (int *)(scratch + CONTROL_BYTES);
    const int stride = gridDim.x * blockDim.x;
    int mine = 0;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < n; b += stride)
    {
        bool v = vertex[b] != 0;
        __stcg(&state[b], v ? -1 : -2);
        mine += v ? 1 : 0;
    }
    int bs = block_sum(mine);
    if (threadIdx.x == 0 && bs)
        atomicAdd(&ctl->vertices, bs);
    unsigned target = 0;
    if (!grid_barrier(ctl, target))
        return;
    const int total = ((volatile int *)&ctl->vertices)[0];
    int done = 0, round = 0;
    for (; round < MAX_COLOUR_ROUNDS && done < total; ++round)
    {
        mine = 0;
        for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
        {
            if (__ldcg(&state[v]) != -1)
                continue;
            unsigned pv = mode ? colour_priority((unsigned)v) : 0xFFFFFFFFu - (unsigned)v;
            unsigned long long used[4] = {0ull, 0ull, 0ull, 0ull};
            bool isMax = true;
            for (int k = adjStart[v]; k < adjStart[v + 1]; ++k)
            {
                int u = adjOther[k];
                if (u < 0 || u >= n || u == v)
                    continue;
                int su = __ldcg(&state[u]);
                if (su == -2)
                    continue;
                if (su == -1 || (su >> 16) == round)
                {
                    unsigned pu = mode ? colour_priority((unsigned)u) : 0xFFFFFFFFu - (unsigned)u;
                    if (!(pv > pu || (pv == pu && v > u)))
                    {
                        isMax = false;
                        break;
                    }
                }
                else
                {
                    int c = su & 0xFFFF;
                    if (c < 256)
                        used[c >> 6] |= 1ull << (c & 63);
                }
            }
            if (!isMax)
                continue;
            int c = 0;
            while (c < 256 && ((used[c >> 6] >> (c & 63)) & 1ull))
                c++;
            if (c >= 256)
            {
                atomicExch(&ctl->error, 3);
                c = 255;
            }
            __stcg(&state[v], (round << 16) | c);
            atomicMax(&ctl->maxColour, c);
            mine++;
        }
        bs = block_sum(mine);
        if (threadIdx.x == 0 && bs)
            atomicAdd(&ctl->coloured[round], bs);
        if (!grid_barrier(ctl, target))
            return;
        done += ((volatile int *)ctl->coloured)[round];
    }
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < n; b += stride)
    {
        int s = __ldcg(&state[b]);
        colourOut[b] = s >= 0 ? (s & 0xFFFF) : -1;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
    {
        ctl->rounds = round;
        if (done < total)
            atomicCAS(&ctl->error, 0, 2);
    }
}

// Once per device, with that device current: the scratch array's device address and the
// co-resident block count for the cooperative launch.
int setup_device(int dev)
{
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (g_scratch_address[dev])
        return AVBD_OK;
    void *ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr)
        return AVBD_ERR_CUDA;
    int sms = 0, perSm = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_colour_csr_noalloc, 256, 0) != cudaSuccess)
        return AVBD_ERR_CUDA;
    g_coop_blocks[dev] = sms * (perSm > 0 ? perSm : 1);
    g_scratch_address[dev] = ptr;
    return AVBD_OK;
}

} // namespace

extern "C" int avbd_colour_graph_noalloc(int32_t n, const int32_t *vertex, const int32_t *adj_start,
                                         const int32_t *adj_other, int32_t mode, int32_t *colour,
                                         int32_t *num_colours, void *cuda_stream)
{
    if (!num_colours || n < 0 || (mode != AVBD_COLOUR_GREEDY && mode != AVBD_COLOUR_HASHED))
        return AVBD_ERR_ARGUMENT;
    if (n > NOALLOC_MAX_BODIES)
        return AVBD_ERR_CAPACITY;
    *num_colours = 0;
    if (n == 0)
        return AVBD_OK;
    if (!vertex || !adj_start || !adj_other || !colour)
        return AVBD_ERR_ARGUMENT;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES)
        return AVBD_ERR_CUDA;
    int rc = setup_device(dev);
    if (rc != AVBD_OK)
        return rc;
    cudaStream_t stream = (cudaStream_t)cuda_stream;
    unsigned char *scratch = (unsigned char *)g_scratch_address[dev];
    // the control block must start at zero; the state words are all written by the kernel
    if (cudaMemsetAsync(scratch, 0, sizeof(ColourControl), stream) != cudaSuccess)
        return AVBD_ERR_CUDA;
    int blocks = (n + 255) / 256;
    if (blocks > g_coop_blocks[dev])
        blocks = g_coop_blocks[dev];
    void *args[] = {&n, (void *)&vertex, (void *)&adj_start, (void *)&adj_other, &mode, &scratch, (void *)&colour};
    if (cudaLaunchCooperativeKernel((void *)k_colour_csr_noalloc, blocks, 256, args, 0, stream) != cudaSuccess)
        return AVBD_ERR_CUDA;
    int summary[6] = {0}; // arrive, unused, error, vertices, rounds, maxColour
    if (cudaMemcpyAsync(summary, scratch, sizeof(summary), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess)
        return AVBD_ERR_CUDA;
    if (summary[2] == 3)
        return AVBD_ERR_CAPACITY; // more than 256 colours needed
    if (summary[2] != 0)
        return AVBD_ERR_STATE; // a barrier wait expired or the round cap was reached
    *num_colours = summary[3] > 0 ? summary[5] + 1 : 0;
    return AVBD_OK;
}
