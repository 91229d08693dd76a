// Device kernels of the AVBD step for sm_100a.
//
// Data layout (HBM, structure of arrays, one float4 per 3-vector so every load is a
// single 128-bit transaction):
//   bodies     pos/quat/initLin/initAng/inertLin/inertAng/vel/angvel/prevVel float4[n],
//              massMoment float4 (mass, moment xyz), sizeRad float4 (size xyz, radius), friction float
//   manifolds  ab int2, seq u64, n int, basis float4[3] (row0.w = friction),
//              contact float4[8][4]: (rA.xyz, rB.x) (rB.yz, C0.xy) (C0.z, penalty.xyz)
//                                     (lambda.xyz, key | stick << 31)
//   joints     ab int2, seq u64, float4[8]: (rA, stiffLin) (rB, stiffAng) (C0Lin, fracture)
//              (C0Ang, torqueArm) (penLin, broken) (penAng) (lamLin) (lamAng)
//   springs    ab int2, seq u64, float4[2]: (rA, rest) (rB, stiffness)
//   adjacency  CSR over bodies: entry = type << 30 | isA << 29 | index, newest force first
//
// Reference behaviour each kernel reproduces is cited at the kernel.
#pragma once

#include "avbd_colour.cuh"
#include "avbd_math.cuh"

namespace avbd
{

constexpr float PENALTY_MIN = 1.0f;
constexpr float PENALTY_MAX = 10000000000.0f;
constexpr float COLLISION_MARGIN = 0.01f;
constexpr float STICK_THRESH = 0.00001f;

constexpr unsigned ADJ_MANIFOLD = 0u, ADJ_JOINT = 1u, ADJ_SPRING = 2u, ADJ_IGNORE = 3u;
constexpr unsigned ADJ_INDEX_MASK = (1u << 29) - 1u;
constexpr unsigned ADJ_NONE = 0xFFFFFFFFu;

struct Params
{
    float dt, gravity;
    int iterations;
    float alpha, betaLin, betaAng, gamma;
};

struct DevBodies
{
    int n;
    float4 *pos, *quat, *initLin, *initAng, *inertLin, *inertAng, *vel, *angvel, *prevVel;
    // pose - initial pose: (pos - initLin, qdiff(quat, initAng)), written with the pose
    float4 *dqLin, *dqAng;
    // inverse(initAng) and inverse(inertAng), formed once per step by the warm start: every
    // qdiff against them in the iterations multiplies by the same inverse
    float4 *initAngInv, *inertAngInv;
    float4 *massMoment, *sizeRad;
    float *friction;
    float4 *shape; // (type, radius, half length, 0) per body; null when every body is a box
};

struct DevManifolds
{
    int2 *ab;
    unsigned long long *seq;
    int *n;
    float4 *basis;   // 3 per manifold
    float4 *contact; // 32 per manifold
};

struct DevForces
{
    int nMan;
    DevManifolds man;
    int nJoint;
    int2 *jointAB;
    unsigned long long *jointSeq;
    float4 *joint; // 8 per joint
    int nSpring;
    int2 *springAB;
    unsigned long long *springSeq;
    float4 *spring; // 2 per spring
    int nIgnore;
    int2 *ignoreAB;
    unsigned long long *ignoreSeq;
    int *adjStart; // n + 1
    unsigned *adj;
    // the constraint rows each body's primal solve stamps, in force order (rows_listed)
    int *rowStart; // n + 1
    int2 *rows;    // (force-list entry, (partner body + 1) << 3 | row of that force)
};

// The reference caps each grid at 2^22 cells (solver.cpp:341-357).
constexpr unsigned long long MAX_GRID_CELLS = 1ull << 22;

struct GridParams
{
    float bminx, bminy, bminz;
    float cellSize;
    int nx, ny, nz;
    unsigned long long numCells;
    float extx, exty, extz; // bounds extent of the binned centres
    float cellSize0;        // twice the binned radius, before the cell-count cap
    int capped;             // 1: the cell-count cap applies; the host recomputes the grid
};

// Device-side counters of one step.
struct StepCounters
{
    unsigned long long pairChecks;
    unsigned long long sphereHits;
    unsigned long long constrainedHits;
    int largePairs;
    int colouredThisRound;
    int maxColour;
    int error;
    int pairOverflow; // a grid entry found more new pairs than its recorded slots
    int orphans;      // live contacts or joints without a dynamic body (no row owns them)
};

enum DeviceError
{
    DERR_NONE = 0,
    DERR_TOO_MANY_COLOURS = 1,
    DERR_TOO_MANY_CELLS = 2
};

// Counts of a step that the device keeps for itself, so that a step runs without reading
// anything back to the host. Every kernel that changes the world checks `abort` first.
// The reasons a step stops before changing anything (the host redoes it with the
// synchronous path, which handles each case) come first; an error stops the step where it
// happens, latches, and every later step does nothing until the host reloads or clears.
enum StepAbort
{
    ABORT_NONE = 0,
    ABORT_JOINTS = 1,    // a joint broke in an earlier step: the joint list is compacted first
    ABORT_GRID = 2,      // the grid needs the reference's cell-count cap (host cbrtf)
    ABORT_MANIFOLDS = 3, // the new pairs do not fit the manifold buffers
    ABORT_NONFINITE = 4, // a body's position, orientation or velocity is not finite
    ABORT_ERROR = 5      // the colouring or an iteration wait failed (see `error`)
};

enum StepError
{
    STEP_ERR_NONE = 0,
    STEP_ERR_COLOURING = 1,     // the colouring's barrier wait expired or it ran out of rounds
    STEP_ERR_COLOURS = 2,       // the constraint graph needs more than 256 colours
    STEP_ERR_ITERATION = 3      // a grid barrier or partner wait of the iteration kernel expired
};

struct StepState
{
    int nMan;                    // live manifolds after the last compaction
    int nManBp;                  // live manifolds plus this step's new pairs
    int manBase;                 // first new manifold of this step
    int newBinned;               // new pairs from grid entries (the large-large pairs follow)
    unsigned long long nextSeq;  // sequence counter after this step's new pairs
    unsigned long long seqBase;  // sequence number of the step's first new manifold
    int abort;                   // StepAbort, sticky until the host clears it
    int error;                   // StepError of the failure that set ABORT_ERROR
    int stepsDone;               // steps that ran to the end
    int flips;                   // compactions that swapped the manifold buffers (a device step's compacts back without one)
    int nColours, nSolve, rounds;
    int created;                 // new manifolds of the last step
};

AVBD_DEV bool step_aborted(const StepState *st) { return st && ((volatile const int *)&st->abort)[0] != 0; }

AVBD_DEV void step_abort(StepState *st, int reason) { atomicCAS(&st->abort, 0, reason); }

AVBD_DEV unsigned adj_type(unsigned e) { return e >> 30; }
AVBD_DEV unsigned adj_isA(unsigned e) { return (e >> 29) & 1u; }
AVBD_DEV unsigned adj_index(unsigned e) { return e & ADJ_INDEX_MASK; }
AVBD_DEV unsigned make_adj(unsigned type, unsigned isA, unsigned index) { return (type << 30) | (isA << 29) | index; }

AVBD_DEV int2 force_bodies(const DevForces &F, unsigned e)
{
    unsigned i = adj_index(e);
    switch (adj_type(e))
    {
    case ADJ_MANIFOLD:
        return F.man.ab[i];
    case ADJ_JOINT:
        return F.jointAB[i];
    case ADJ_SPRING:
        return F.springAB[i];
    default:
        return F.ignoreAB[i];
    }
}

// Rigid::constrainedTo, walking the shorter force list (solver.cpp:197-205, rigid.cpp:105-116)
AVBD_DEV bool constrained(const DevForces &F, int a, int b)
{
    int da = F.adjStart[a + 1] - F.adjStart[a];
    int db = F.adjStart[b + 1] - F.adjStart[b];
    int self = da <= db ? a : b;
    int other = self == a ? b : a;
    for (int k = F.adjStart[self]; k < F.adjStart[self + 1]; ++k)
    {
        int2 ab = force_bodies(F, F.adj[k]);
        if ((ab.x == self && ab.y == other) || (ab.x == other && ab.y == self))
            return true;
    }
    return false;
}

// The set of body pairs some force links, as open-addressing keys (min << 32 | max), built
// from the force lists at the start of a step's broadphase: membership is exactly
// Rigid::constrainedTo (some force of either body joins the two), answered with one probe
// run instead of walking a force list. World-anchored joints never match a pair.
struct PairSet
{
    unsigned long long *keys = nullptr;
    unsigned mask = 0;
};

AVBD_DEV unsigned long long pair_key(int a, int b)
{
    unsigned lo = (unsigned)min(a, b), hi = (unsigned)max(a, b);
    return ((unsigned long long)lo << 32) | hi;
}

AVBD_DEV unsigned pair_slot(unsigned long long k, unsigned mask)
{
    k ^= k >> 31;
    k *= 0x9E3779B97F4A7C15ull;
    k ^= k >> 29;
    return (unsigned)k & mask;
}

AVBD_DEV bool pair_linked(const PairSet &S, int a, int b)
{
    const unsigned long long key = pair_key(a, b);
    unsigned h = pair_slot(key, S.mask);
    for (unsigned p = 0; p <= S.mask; ++p)
    {
        unsigned long long k = S.keys[h];
        if (k == key)
            return true;
        if (k == ~0ull)
            return false;
        h = (h + 1) & S.mask;
    }
    return false;
}

// constrainedTo through the pair set when there is one, else by walking the force lists.
AVBD_DEV bool linked(const DevForces &F, const PairSet &S, int a, int b)
{
    return S.keys ? pair_linked(S, a, b) : constrained(F, a, b);
}

// One thread per force (manifolds, joints, springs, ignore pairs): insert its body pair.
__global__ void k_pair_set(DevForces F, PairSet S, const StepState *st = nullptr)
{
    if (st)
        F.nMan = st->nMan;
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    int2 ab;
    if (f < F.nMan)
        ab = F.man.ab[f];
    else if ((f -= F.nMan) < F.nJoint)
        ab = F.jointAB[f];
    else if ((f -= F.nJoint) < F.nSpring)
        ab = F.springAB[f];
    else if ((f -= F.nSpring) < F.nIgnore)
        ab = F.ignoreAB[f];
    else
        return;
    if (ab.x < 0 || ab.y < 0)
        return;
    const unsigned long long key = pair_key(ab.x, ab.y);
    unsigned h = pair_slot(key, S.mask);
    for (unsigned p = 0; p <= S.mask; ++p)
    {
        unsigned long long prev = atomicCAS(&S.keys[h], ~0ull, key);
        if (prev == ~0ull || prev == key)
            return;
        h = (h + 1) & S.mask;
    }
}

// ---------------------------------------------------------------------------
// Broadphase: the reference's uniform grid (solver.cpp:284-486), one grid per world.
// W independent worlds are stepped together (W = 1 for one solver); each keeps its own
// 95th-percentile split, bounds, cell size, cell cap and large-body list, and pairs never
// cross worlds. Pairs come out in each world's creation order: sorted entry i, then the
// rest of its own cell, the 13 forward cells, the large bodies; large-large pairs last.
// Grid cells are found through hash tables keyed by (world, cell).
// ---------------------------------------------------------------------------

struct DevGrid
{
    int W;
    const int *bodyWorld;       // world of each body
    const int *worldStart;      // W + 1 body ranges
    const float *binnedRadius;  // per world
    const int *worldLargeStart; // W + 1 ranges in the large-body list
    unsigned *bounds;           // per world 8 words: ordered min xyz, max xyz, max binned slack
    GridParams *grid;           // per world
    int *cappedAny;
};

struct HashTable
{
    unsigned long long *keys;
    unsigned *vals;
    unsigned mask;
};

constexpr unsigned long long HASH_EMPTY = 0xFFFFFFFFFFFFFFFFull;
constexpr unsigned HASH_NONE = 0xFFFFFFFFu;

AVBD_DEV unsigned hash_slot(unsigned long long k, unsigned mask)
{
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return (unsigned)k & mask;
}

AVBD_DEV void hash_insert(const HashTable &t, unsigned long long key, unsigned val)
{
    unsigned h = hash_slot(key, t.mask);
    for (unsigned probe = 0; probe <= t.mask; ++probe)
    {
        unsigned long long prev = atomicCAS(&t.keys[h], HASH_EMPTY, key);
        if (prev == HASH_EMPTY || prev == key)
        {
            t.vals[h] = val;
            return;
        }
        h = (h + 1) & t.mask;
    }
}

AVBD_DEV unsigned hash_find(const HashTable &t, unsigned long long key)
{
    unsigned h = hash_slot(key, t.mask);
    for (unsigned probe = 0; probe <= t.mask; ++probe)
    {
        unsigned long long k = t.keys[h];
        if (k == key)
            return t.vals[h];
        if (k == HASH_EMPTY)
            return HASH_NONE;
        h = (h + 1) & t.mask;
    }
    return HASH_NONE;
}

// Sorted grid entry: world (16 bits) | cell (22) | body (24); its run id (world, cell)
// is key >> 24. Body indices within a world keep the world's list order.
AVBD_DEV unsigned long long grid_key(int w, unsigned cell, int b)
{
    return ((unsigned long long)w << 46) | ((unsigned long long)cell << 24) | (unsigned)b;
}
AVBD_DEV int key_body(unsigned long long k) { return (int)(k & 0xFFFFFFull); }
AVBD_DEV int key_world(unsigned long long k) { return (int)(k >> 46); }
AVBD_DEV unsigned key_cell(unsigned long long k) { return (unsigned)((k >> 24) & 0x3FFFFFull); }

AVBD_DEV unsigned float_order(float f)
{
    unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
AVBD_DEV float float_unorder(unsigned u) { return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u); }

__global__ void k_bp_bounds_init(unsigned *bounds, int W)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= 8 * W)
        return;
    int slot = k & 7;
    bounds[k] = slot < 3 ? 0xFFFFFFFFu : 0u; // min slots, then max slots and the largest binned slack
}

// Bounds of each world's binned centres and its largest binned travel slack
// (solver.cpp:306-333). Each thread folds its grid-stride items while they stay in one world
// (bodies of a world are contiguous in the binned list), then warps and the block combine
// the folds of one world before their atomics: a single world costs one set of atomics per
// block.
AVBD_DEV void bounds_reset(unsigned v[7])
{
#pragma unroll
    for (int d = 0; d < 7; ++d)
        v[d] = d < 3 ? 0xFFFFFFFFu : 0u;
}
AVBD_DEV void bounds_flush(const DevGrid &G, int w, const unsigned v[7])
{
    unsigned *bw = G.bounds + 8 * w;
    for (int d = 0; d < 3; ++d)
        atomicMin(&bw[d], v[d]);
    for (int d = 3; d < 7; ++d)
        atomicMax(&bw[d], v[d]);
}
// Warp combine of (world, fold): when every lane with a fold shares one world, the warp's
// fold ends in every lane and the world is returned; otherwise each lane flushes its own
// fold and -1 is returned.
AVBD_DEV int bounds_warp_combine(const DevGrid &G, int w, unsigned v[7])
{
    int wref = __reduce_max_sync(0xFFFFFFFFu, w);
    if (!__all_sync(0xFFFFFFFFu, w == wref || w < 0))
    {
        if (w >= 0)
            bounds_flush(G, w, v);
        bounds_reset(v);
        return -1;
    }
#pragma unroll
    for (int d = 0; d < 3; ++d)
        v[d] = __reduce_min_sync(0xFFFFFFFFu, v[d]);
#pragma unroll
    for (int d = 3; d < 7; ++d)
        v[d] = __reduce_max_sync(0xFFFFFFFFu, v[d]);
    return wref;
}
__global__ void __launch_bounds__(256) k_bp_bounds(DevBodies B, DevGrid G, const int *binned, int nBinned, float dt)
{
    __shared__ unsigned sv[8][7];
    __shared__ int sw[8];
    unsigned v[7];
    bounds_reset(v);
    int cw = -1;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nBinned; k += gridDim.x * blockDim.x)
    {
        int b = binned[k];
        int w = G.bodyWorld[b];
        if (w != cw)
        {
            if (cw >= 0)
                bounds_flush(G, cw, v);
            bounds_reset(v);
            cw = w;
        }
        float4 p = B.pos[b];
        unsigned x = float_order(p.x), y = float_order(p.y), z = float_order(p.z);
        v[0] = min(v[0], x);
        v[1] = min(v[1], y);
        v[2] = min(v[2], z);
        v[3] = max(v[3], x);
        v[4] = max(v[4], y);
        v[5] = max(v[5], z);
        v[6] = max(v[6], __float_as_uint(len(xyz(B.vel[b])) * dt));
    }
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int ww = bounds_warp_combine(G, cw, v);
    if (lane == 0)
    {
        sw[warp] = ww;
#pragma unroll
        for (int d = 0; d < 7; ++d)
            sv[warp][d] = v[d];
    }
    __syncthreads();
    if (warp != 0)
        return;
    int bw = -1;
    if (lane < (int)(blockDim.x >> 5))
    {
        bw = sw[lane];
#pragma unroll
        for (int d = 0; d < 7; ++d)
            v[d] = sv[lane][d];
    }
    else
        bounds_reset(v);
    bw = bounds_warp_combine(G, bw, v);
    if (lane == 0 && bw >= 0)
        bounds_flush(G, bw, v);
}

// World AABB plus travel slack of the bodies too large for the grid (solver.cpp:311-327)
__global__ void k_bp_large(DevBodies B, const int *large, int nLarge, float dt, float4 *lo, float4 *hi,
                           float4 *sphere)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nLarge)
        return;
    int b = large[k];
    float3 p = xyz(B.pos[b]);
    float4 q = B.quat[b];
    float4 sr = B.sizeRad[b];
    float slack = len(xyz(B.vel[b])) * dt;
    float3 h = f3(sr.w, sr.w, sr.w); // round shapes: the bounding radius (solver.cpp:315-326)
    if (!B.shape || B.shape[b].x == 0.0f)
    {
        float3 e = mul(xyz(sr), 0.5f);
        float3 cx = rotate(q, f3(1, 0, 0));
        float3 cy = rotate(q, f3(0, 1, 0));
        float3 cz = rotate(q, f3(0, 0, 1));
        h = f3(fabsf(cx.x) * e.x + fabsf(cy.x) * e.y + fabsf(cz.x) * e.z,
               fabsf(cx.y) * e.x + fabsf(cy.y) * e.y + fabsf(cz.y) * e.z,
               fabsf(cx.z) * e.x + fabsf(cy.z) * e.y + fabsf(cz.z) * e.z);
    }
    lo[k] = f4(sub(p, h), slack);
    hi[k] = f4(add(p, h), slack);
    sphere[k] = f4(p, sr.w);
}

// Cell size and grid dimensions per world (solver.cpp:338-357). When the cell count
// exceeds the cap the reference grows the cells by cbrtf factors; that rescaling is redone
// on the host with the C library's cbrtf (the one the reference calls), so the device only
// flags it and leaves a one-cell placeholder grid.
__global__ void k_bp_params(DevGrid G, const int *worldBinned)
{
    int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= G.W)
        return;
    GridParams g;
    const unsigned *bw = G.bounds + 8 * w;
    float cellSize = G.binnedRadius[w] * 2.0f;
    if (worldBinned[w] == 0)
    {
        g.bminx = g.bminy = g.bminz = 0.0f;
        g.extx = g.exty = g.extz = 0.0f;
        g.cellSize = g.cellSize0 = cellSize;
        g.nx = g.ny = g.nz = 1;
        g.numCells = 1;
        g.capped = 0;
        G.grid[w] = g;
        return;
    }
    float bminx = float_unorder(bw[0]), bminy = float_unorder(bw[1]), bminz = float_unorder(bw[2]);
    float bmaxx = float_unorder(bw[3]), bmaxy = float_unorder(bw[4]), bmaxz = float_unorder(bw[5]);
    float3 extent = f3(bmaxx - bminx, bmaxy - bminy, bmaxz - bminz);
    g.extx = extent.x;
    g.exty = extent.y;
    g.extz = extent.z;
    g.cellSize0 = cellSize;
    int nx = (int)(extent.x / cellSize) + 1;
    int ny = (int)(extent.y / cellSize) + 1;
    int nz = (int)(extent.z / cellSize) + 1;
    unsigned long long numCells = (unsigned long long)nx * (unsigned long long)ny * (unsigned long long)nz;
    g.capped = numCells > MAX_GRID_CELLS ? 1 : 0;
    if (g.capped)
    {
        nx = ny = nz = 1;
        numCells = 1;
        atomicOr(G.cappedAny, 1);
    }
    g.bminx = bminx;
    g.bminy = bminy;
    g.bminz = bminz;
    g.cellSize = cellSize;
    g.nx = nx;
    g.ny = ny;
    g.nz = nz;
    g.numCells = numCells;
    G.grid[w] = g;
}

AVBD_DEV int grid_axis(float x, float bmin, float cellSize, int n)
{
    return (int)rclamp((x - bmin) / cellSize, 0.0f, (float)(n - 1));
}

__global__ void k_bp_keys(DevBodies B, DevGrid G, const int *binned, int nBinned, unsigned long long *keys)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nBinned)
        return;
    int b = binned[k];
    int w = G.bodyWorld[b];
    float4 c = B.pos[b];
    GridParams g = G.grid[w];
    int ix = grid_axis(c.x, g.bminx, g.cellSize, g.nx);
    int iy = grid_axis(c.y, g.bminy, g.cellSize, g.ny);
    int iz = grid_axis(c.z, g.bminz, g.cellSize, g.nz);
    unsigned cell = (unsigned)(ix + g.nx * (iy + g.ny * iz));
    if (g.numCells > MAX_GRID_CELLS || cell >= MAX_GRID_CELLS)
        cell = 0; // only with a placeholder grid or non-finite positions; that step is recounted
    keys[k] = grid_key(w, cell, b);
}

// First entry of every (world, cell) run, into a hash table (the reference's cell-start table).
__global__ void k_bp_hash_runs(const unsigned long long *keys, int n, HashTable t)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    unsigned long long run = keys[k] >> 24;
    if (keys[k] == HASH_EMPTY)
        return;
    if (k == 0 || (keys[k - 1] >> 24) != run)
        hash_insert(t, run, (unsigned)k);
}

// Large bodies are binned into their world's grid with their AABB inflated by an upper
// bound of the reference's reach (binned radius + travel slacks + 4 margins,
// solver.cpp:449-458), so a binned body only tests the large bodies listed for its own
// cell; the reference's exact predicate still decides every pair. Bodies spanning more than
// LARGE_MAX_CELLS cells (ground slabs) go to their world's global list, which every binned
// body of that world tests. Key: world (16) | global (1) | cell (22) | large index (24).
constexpr int LARGE_MAX_CELLS = 64;

AVBD_DEV unsigned long long large_key(int w, int global, unsigned cell, int l)
{
    return ((unsigned long long)w << 47) | ((unsigned long long)global << 46) | ((unsigned long long)cell << 24) |
           (unsigned)l;
}
AVBD_DEV unsigned long long large_run(int w, int global, unsigned cell)
{
    return ((unsigned long long)w << 23) | ((unsigned long long)global << 22) | cell;
}

__global__ void k_bp_large_cells(DevGrid G, const int *large, const float4 *largeLo, const float4 *largeHi, int nLarge,
                                 unsigned long long *keys)
{
    int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nLarge)
        return;
    int w = G.bodyWorld[large[l]];
    GridParams g = G.grid[w];
    float4 lo = largeLo[l], hi = largeHi[l];
    float slackMax = __uint_as_float(G.bounds[8 * w + 6]);
    float R = (G.binnedRadius[w] + slackMax + lo.w + 4.0f * COLLISION_MARGIN) * 1.001f + 1.0e-4f;
    int x0 = grid_axis(lo.x - R, g.bminx, g.cellSize, g.nx), x1 = grid_axis(hi.x + R, g.bminx, g.cellSize, g.nx);
    int y0 = grid_axis(lo.y - R, g.bminy, g.cellSize, g.ny), y1 = grid_axis(hi.y + R, g.bminy, g.cellSize, g.ny);
    int z0 = grid_axis(lo.z - R, g.bminz, g.cellSize, g.nz), z1 = grid_axis(hi.z + R, g.bminz, g.cellSize, g.nz);
    long long cells = (long long)(x1 - x0 + 1) * (y1 - y0 + 1) * (z1 - z0 + 1);
    bool finite = isfinite(lo.x) && isfinite(lo.y) && isfinite(lo.z) && isfinite(hi.x) && isfinite(hi.y) &&
                  isfinite(hi.z) && isfinite(R);
    unsigned long long *out = keys + (size_t)l * LARGE_MAX_CELLS;
    int k = 0;
    if (!finite || cells <= 0 || cells > LARGE_MAX_CELLS || g.numCells > MAX_GRID_CELLS)
        out[k++] = large_key(w, 1, 0u, l);
    else
        for (int z = z0; z <= z1; ++z)
            for (int y = y0; y <= y1; ++y)
                for (int x = x0; x <= x1; ++x)
                    out[k++] = large_key(w, 0, (unsigned)(x + g.nx * (y + g.ny * z)), l);
    for (; k < LARGE_MAX_CELLS; ++k)
        out[k] = HASH_EMPTY;
}

__global__ void k_bp_hash_large_runs(const unsigned long long *keys, int n, HashTable t)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n || keys[k] == HASH_EMPTY)
        return;
    unsigned long long run = keys[k] >> 24;
    if (k == 0 || (keys[k - 1] >> 24) != run)
        hash_insert(t, run, (unsigned)k);
}

__constant__ int c_forward[13][3] = {{1, 0, 0},   {-1, 1, 0}, {0, 1, 0},  {1, 1, 0}, {-1, -1, 1},
                                     {0, -1, 1},  {1, -1, 1}, {-1, 0, 1}, {0, 0, 1}, {1, 0, 1},
                                     {-1, 1, 1},  {0, 1, 1},  {1, 1, 1}};

constexpr int LL_CHUNK = 128;

// Warp-aggregated add of per-thread statistics (one atomic per warp).
AVBD_DEV void warp_add(unsigned long long *dst, unsigned v)
{
    unsigned s = __reduce_add_sync(0xFFFFFFFFu, v);
    if ((threadIdx.x & 31) == 0 && s)
        atomicAdd(dst, (unsigned long long)s);
}

// Modes of the grid-entry pass: count (and record), emit every entry's pairs by searching
// again, or emit what the counting pass recorded and search again only for the parts of an
// entry that found more than BP_SLOTS.
constexpr int BP_COUNT = 0, BP_EMIT = 1, BP_EMIT_RECORDED = 2;

// Each sorted grid entry i (solver.cpp:405-465) is worked on by BP_LANES lanes, one per part
// of its search, in the reference's visiting order: lane 0 the rest of its own cell, lanes 1
// to 13 the 13 forward cells, lane 14 the large bodies (visited in list order: the entry's
// cell candidates merged with its world's global list, both sorted by large index); lane 15
// idles. A lane's new (unconstrained) hits form a consecutive run of the entry's pairs, placed
// after the runs of the lanes before it, so the entry's hit order is the reference's.
// BP_COUNT counts each lane's hits (laneCounts), records its first BP_SLOTS partners and
// writes the entry's total (counts); the emitting modes write them as fresh manifolds at
// base + offset[i] + the lane's place; with a device step state they take base and seqBase
// from it.
constexpr int BP_SLOTS = 8;  // new pairs each lane records in the counting pass
constexpr unsigned BP_UNRECORDED = 1u << 30; // lane count flag: its partners were not recorded
constexpr int BP_LANES = 16; // lanes per grid entry (15 parts)

template <int MODE>
__global__ void __launch_bounds__(128) k_bp_pairs(DevBodies B, DevForces F, DevGrid G, const unsigned long long *keys,
                                                  int nBinned, HashTable cells, const int *large,
                                                  const float4 *largeLo, const float4 *largeHi,
                                                  const unsigned long long *largeKeys, HashTable largeCells, float dt,
                                                  int *counts, const int *offsets, int base, unsigned long long seqBase,
                                                  StepCounters *cnt, int *recorded, int *laneCounts,
                                                  const StepState *st = nullptr, PairSet S = PairSet(),
                                                  unsigned partMask = 0x7FFFu)
{
    constexpr bool EMIT = MODE != BP_COUNT;
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int i = (int)(tid / BP_LANES);
    const int part = (int)(tid % BP_LANES);
    const bool entry = i < nBinned;
    if (EMIT && st)
    {
        if (step_aborted(st))
            return;
        base = st->manBase;
        seqBase = st->seqBase;
    }
    const size_t slot0 = ((size_t)i * BP_LANES + part) * BP_SLOTS;
    // the lane's place among the entry's new pairs: the runs of the lanes before it
    int place = 0, mine = 0;
    bool recordedOk = true;
    if (EMIT)
    {
        const int raw = entry ? laneCounts[(size_t)i * BP_LANES + part] : 0;
        mine = raw & ~(int)BP_UNRECORDED;
        recordedOk = (raw & (int)BP_UNRECORDED) == 0;
        int incl = mine;
#pragma unroll
        for (int d = 1; d < BP_LANES; d <<= 1)
        {
            int v = __shfl_up_sync(0xFFFFFFFFu, incl, d, BP_LANES);
            if (part >= d)
                incl += v;
        }
        place = incl - mine;
    }
    bool active = entry && part < 15 && ((partMask >> part) & 1u);
    if (MODE == BP_EMIT_RECORDED && active && mine <= BP_SLOTS && recordedOk)
    {
        if (mine > 0)
        {
            const int a = key_body(keys[i]);
            const int out = base + offsets[i] + place;
            for (int f = 0; f < mine; ++f)
            {
                const int m = out + f;
                F.man.ab[m] = make_int2(a, recorded[slot0 + f]);
                F.man.seq[m] = seqBase + (unsigned long long)(m - base);
                F.man.n[m] = 0;
            }
        }
        active = false;
    }
    if (MODE == BP_EMIT_RECORDED && active && mine == 0)
        active = false;
    unsigned checks = 0, hits = 0, cons = 0;
    int found = 0;
    if (active)
    {
        unsigned long long ki = keys[i];
        const int w = key_world(ki);
        const unsigned akey = key_cell(ki);
        const int a = key_body(ki);
        float3 ac = xyz(B.pos[a]);
        float ar = B.sizeRad[a].w;
        int out = EMIT ? base + offsets[i] + place : 0;

        auto hit = [&](int bIdx) {
            hits++;
            if (linked(F, S, a, bIdx))
            {
                cons++;
                return;
            }
            if (EMIT)
            {
                int m = out + found;
                F.man.ab[m] = make_int2(a, bIdx);
                F.man.seq[m] = seqBase + (unsigned long long)(m - base);
                F.man.n[m] = 0;
            }
            else if (found < BP_SLOTS)
                recorded[slot0 + found] = bIdx;
            found++;
        };
        auto test = [&](int j) {
            checks++;
            int bIdx = key_body(keys[j]);
            float3 dp = sub(ac, xyz(B.pos[bIdx]));
            float r = ar + B.sizeRad[bIdx].w;
            if (!(dot(dp, dp) > r * r))
                hit(bIdx);
        };
        if (part == 0)
        {
            const unsigned long long arun = ki >> 24;
            for (int j = i + 1; j < nBinned && (keys[j] >> 24) == arun; ++j)
                test(j);
        }
        else if (part <= 13)
        {
            const GridParams g = G.grid[w];
            const int d = part - 1;
            int ix = (int)(akey % (unsigned)g.nx);
            unsigned t = akey / (unsigned)g.nx;
            int iy = (int)(t % (unsigned)g.ny);
            int iz = (int)(t / (unsigned)g.ny);
            int cx = ix + c_forward[d][0], cy = iy + c_forward[d][1], cz = iz + c_forward[d][2];
            if (!(cx < 0 || cx >= g.nx || cy < 0 || cy >= g.ny || cz < 0 || cz >= g.nz))
            {
                unsigned long long nrun = ((unsigned long long)w << 22) | (unsigned)(cx + g.nx * (cy + g.ny * cz));
                unsigned s = hash_find(cells, nrun);
                if (s != HASH_NONE)
                    for (int j = (int)s; j < nBinned && (keys[j] >> 24) == nrun; ++j)
                        test(j);
            }
        }
        else
        {
            const int nLargeW = G.worldLargeStart[w + 1] - G.worldLargeStart[w];
            if (nLargeW > 0)
            {
                // the reference tests every large body of the world; all that can pass are here
                checks += (unsigned)nLargeW;
                const float aslack = len(xyz(B.vel[a])) * dt;
                const float margin4 = 4.0f * COLLISION_MARGIN;
                auto test_large = [&](int l) {
                    float4 lo = largeLo[l], hi = largeHi[l];
                    float3 q = f3(rclamp(ac.x, lo.x, hi.x), rclamp(ac.y, lo.y, hi.y), rclamp(ac.z, lo.z, hi.z));
                    float3 dp = sub(ac, q);
                    float reach = ar + aslack + lo.w + margin4;
                    if (dot(dp, dp) > reach * reach)
                        return;
                    hit(large[l]);
                };
                const unsigned long long crun = large_run(w, 0, akey), grun = large_run(w, 1, 0u);
                unsigned cs = hash_find(largeCells, crun);
                unsigned gs = hash_find(largeCells, grun);
                int jc = cs == HASH_NONE ? -1 : (int)cs;
                int jg = gs == HASH_NONE ? -1 : (int)gs;
                auto next = [&](int j, unsigned long long run) -> unsigned {
                    if (j < 0)
                        return 0xFFFFFFFFu;
                    unsigned long long v = largeKeys[j];
                    return (v != HASH_EMPTY && (v >> 24) == run) ? (unsigned)(v & 0xFFFFFFull) : 0xFFFFFFFFu;
                };
                unsigned lc = next(jc, crun), lg = next(jg, grun);
                while (lc != 0xFFFFFFFFu || lg != 0xFFFFFFFFu)
                {
                    if (lc < lg)
                    {
                        test_large((int)lc);
                        lc = next(++jc, crun);
                    }
                    else
                    {
                        test_large((int)lg);
                        lg = next(++jg, grun);
                    }
                }
            }
        }
    }
    if (!EMIT)
    {
        if (entry)
            laneCounts[(size_t)i * BP_LANES + part] = found;
        if (found > BP_SLOTS)
            cnt->pairOverflow = 1;
        // the entry's total
        int total = found;
#pragma unroll
        for (int d = BP_LANES / 2; d > 0; d >>= 1)
            total += __shfl_down_sync(0xFFFFFFFFu, total, d, BP_LANES);
        if (entry && part == 0)
            counts[i] = total;
        warp_add(&cnt->pairChecks, checks);
        warp_add(&cnt->sphereHits, hits);
        warp_add(&cnt->constrainedHits, cons);
    }
}

// ---------------------------------------------------------------------------
// Sorted-Morton LBVH broadphase mode: a bounding volume hierarchy over each world's binned
// bodies (Morton codes of the centres, radix-sorted; Karras's radix-tree construction;
// bottom-up refit of the spheres' boxes) finds each grid entry's binned partners. It is only
// the candidate generator: every candidate keeps the grid's own order and test (the entry
// owns a pair when the partner lies later in its own cell or in one of its 13 forward
// cells, solver.cpp:405-447; the reference's exact FP32 sphere predicate decides), so the
// pair set and creation order are the grid's.
// ---------------------------------------------------------------------------

AVBD_DEV unsigned morton_spread10(unsigned v)
{
    v &= 0x3FFu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

AVBD_DEV unsigned morton_axis(float x, float bmin, float extent)
{
    float f = extent > 0.0f ? (x - bmin) / extent : 0.0f;
    f = fminf(fmaxf(f, 0.0f), 1.0f); // also maps NaN to 0
    return (unsigned)(f * 1023.0f);
}

// Morton code of every binned centre inside its world's bounds, keyed by world.
__global__ void k_lbvh_codes(DevBodies B, DevGrid G, const int *binned, int nB, unsigned long long *keys, int *bodies)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nB)
        return;
    int b = binned[k];
    int w = G.bodyWorld[b];
    GridParams g = G.grid[w];
    float4 c = B.pos[b];
    unsigned code = (morton_spread10(morton_axis(c.x, g.bminx, g.extx)) << 2) |
                    (morton_spread10(morton_axis(c.y, g.bminy, g.exty)) << 1) |
                    morton_spread10(morton_axis(c.z, g.bminz, g.extz));
    keys[k] = ((unsigned long long)w << 32) | code;
    bodies[k] = b;
}

// A radius padded far above the FP32 rounding of boxes and distances at this position
// (relative 1e-5 of the radius, 4e-7 of the coordinates, 1e-4 m).
AVBD_DEV float lbvh_pad(float r, float4 c)
{
    return r * 1.00001f + 1.0e-4f + 4.0e-7f * (fabsf(c.x) + fabsf(c.y) + fabsf(c.z));
}

struct Lbvh
{
    const unsigned long long *codes; // sorted (world, Morton) keys
    const int *bodies;               // body of each sorted leaf
    const int *segStart;             // W + 1 leaf ranges, one tree per world
    int W, n;                        // worlds, leaves
    int *child;                      // 2 per internal node; a leaf child is encoded as -1 - leaf
    int *parent;                     // internal nodes [0, n), leaves [n, 2n); -1 at a root
    float4 *lo, *hi;                 // boxes: internal nodes [0, n), leaves [n, 2n)
    unsigned *arrivals;              // per internal node, for the refit
};

AVBD_DEV int lbvh_world(const Lbvh &T, int k)
{
    int lo = 0, hi = T.W; // last w with segStart[w] <= k
    while (hi - lo > 1)
    {
        int mid = (lo + hi) >> 1;
        if (T.segStart[mid] <= k)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// Common-prefix length of leaves i and j of a segment (the index breaks ties of equal codes).
AVBD_DEV int lbvh_delta(const Lbvh &T, int s, int m, int i, int j)
{
    if (j < 0 || j >= m)
        return -1;
    unsigned a = (unsigned)T.codes[s + i], b = (unsigned)T.codes[s + j];
    return a == b ? 32 + __clz((unsigned)(i ^ j)) : __clz(a ^ b);
}

// Internal node i of its world's tree (Karras, "Maximizing parallelism in the construction
// of BVHs, octrees and k-d trees", 2012): the range it covers and the split inside it. A
// world of m leaves has m - 1 internal nodes, stored from the world's first leaf slot on.
__global__ void k_lbvh_build(Lbvh T)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= T.n)
        return;
    const int w = lbvh_world(T, k);
    const int s = T.segStart[w], m = T.segStart[w + 1] - s, i = k - s;
    if (i >= m - 1)
        return;
    const int d = lbvh_delta(T, s, m, i, i + 1) > lbvh_delta(T, s, m, i, i - 1) ? 1 : -1;
    const int dmin = lbvh_delta(T, s, m, i, i - d);
    int lmax = 2;
    while (lbvh_delta(T, s, m, i, i + lmax * d) > dmin)
        lmax *= 2;
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2)
        if (lbvh_delta(T, s, m, i, i + (l + t) * d) > dmin)
            l += t;
    const int j = i + l * d;
    const int dnode = lbvh_delta(T, s, m, i, j);
    int split = 0;
    for (int div = 2;; div *= 2)
    {
        int t = (l + div - 1) / div;
        if (lbvh_delta(T, s, m, i, i + (split + t) * d) > dnode)
            split += t;
        if (t <= 1)
            break;
    }
    const int gamma = i + split * d + min(d, 0);
    const int left = min(i, j) == gamma ? -1 - (s + gamma) : s + gamma;
    const int right = max(i, j) == gamma + 1 ? -1 - (s + gamma + 1) : s + gamma + 1;
    T.child[2 * k] = left;
    T.child[2 * k + 1] = right;
    T.parent[left < 0 ? T.n + (-1 - left) : left] = k;
    T.parent[right < 0 ? T.n + (-1 - right) : right] = k;
}

// Leaf boxes (the sphere, padded far above FP32 rounding) and, bottom-up, every internal
// node's box: the second child to arrive at a node combines both.
__global__ void k_lbvh_refit(Lbvh T, DevBodies B)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= T.n)
        return;
    const int b = T.bodies[k];
    const float4 c = B.pos[b];
    const float r = lbvh_pad(B.sizeRad[b].w, c);
    float4 lo = make_float4(c.x - r, c.y - r, c.z - r, 0.0f), hi = make_float4(c.x + r, c.y + r, c.z + r, 0.0f);
    __stcg(&T.lo[T.n + k], lo);
    __stcg(&T.hi[T.n + k], hi);
    int node = T.parent[T.n + k];
    while (node >= 0)
    {
        __threadfence();
        if (atomicAdd(&T.arrivals[node], 1u) == 0u)
            return; // the other child finishes this node
        const int cl = T.child[2 * node], cr = T.child[2 * node + 1];
        const int il = cl < 0 ? T.n + (-1 - cl) : cl, ir = cr < 0 ? T.n + (-1 - cr) : cr;
        const float4 al = __ldcg(&T.lo[il]), ah = __ldcg(&T.hi[il]), bl = __ldcg(&T.lo[ir]), bh = __ldcg(&T.hi[ir]);
        lo = make_float4(fminf(al.x, bl.x), fminf(al.y, bl.y), fminf(al.z, bl.z), 0.0f);
        hi = make_float4(fmaxf(ah.x, bh.x), fmaxf(ah.y, bh.y), fmaxf(ah.z, bh.z), 0.0f);
        __stcg(&T.lo[node], lo);
        __stcg(&T.hi[node], hi);
        node = T.parent[node];
    }
}

// Sorted grid position of every binned body.
__global__ void k_grid_entry_of(const unsigned long long *keys, int nB, int *entryOf)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nB)
        entryOf[key_body(keys[k])] = k;
}

// Forward-stencil slot (0..12) of a neighbour cell offset, -1 when it is not forward.
AVBD_DEV int forward_slot(int dx, int dy, int dz)
{
    if (dx < -1 || dx > 1 || dy < -1 || dy > 1 || dz < -1 || dz > 1)
        return -1;
    const int code = (dx + 1) + 3 * (dy + 1) + 9 * (dz + 1); // 13 = (0, 0, 0)
    return code > 13 ? code - 14 : -1;
}

constexpr int LBVH_TUPLES = 32;              // owned hits an entry keeps for recording
constexpr int LBVH_STACK = 128; // tree depth is at most 64 (32 code + 32 index bits)

// The binned parts (lanes 0..13 of k_bp_pairs) of grid entry i, found by traversing its
// world's tree with its bounding sphere: each owned candidate is tested with the grid's
// predicate; hits that no force links are counted per part and recorded in the part's
// order (ascending grid position); the large-body part was counted by k_bp_pairs already
// (laneCounts lane 14), so the entry's total is written here.
__global__ void k_lbvh_count(DevBodies B, DevForces F, DevGrid G, Lbvh T, const unsigned long long *keys, int nB,
                             const int *entryOf, int *counts, int *laneCounts, int *recorded, StepCounters *cnt,
                             PairSet S)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned checks = 0, hits = 0, cons = 0;
    if (i < nB)
    {
        const unsigned long long ki = keys[i];
        const int a = key_body(ki), w = key_world(ki);
        const unsigned ca = key_cell(ki);
        const GridParams g = G.grid[w];
        const int ax = (int)(ca % (unsigned)g.nx);
        const unsigned t0 = ca / (unsigned)g.nx;
        const int ay = (int)(t0 % (unsigned)g.ny), az = (int)(t0 / (unsigned)g.ny);
        const float4 pa = B.pos[a];
        const float3 ac = xyz(pa);
        const float ar = B.sizeRad[a].w, reach = lbvh_pad(ar, pa);
        int partCount[14];
#pragma unroll
        for (int q = 0; q < 14; ++q)
            partCount[q] = 0;
        unsigned tupleKey[LBVH_TUPLES];
        int tupleBody[LBVH_TUPLES];
        int tuples = 0;
        bool complete = true;
        const int s0 = T.segStart[w], m = T.segStart[w + 1] - s0;
        int stack[LBVH_STACK];
        int top = 0;
        if (m >= 2)
            stack[top++] = s0;
        while (top > 0)
        {
            const int node = stack[--top];
            const int cl = T.child[2 * node], cr = T.child[2 * node + 1];
#pragma unroll
            for (int side = 0; side < 2; ++side)
            {
                const int c = side == 0 ? cl : cr;
                const int box = c < 0 ? T.n + (-1 - c) : c;
                const float4 lo = T.lo[box], hi = T.hi[box];
                const float3 q = f3(fminf(fmaxf(ac.x, lo.x), hi.x), fminf(fmaxf(ac.y, lo.y), hi.y),
                                    fminf(fmaxf(ac.z, lo.z), hi.z));
                const float3 dq = sub(ac, q);
                if (!(dot(dq, dq) <= reach * reach) && isfinite(ac.x + ac.y + ac.z))
                    continue;
                if (c >= 0)
                {
                    if (top < LBVH_STACK)
                        stack[top++] = c;
                    else
                        cnt->error = DERR_TOO_MANY_CELLS; // the step fails rather than miss a pair
                    continue;
                }
                const int b = T.bodies[-1 - c];
                if (b == a)
                    continue;
                const int j = entryOf[b];
                const unsigned cb = key_cell(keys[j]);
                int part;
                if (cb == ca)
                    part = j > i ? 0 : -1;
                else
                {
                    const int bx = (int)(cb % (unsigned)g.nx);
                    const unsigned t1 = cb / (unsigned)g.nx;
                    const int by = (int)(t1 % (unsigned)g.ny), bz = (int)(t1 / (unsigned)g.ny);
                    const int d = forward_slot(bx - ax, by - ay, bz - az);
                    part = d < 0 ? -1 : d + 1;
                }
                if (part < 0)
                    continue;
                checks++;
                const float3 dp = sub(ac, xyz(B.pos[b]));
                const float r = ar + B.sizeRad[b].w;
                if (dot(dp, dp) > r * r)
                    continue;
                hits++;
                if (linked(F, S, a, b))
                {
                    cons++;
                    continue;
                }
                partCount[part]++;
                if (tuples < LBVH_TUPLES)
                {
                    tupleKey[tuples] = ((unsigned)part << 24) | (unsigned)j;
                    tupleBody[tuples] = b;
                    tuples++;
                }
                else
                    complete = false;
            }
        }
        // the recorded hits in the grid's order: by part, then by grid position
        for (int x = 1; x < tuples; ++x)
        {
            unsigned kx = tupleKey[x];
            int bx = tupleBody[x], y = x - 1;
            while (y >= 0 && tupleKey[y] > kx)
            {
                tupleKey[y + 1] = tupleKey[y];
                tupleBody[y + 1] = tupleBody[y];
                --y;
            }
            tupleKey[y + 1] = kx;
            tupleBody[y + 1] = bx;
        }
        int total = laneCounts[(size_t)i * BP_LANES + 14];
        int x = 0;
        for (int part = 0; part < 14; ++part)
        {
            const int c = partCount[part];
            total += c;
            const bool keep = complete && c <= BP_SLOTS;
            laneCounts[(size_t)i * BP_LANES + part] = c | (keep ? 0 : (int)BP_UNRECORDED);
            for (int f = 0; f < c && x < tuples; ++f, ++x)
                if (keep)
                    recorded[((size_t)i * BP_LANES + part) * BP_SLOTS + f] = tupleBody[x];
        }
        counts[i] = total;
    }
    warp_add(&cnt->pairChecks, checks);
    warp_add(&cnt->sphereHits, hits);
    warp_add(&cnt->constrainedHits, cons);
}

// Large-vs-large pairs of each world (solver.cpp:476-479), tested by the reference serially
// after all grid pairs. Work item = (world's large base, world's large count, i, chunk); the
// items are ordered by world, i, chunk, which reproduces each world's serial i < j order.
// Modes as k_bp_pairs: BP_COUNT counts and records the first LL_SLOTS partners of each
// item, BP_EMIT_RECORDED writes them (searching again only for items that found more).
// A chunk whose bounding box (of every sphere in it, with a relative margin far above FP32
// rounding) is out of reach of body i's sphere holds no hit: its pairs are counted as
// checked, as the reference checks them, without loading them.
constexpr int LL_SLOTS = 8;

// Bounding box of the spheres of each LL_CHUNK-body chunk of every world's large list, at
// the chunk's first global large index, as order-preserving integers (float_order): every
// large body folds its sphere into its chunk's box with atomic min / max. The boxes start at
// (all ones, 0) for the minima and 0 for the maxima; w of the minimum marks a non-finite
// sphere in the chunk (no culling there).
__global__ void k_ll_chunk_init(uint4 *lo, uint4 *hi, int nLarge)
{
    int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l < nLarge)
    {
        lo[l] = make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u);
        hi[l] = make_uint4(0u, 0u, 0u, 0u);
    }
}

__global__ void k_ll_chunk_bounds(DevGrid G, const int *large, const float4 *largeSphere, int nLarge, uint4 *lo,
                                  uint4 *hi)
{
    int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nLarge)
        return;
    const int w = G.bodyWorld[large[l]];
    const int l0 = G.worldLargeStart[w];
    const int c = l0 + (l - l0) / LL_CHUNK * LL_CHUNK;
    const float4 sp = largeSphere[l];
    const float r = sp.w * 1.001f + 1.0e-4f;
    if (!(isfinite(sp.x) && isfinite(sp.y) && isfinite(sp.z) && isfinite(r)))
    {
        atomicOr(&lo[c].w, 1u);
        return;
    }
    atomicMin(&lo[c].x, float_order(sp.x - r));
    atomicMin(&lo[c].y, float_order(sp.y - r));
    atomicMin(&lo[c].z, float_order(sp.z - r));
    atomicMax(&hi[c].x, float_order(sp.x + r));
    atomicMax(&hi[c].y, float_order(sp.y + r));
    atomicMax(&hi[c].z, float_order(sp.z + r));
}

template <int MODE>
__global__ void k_bp_large_large(DevForces F, const int *large, const float4 *largeSphere, const int4 *items,
                                 int nItems, int *counts, const int *offsets, int base, unsigned long long seqBase,
                                 StepCounters *cnt, const StepState *st, const uint4 *chunkLo,
                                 const uint4 *chunkHi, int *recorded, PairSet S = PairSet())
{
    constexpr bool EMIT = MODE != BP_COUNT;
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (EMIT && st)
    {
        if (step_aborted(st))
            return;
        base = st->manBase + st->newBinned;
        seqBase = st->seqBase + (unsigned long long)st->newBinned;
    }
    bool active = w < nItems;
    if (MODE == BP_EMIT_RECORDED && active)
    {
        const int c = counts[w];
        if (c <= LL_SLOTS)
        {
            if (c > 0)
            {
                const int a = large[items[w].x + items[w].z];
                const int out = base + offsets[w];
                for (int f = 0; f < c; ++f)
                {
                    const int m = out + f;
                    F.man.ab[m] = make_int2(a, recorded[(size_t)w * LL_SLOTS + f]);
                    F.man.seq[m] = seqBase + (unsigned long long)(m - base);
                    F.man.n[m] = 0;
                }
            }
            active = false;
        }
    }
    unsigned checks = 0, hits = 0, cons = 0;
    if (active)
    {
        int4 it = items[w];
        int lbase = it.x, nL = it.y, i = it.z, c = it.w;
        int jBeg = max(i + 1, c * LL_CHUNK), jEnd = min(nL, (c + 1) * LL_CHUNK);
        float4 si = largeSphere[lbase + i];
        bool reach = true;
        if (chunkLo && jBeg < jEnd)
        {
            const uint4 lo = chunkLo[lbase + c * LL_CHUNK], hi = chunkHi[lbase + c * LL_CHUNK];
            const float r = si.w * 1.001f + 1.0e-4f;
            const float3 mn = f3(float_unorder(lo.x), float_unorder(lo.y), float_unorder(lo.z));
            const float3 mx = f3(float_unorder(hi.x), float_unorder(hi.y), float_unorder(hi.z));
            const float3 q = f3(fminf(fmaxf(si.x, mn.x), mx.x), fminf(fmaxf(si.y, mn.y), mx.y),
                                fminf(fmaxf(si.z, mn.z), mx.z));
            const float3 d = sub(xyz(si), q);
            reach = lo.w != 0u || !isfinite(si.x) || !isfinite(si.y) || !isfinite(si.z) || !isfinite(r) ||
                    dot(d, d) <= r * r;
        }
        int a = large[lbase + i];
        int found = 0;
        int out = EMIT ? base + offsets[w] : 0;
        if (!reach)
            checks += (unsigned)max(0, jEnd - jBeg);
        for (int j = reach ? jBeg : jEnd; j < jEnd; ++j)
        {
            checks++;
            float4 sj = largeSphere[lbase + j];
            float3 dp = sub(xyz(si), xyz(sj));
            float r = si.w + sj.w;
            if (!(dot(dp, dp) <= r * r))
                continue;
            hits++;
            int b = large[lbase + j];
            if (linked(F, S, a, b))
            {
                cons++;
                continue;
            }
            if (EMIT)
            {
                int m = out + found;
                F.man.ab[m] = make_int2(a, b);
                F.man.seq[m] = seqBase + (unsigned long long)(m - base);
                F.man.n[m] = 0;
            }
            else if (found < LL_SLOTS && recorded)
                recorded[(size_t)w * LL_SLOTS + found] = b;
            found++;
        }
        if (!EMIT)
            counts[w] = found;
    }
    if (!EMIT)
    {
        warp_add(&cnt->pairChecks, checks);
        warp_add(&cnt->sphereHits, hits);
        warp_add(&cnt->constrainedHits, cons);
    }
}

// Pairs a caller injects in place of the broadphase (broadphaseExternalPairs,
// solver.cpp:579-626), classified against the forces that exist before the step: bit 0 the
// bounding spheres overlap (generatePair's test, solver.cpp:165-174; contact entries skip
// it), bit 1 an existing force already links the bodies (Rigid::constrainedTo). The host
// then applies them in list order, where an earlier pair of the list also constrains a
// later one.
__global__ void k_external_classify(DevBodies B, DevForces F, const int2 *pairs, int count, int sphereTest,
                                    unsigned char *flags)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count)
        return;
    int2 p = pairs[k];
    bool hit = true;
    if (sphereTest)
    {
        float3 dp = sub(xyz(B.pos[p.x]), xyz(B.pos[p.y]));
        float r = B.sizeRad[p.x].w + B.sizeRad[p.y].w;
        hit = dot(dp, dp) <= r * r;
    }
    flags[k] = (hit ? 1 : 0) | ((hit && constrained(F, p.x, p.y)) ? 2 : 0);
}

// New manifolds for the injected pairs that the host kept, in its order.
__global__ void k_external_emit(DevManifolds M, const int2 *pairs, int count, int base, unsigned long long seqBase)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count)
        return;
    M.ab[base + k] = pairs[k];
    M.seq[base + k] = seqBase + (unsigned long long)k;
    M.n[base + k] = 0;
}

// All-pairs broadphase (solver.cpp:176-185): thread per body a, pairs (a, b > a) of its world.
// ---------------------------------------------------------------------------
// Sweep and prune (broadphaseSweepAndPrune, solver.cpp:488-577), one sweep per world.
// ---------------------------------------------------------------------------

// Sweep axis of each world: the axis of largest centre variance. The reference sums the
// centres and the squared deviations serially in list order; one block per world stages
// the positions through shared memory and one thread adds them in that order, so the
// float sums (and the chosen axis) are the reference's.
constexpr int SAP_TILE = 256;

__global__ void __launch_bounds__(SAP_TILE) k_sap_axis(DevBodies B, const int *worldStart, int *axisOut)
{
    __shared__ float3 tile[SAP_TILE];
    __shared__ float3 mean;
    const int w = blockIdx.x;
    const int b0 = worldStart[w], b1 = worldStart[w + 1];
    float3 acc = f3(0, 0, 0);
    for (int pass = 0; pass < 2; ++pass)
    {
        if (pass == 1)
        {
            if (threadIdx.x == 0)
                mean = divs(acc, (float)(b1 - b0));
            acc = f3(0, 0, 0);
            __syncthreads();
        }
        for (int base = b0; base < b1; base += SAP_TILE)
        {
            int k = base + (int)threadIdx.x;
            if (k < b1)
            {
                float3 p = xyz(B.pos[k]);
                if (pass == 1)
                {
                    float3 d = sub(p, mean);
                    p = f3(d.x * d.x, d.y * d.y, d.z * d.z);
                }
                tile[threadIdx.x] = p;
            }
            __syncthreads();
            if (threadIdx.x == 0)
            {
                int m = min(SAP_TILE, b1 - base);
                for (int i = 0; i < m; ++i)
                    acc = add(acc, tile[i]);
            }
            __syncthreads();
        }
    }
    if (threadIdx.x == 0)
    {
        int axis = 0;
        if (acc.y > comp(acc, axis))
            axis = 1;
        if (acc.z > comp(acc, axis))
            axis = 2;
        axisOut[w] = axis;
    }
}

// Interval keys: (world, order-preserving bits of min = centre - radius on the world's axis);
// the value is the body. A stable sort of bodies given in list order then orders equal
// minima by body index, as the reference's comparator does.
__global__ void k_sap_keys(DevBodies B, const int *bodyWorld, const int *axis, unsigned long long *keys, int *vals)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B.n)
        return;
    int w = bodyWorld[b];
    float c = comp(xyz(B.pos[b]), axis[w]);
    float lo = c - B.sizeRad[b].w;
    keys[b] = ((unsigned long long)w << 32) | float_order(lo);
    vals[b] = b;
}

// Sweep from sorted interval i over the following intervals of its world until one starts
// past its maximum; bounding-sphere hits become new manifolds (A = interval i's body,
// B = the later one) unless the bodies are already constrained, in sweep order.
template <bool EMIT>
__global__ void k_sap_sweep(DevBodies B, DevForces F, const int *axis, const unsigned long long *keys,
                            const int *vals, int n, int *counts, const int *offsets, int base,
                            unsigned long long seqBase, StepCounters *cnt)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const unsigned world = (unsigned)(keys[i] >> 32);
    const int a = vals[i];
    const int ax = axis[world];
    float3 pa = xyz(B.pos[a]);
    float ra = B.sizeRad[a].w;
    float ahi = comp(pa, ax) + ra;
    int found = 0;
    int out = EMIT ? base + offsets[i] : 0;
    unsigned long long checks = 0, hits = 0, cons = 0;
    for (int j = i + 1; j < n; ++j)
    {
        if ((unsigned)(keys[j] >> 32) != world)
            break;
        int b = vals[j];
        float3 pb = xyz(B.pos[b]);
        float rb = B.sizeRad[b].w;
        if (comp(pb, ax) - rb > ahi)
            break;
        checks++;
        float3 dp = sub(pa, pb);
        float r = ra + rb;
        if (dot(dp, dp) > r * r)
            continue;
        hits++;
        if (constrained(F, a, b))
        {
            cons++;
            continue;
        }
        if (EMIT)
        {
            int m = out + found;
            F.man.ab[m] = make_int2(a, b);
            F.man.seq[m] = seqBase + (unsigned long long)(m - base);
            F.man.n[m] = 0;
        }
        found++;
    }
    if (!EMIT)
    {
        counts[i] = found;
        atomicAdd(&cnt->pairChecks, checks);
        atomicAdd(&cnt->sphereHits, hits);
        atomicAdd(&cnt->constrainedHits, cons);
    }
}

template <bool EMIT>
__global__ void k_bp_all_pairs(DevBodies B, DevForces F, DevGrid G, int n, int *counts, const int *offsets, int base,
                               unsigned long long seqBase, StepCounters *cnt)
{
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n)
        return;
    int wEnd = G.worldStart[G.bodyWorld[a] + 1];
    float3 pa = xyz(B.pos[a]);
    float ra = B.sizeRad[a].w;
    int found = 0;
    int out = EMIT ? base + offsets[a] : 0;
    unsigned long long hits = 0, cons = 0;
    for (int b = a + 1; b < wEnd; ++b)
    {
        float3 dp = sub(pa, xyz(B.pos[b]));
        float r = ra + B.sizeRad[b].w;
        if (!(dot(dp, dp) <= r * r))
            continue;
        hits++;
        if (constrained(F, a, b))
        {
            cons++;
            continue;
        }
        if (EMIT)
        {
            int m = out + found;
            F.man.ab[m] = make_int2(a, b);
            F.man.seq[m] = seqBase + (unsigned long long)(m - base);
            F.man.n[m] = 0;
        }
        found++;
    }
    if (!EMIT)
    {
        counts[a] = found;
        atomicAdd(&cnt->pairChecks, (unsigned long long)(wEnd - 1 - a));
        atomicAdd(&cnt->sphereHits, hits);
        atomicAdd(&cnt->constrainedHits, cons);
    }
}

// ---------------------------------------------------------------------------
// Box-box narrowphase (collide.cpp:60-433, 898-955)
// ---------------------------------------------------------------------------

struct Obb
{
    float3 c;
    float4 q;
    float3 h;
    float3 ax[3];
};

struct NewContact
{
    int key;
    float3 rA, rB;
};

AVBD_DEV Obb make_obb(float3 p, float4 q, float3 size)
{
    Obb o;
    o.c = p;
    o.q = q;
    o.h = mul(size, 0.5f);
    o.ax[0] = rotate(q, f3(1.0f, 0.0f, 0.0f));
    o.ax[1] = rotate(q, f3(0.0f, 1.0f, 0.0f));
    o.ax[2] = rotate(q, f3(0.0f, 0.0f, 1.0f));
    return o;
}

AVBD_DEV float absdot(float3 a, float3 b) { return fabsf(dot(a, b)); }

AVBD_DEV float3 support_point(const Obb &o, float3 d)
{
    float sx = dot(d, o.ax[0]) >= 0.0f ? 1.0f : -1.0f;
    float sy = dot(d, o.ax[1]) >= 0.0f ? 1.0f : -1.0f;
    float sz = dot(d, o.ax[2]) >= 0.0f ? 1.0f : -1.0f;
    return add(add(add(o.c, mul(o.ax[0], o.h.x * sx)), mul(o.ax[1], o.h.y * sy)), mul(o.ax[2], o.h.z * sz));
}

AVBD_DEV void face_axes(const Obb &o, int ax, float3 &u, float3 &v, float &eu, float &ev)
{
    if (ax == 0)
    {
        u = o.ax[1];
        v = o.ax[2];
        eu = o.h.y;
        ev = o.h.z;
    }
    else if (ax == 1)
    {
        u = o.ax[0];
        v = o.ax[2];
        eu = o.h.x;
        ev = o.h.z;
    }
    else
    {
        u = o.ax[0];
        v = o.ax[1];
        eu = o.h.x;
        ev = o.h.y;
    }
}

// Sutherland-Hodgman step against one side plane (collide.cpp:159-195)
AVBD_DEV int clip_plane(const float3 *in, int cnt, float3 pn, float off, float3 *out)
{
    if (cnt <= 0)
        return 0;
    int k = 0;
    float3 a = in[cnt - 1];
    float da = dot(pn, a) - off;
    for (int i = 0; i < cnt; ++i)
    {
        float3 b = in[i];
        float db = dot(pn, b) - off;
        bool ain = da <= 1.0e-5f;
        bool bin = db <= 1.0e-5f;
        if (ain != bin)
        {
            float t = 0.0f;
            float denom = da - db;
            if (fabsf(denom) > 1.0e-6f)
                t = rclamp(da / denom, 0.0f, 1.0f);
            if (k < 16)
                out[k++] = add(a, mul(sub(b, a), t));
        }
        if (bin && k < 16)
            out[k++] = b;
        a = b;
        da = db;
    }
    return k;
}

// addContact (collide.cpp:197-222): merge by midpoint distance, store body-local offsets
AVBD_DEV void add_contact(float3 pA, float4 qA, float3 pB, float4 qB, NewContact *cs, int &count, float3 *mids,
                          float3 xA, float3 xB, int key)
{
    float3 mid = mul(add(xA, xB), 0.5f);
    for (int i = 0; i < count; ++i)
        if (lensq(sub(mid, mids[i])) < 1.0e-6f)
            return;
    if (count >= 8)
        return;
    cs[count].key = key;
    cs[count].rA = rotate(qconj(qA), sub(xA, pA));
    cs[count].rB = rotate(qconj(qB), sub(xB, pB));
    mids[count] = mid;
    count++;
}

struct SatBest
{
    int type, ia, ib;
    float sep;
    float3 n;
    bool valid;
};

AVBD_DEV bool test_axis(const Obb &A, const Obb &B, float3 delta, float3 axis, int type, int ia, int ib, SatBest &best)
{
    float lenSq = lensq(axis);
    if (lenSq < 1.0e-6f)
        return true;
    float invLen = 1.0f / sqrtf(lenSq);
    float3 n = mul(axis, invLen);
    if (dot(n, delta) < 0.0f)
        n = neg(n);
    float distance = fabsf(dot(delta, n));
    float rA = A.h.x * absdot(n, A.ax[0]) + A.h.y * absdot(n, A.ax[1]) + A.h.z * absdot(n, A.ax[2]);
    float rB = B.h.x * absdot(n, B.ax[0]) + B.h.y * absdot(n, B.ax[1]) + B.h.z * absdot(n, B.ax[2]);
    float sep = distance - (rA + rB);
    if (sep > 0.0f)
        return false;
    if (!best.valid || sep > best.sep)
    {
        best.valid = true;
        best.type = type;
        best.ia = ia;
        best.ib = ib;
        best.sep = sep;
        best.n = n;
    }
    return true;
}

AVBD_DEV void support_edge(const Obb &o, int ax, float3 d, float3 &ea, float3 &eb)
{
    int a1 = (ax + 1) % 3, a2 = (ax + 2) % 3;
    float s1 = dot(d, o.ax[a1]) >= 0.0f ? 1.0f : -1.0f;
    float s2 = dot(d, o.ax[a2]) >= 0.0f ? 1.0f : -1.0f;
    float3 ec = add(add(o.c, mul(o.ax[a1], comp(o.h, a1) * s1)), mul(o.ax[a2], comp(o.h, a2) * s2));
    ea = sub(ec, mul(o.ax[ax], comp(o.h, ax)));
    eb = add(ec, mul(o.ax[ax], comp(o.h, ax)));
}

AVBD_DEV void closest_segments(float3 p0, float3 p1, float3 q0, float3 q1, float3 &c0, float3 &c1)
{
    float3 d1 = sub(p1, p0), d2 = sub(q1, q0), r = sub(p0, q0);
    float a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
    float s = 0.0f, t = 0.0f;
    if (a <= 1.0e-6f && e <= 1.0e-6f)
    {
        c0 = p0;
        c1 = q0;
        return;
    }
    if (a <= 1.0e-6f)
        t = rclamp(f / e, 0.0f, 1.0f);
    else
    {
        float c = dot(d1, r);
        if (e <= 1.0e-6f)
            s = rclamp(-c / a, 0.0f, 1.0f);
        else
        {
            float b = dot(d1, d2);
            float denom = a * e - b * b;
            if (fabsf(denom) > 1.0e-6f)
                s = rclamp((b * f - c * e) / denom, 0.0f, 1.0f);
            t = (b * s + f) / e;
            if (t < 0.0f)
            {
                t = 0.0f;
                s = rclamp(-c / a, 0.0f, 1.0f);
            }
            else if (t > 1.0f)
            {
                t = 1.0f;
                s = rclamp((b - c) / a, 0.0f, 1.0f);
            }
        }
    }
    c0 = add(p0, mul(d1, s));
    c1 = add(q0, mul(d2, t));
}

// Reference face clipped against the incident face (collide.cpp:337-405)
AVBD_DEV int face_manifold(const Obb &A, const Obb &B, bool refIsA, int refAxis, float3 nAB, NewContact *cs)
{
    const Obb &R = refIsA ? A : B;
    const Obb &I = refIsA ? B : A;
    float3 outward = refIsA ? nAB : neg(nAB);
    float sgn = dot(outward, R.ax[refAxis]) >= 0.0f ? 1.0f : -1.0f;
    float3 rn = mul(R.ax[refAxis], sgn);
    float3 rc = add(R.c, mul(rn, comp(R.h, refAxis)));
    float3 ru, rv;
    float reu, rev;
    face_axes(R, refAxis, ru, rv, reu, rev);

    int incAxis = 0;
    float best = -3.402823466e+38f;
    for (int i = 0; i < 3; ++i)
    {
        float d = absdot(I.ax[i], rn);
        if (d > best)
        {
            best = d;
            incAxis = i;
        }
    }
    float3 c0[16], c1[16];
    {
        float s = dot(I.ax[incAxis], rn) > 0.0f ? -1.0f : 1.0f;
        float3 fn = mul(I.ax[incAxis], s);
        float3 fc = add(I.c, mul(fn, comp(I.h, incAxis)));
        float3 u, v;
        float eu, ev;
        face_axes(I, incAxis, u, v, eu, ev);
        c0[0] = add(add(fc, mul(u, eu)), mul(v, ev));
        c0[1] = add(sub(fc, mul(u, eu)), mul(v, ev));
        c0[2] = sub(sub(fc, mul(u, eu)), mul(v, ev));
        c0[3] = sub(add(fc, mul(u, eu)), mul(v, ev));
    }
    int cnt = 4;
    float3 n0 = ru;
    cnt = clip_plane(c0, cnt, n0, dot(n0, rc) + reu, c1);
    if (!cnt)
        return 0;
    float3 n1 = neg(ru);
    cnt = clip_plane(c1, cnt, n1, dot(n1, rc) + reu, c0);
    if (!cnt)
        return 0;
    float3 n2 = rv;
    cnt = clip_plane(c0, cnt, n2, dot(n2, rc) + rev, c1);
    if (!cnt)
        return 0;
    float3 n3 = neg(rv);
    cnt = clip_plane(c1, cnt, n3, dot(n3, rc) + rev, c0);
    if (!cnt)
        return 0;

    int count = 0;
    float3 mids[8];
    int prefix = (refIsA ? 0 : 1) << 24;
    prefix |= (refAxis & 0xFF) << 16;
    prefix |= (incAxis & 0xFF) << 8;
    for (int i = 0; i < cnt && count < 8; ++i)
    {
        float3 p = c0[i];
        float dist = dot(sub(p, rc), rn);
        if (dist > 1.0e-5f)
            continue;
        float3 pr = sub(p, mul(rn, dist));
        add_contact(A.c, A.q, B.c, B.q, cs, count, mids, refIsA ? pr : p, refIsA ? p : pr, prefix | (i & 0xFF));
    }
    if (!count)
        add_contact(A.c, A.q, B.c, B.q, cs, count, mids, support_point(A, nAB), support_point(B, neg(nAB)), prefix);
    return count;
}

// Edge-edge contact (collide.cpp:407-433)
AVBD_DEV int edge_contact(const Obb &A, const Obb &B, int axA, int axB, float3 nAB, NewContact *cs)
{
    float3 a0, a1, b0, b1, xA, xB;
    support_edge(A, axA, nAB, a0, a1);
    support_edge(B, axB, neg(nAB), b0, b1);
    closest_segments(a0, a1, b0, b1, xA, xB);
    int count = 0;
    float3 mids[8];
    int key = (2 << 24) | ((axA & 0xFF) << 8) | (axB & 0xFF);
    add_contact(A.c, A.q, B.c, B.q, cs, count, mids, xA, xB, key);
    if (!count)
        add_contact(A.c, A.q, B.c, B.q, cs, count, mids, support_point(A, nAB), support_point(B, neg(nAB)), key);
    return count;
}

// collideBoxes (collide.cpp:898-955): 15-axis SAT with early out, edge preference, clipping
AVBD_DEV int collide_boxes(float3 pA, float4 qA, float3 sA, float3 pB, float4 qB, float3 sB, NewContact *cs,
                           M3 &basis)
{
    Obb A = make_obb(pA, qA, sA), B = make_obb(pB, qB, sB);
    float3 delta = sub(B.c, A.c);
    SatBest face, edge;
    face.valid = false;
    face.sep = -3.402823466e+38f;
    face.type = face.ia = face.ib = 0;
    face.n = f3(0, 0, 0);
    edge = face;
    for (int i = 0; i < 3; ++i)
        if (!test_axis(A, B, delta, A.ax[i], 0, i, -1, face))
            return 0;
    for (int i = 0; i < 3; ++i)
        if (!test_axis(A, B, delta, B.ax[i], 1, -1, i, face))
            return 0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            if (!test_axis(A, B, delta, cross(A.ax[i], B.ax[j]), 2, i, j, edge))
                return 0;
    if (!face.valid)
        return 0;
    SatBest best = face;
    if (edge.valid && 0.95f * edge.sep > face.sep + 0.01f)
        best = edge;
    basis = orthonormal(neg(best.n));
    if (best.type == 2)
        return edge_contact(A, B, best.ia, best.ib, best.n, cs);
    if (best.type == 0)
        return face_manifold(A, B, true, best.ia, best.n, cs);
    return face_manifold(A, B, false, best.ib, best.n, cs);
}

// ---------------------------------------------------------------------------
// Force initialisation
// ---------------------------------------------------------------------------

struct ContactRec
{
    float3 rA, rB, C0, pen, lam;
    int key;
    bool stick;
};

// Loads of state that other blocks of one persistent launch write between its grid
// barriers (poses, pose differences, contact and joint multipliers and penalties) go to L2
// (ld.global.cg) there, so no block reads a stale L1 line after a barrier. Kernels that
// end before the state changes again use plain loads.
template <bool COH>
AVBD_DEV float4 ld_state(const float4 *p)
{
    if constexpr (COH)
        return __ldcg(p);
    else
        return *p;
}

template <bool COH = false>
AVBD_DEV ContactRec load_contact(const float4 *c)
{
    float4 k0 = c[0], k1 = c[1], k2 = ld_state<COH>(c + 2), k3 = ld_state<COH>(c + 3);
    ContactRec r;
    r.rA = f3(k0.x, k0.y, k0.z);
    r.rB = f3(k0.w, k1.x, k1.y);
    r.C0 = f3(k1.z, k1.w, k2.x);
    r.pen = f3(k2.y, k2.z, k2.w);
    r.lam = f3(k3.x, k3.y, k3.z);
    unsigned bits = __float_as_uint(k3.w);
    r.key = (int)(bits & 0x7FFFFFFFu);
    r.stick = (bits >> 31) != 0;
    return r;
}

AVBD_DEV void store_contact(float4 *c, const ContactRec &r)
{
    c[0] = make_float4(r.rA.x, r.rA.y, r.rA.z, r.rB.x);
    c[1] = make_float4(r.rB.y, r.rB.z, r.C0.x, r.C0.y);
    c[2] = make_float4(r.C0.z, r.pen.x, r.pen.y, r.pen.z);
    c[3] = make_float4(r.lam.x, r.lam.y, r.lam.z, __uint_as_float((unsigned)r.key | (r.stick ? 0x80000000u : 0u)));
}

AVBD_DEV M3 load_basis(const float4 *b) { return rows(xyz(b[0]), xyz(b[1]), xyz(b[2])); }

#include "avbd_round.cuh"

// Contacts a caller injects for one step (ExternalManifoldContact, solver.h:336-344): ordered
// body-pair keys (a << 32 | b, ascending; the last entry given for a key wins, as the
// reference's map assignment does) with each entry's contacts in the manifold layout.
struct ExternalContacts
{
    int count = 0;
    const unsigned long long *keys = nullptr;
    const int *entry = nullptr;
    const int *num = nullptr;       // per entry, at most 8 used
    const float4 *basis = nullptr;  // 3 per entry
    const float4 *contact = nullptr; // 32 per entry
};

AVBD_DEV int ext_find(const ExternalContacts &E, unsigned long long key)
{
    int lo = 0, hi = E.count;
    while (lo < hi)
    {
        int mid = (lo + hi) >> 1;
        if (E.keys[mid] < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo < E.count && E.keys[lo] == key ? E.entry[lo] : -1;
}

// Solver::findExternalManifoldContact (solver.cpp:975-985): (A, B) first, then (B, A).
AVBD_DEV int ext_lookup(const ExternalContacts &E, int a, int b)
{
    int e = ext_find(E, ((unsigned long long)(unsigned)a << 32) | (unsigned)b);
    return e >= 0 ? e : ext_find(E, ((unsigned long long)(unsigned)b << 32) | (unsigned)a);
}

// Manifold::initialize (manifold.cpp:100-174): collide at q- (or take the contacts injected
// for the pair, manifold.cpp:110-117, whole records: their penalty, multipliers and stick
// state seed the new contacts), keep warm-start data of contacts whose feature key
// persists, C0, lambda/penalty decay.
// Ranges with a device step state: INIT_ALL the step's manifolds [0, nManBp); INIT_OLD the
// ones that existed before the step [0, nMan), which need nothing from this step's
// broadphase; INIT_NEW its new pairs [nMan, nManBp). With an output buffer O other than M
// the whole updated record (bodies and sequence number included) goes to O and M is only
// read, so that a step stopped later leaves M as it was.
enum ManifoldInitRange
{
    INIT_ALL = 0,
    INIT_OLD = 1,
    INIT_NEW = 2
};

template <bool ROUND>
__global__ void k_manifold_init(DevBodies B, DevManifolds M, int count, Params P, unsigned char *keep,
                                const StepState *st = nullptr, ExternalContacts E = ExternalContacts(),
                                int *orphanFlag = nullptr, DevManifolds O = DevManifolds(), int range = INIT_ALL)
{
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (st)
    {
        if (step_aborted(st))
            return;
        count = range == INIT_OLD ? st->nMan : st->nManBp;
        if (range == INIT_NEW)
            m += st->nMan;
    }
    if (m >= count)
        return;
    const bool moved = O.ab != nullptr && O.ab != M.ab;
    if (!moved)
        O = M;
    int2 ab = M.ab[m];
    if (moved)
    {
        O.ab[m] = ab;
        O.seq[m] = M.seq[m];
    }
    NpBody A = np_body(B, ab.x), Bb = np_body(B, ab.y);
    float3 pA = A.p, pB = Bb.p;
    float4 qA = A.q, qB = Bb.q;
    float friction = sqrtf(B.friction[ab.x] * B.friction[ab.y]);
    if (ROUND && (A.s.type == SHAPE_SPHERE || Bb.s.type == SHAPE_SPHERE))
        friction = 0.0f;
    // round contacts take the new locations every step and restart their tangential rows
    // (manifold.cpp:120-147; cylinders count as round here); ROUND: the world has round bodies
    const bool round = ROUND && (A.s.type != SHAPE_BOX || Bb.s.type != SHAPE_BOX);
    NewContact nc[8];
    for (int i = 0; i < 8; ++i)
    {
        nc[i].key = 0;
        nc[i].rA = f3(0, 0, 0);
        nc[i].rB = f3(0, 0, 0);
    }
    M3 basis = load_basis(M.basis + 3 * m);
    const int ext = E.count ? ext_lookup(E, ab.x, ab.y) : -1;
    int nn;
    if (ext >= 0)
    {
        basis = load_basis(E.basis + 3 * (size_t)ext);
        nn = min(max(E.num[ext], 0), 8);
    }
    else
        nn = round ? collide_shapes(A, Bb, P.dt, nc, basis) : collide_boxes(pA, qA, A.size, pB, qB, Bb.size, nc, basis);
    int nOld = M.n[m];
    const float4 *cbase = M.contact + (size_t)m * 32;
    float4 *obase = O.contact + (size_t)m * 32;
    ContactRec merged[8];
    for (int i = 0; i < nn; ++i)
    {
        ContactRec r;
        if (ext >= 0)
        {
            r = load_contact(E.contact + 32 * (size_t)ext + 4 * i);
            nc[i].key = r.key;
            nc[i].rA = r.rA;
            nc[i].rB = r.rB;
        }
        else
        {
            r.key = nc[i].key;
            r.rA = nc[i].rA;
            r.rB = nc[i].rB;
            r.C0 = f3(0, 0, 0);
            r.pen = f3(0, 0, 0);
            r.lam = f3(0, 0, 0);
            r.stick = false;
        }
        for (int j = 0; j < nOld; ++j)
        {
            ContactRec o = load_contact(cbase + 4 * j);
            if (o.key == nc[i].key)
            {
                r = o;
                if (round || !o.stick)
                {
                    r.rA = nc[i].rA;
                    r.rB = nc[i].rB;
                }
                if (round)
                {
                    r.lam.y = 0.0f;
                    r.lam.z = 0.0f;
                    r.pen.y = PENALTY_MIN;
                    r.pen.z = PENALTY_MIN;
                    r.stick = false;
                }
                break;
            }
        }
        merged[i] = r;
    }
    for (int i = 0; i < nn; ++i)
    {
        ContactRec &c = merged[i];
        float3 xA = add(pA, contact_offset(A.s, qA, c.rA, basis, true, c.key));
        float3 xB = add(pB, contact_offset(Bb.s, qB, c.rB, basis, false, c.key));
        c.C0 = add(mv(basis, sub(xA, xB)), f3(COLLISION_MARGIN, 0, 0));
        c.lam = mul(mul(c.lam, P.alpha), P.gamma);
        c.pen = clampv(mul(c.pen, P.gamma), PENALTY_MIN, PENALTY_MAX);
        store_contact(obase + 4 * i, c);
    }
    O.n[m] = nn;
    O.basis[3 * m + 0] = f4(basis.r0, friction);
    O.basis[3 * m + 1] = f4(basis.r1, round ? ROUND_FLAG : 0.0f);
    O.basis[3 * m + 2] = f4(basis.r2, 0.0f);
    keep[m] = nn > 0 ? 1 : 0;
    if (nn > 0 && orphanFlag && B.massMoment[ab.x].x <= 0 && B.massMoment[ab.y].x <= 0)
        *orphanFlag = 1;
}

// Joint::initialize (joint.cpp:35-54)
__global__ void k_joint_init(DevBodies B, DevForces F, Params P, unsigned char *keep, const StepState *st = nullptr,
                             int *orphanFlag = nullptr)
{
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= F.nJoint || step_aborted(st))
        return;
    float4 *d = F.joint + 8 * (size_t)j;
    int2 ab = F.jointAB[j];
    float4 d0 = d[0], d1 = d[1], d3 = d[3], d4 = d[4], d5 = d[5], d6 = d[6], d7 = d[7];
    float3 rA = xyz(d0), rB = xyz(d1);
    float stiffLin = d0.w, stiffAng = d1.w, torqueArm = d3.w;
    float3 pB = xyz(B.pos[ab.y]);
    float4 qB = B.quat[ab.y];
    float3 pa = ab.x >= 0 ? xform(xyz(B.pos[ab.x]), B.quat[ab.x], rA) : rA;
    float3 C0Lin = sub(pa, xform(pB, qB, rB));
    float4 qa = ab.x >= 0 ? B.quat[ab.x] : make_float4(0, 0, 0, 1);
    float3 C0Ang = mul(qdiff(qa, qB), torqueArm);
    float3 lamLin = mul(mul(xyz(d6), P.alpha), P.gamma);
    float3 lamAng = mul(mul(xyz(d7), P.alpha), P.gamma);
    float3 penLin = clampv(mul(xyz(d4), P.gamma), PENALTY_MIN, PENALTY_MAX);
    float3 penAng = clampv(mul(xyz(d5), P.gamma), PENALTY_MIN, PENALTY_MAX);
    penLin = minv(penLin, stiffLin);
    penAng = minv(penAng, stiffAng);
    d[2] = f4(C0Lin, d[2].w);
    d[3] = f4(C0Ang, torqueArm);
    d[4] = f4(penLin, d4.w);
    d[5] = f4(penAng, 0.0f);
    d[6] = f4(lamLin, 0.0f);
    d[7] = f4(lamAng, 0.0f);
    keep[j] = d4.w != 0.0f ? 0 : 1;
    if (orphanFlag && (ab.x < 0 || B.massMoment[ab.x].x <= 0) && B.massMoment[ab.y].x <= 0)
        *orphanFlag = 1;
}

// Stable compaction of manifolds into the other buffer. With a device step state the count
// is the state's, and the kernel records the surviving count there (and a swap, with `flip`).
// COMPACT_LANES threads per manifold: the first copies the header and basis, all of them
// the live contacts' float4s.
constexpr int COMPACT_LANES = 8;

// `flip`: dst becomes the live buffer (the state counts the swap); otherwise dst is the
// buffer the step started from and stays the live one.
__global__ void k_manifold_compact(DevManifolds src, DevManifolds dst, int count, const unsigned char *keep,
                                   const int *newIndex, StepState *st = nullptr, bool flip = true)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int m = (int)(t / COMPACT_LANES), lane = (int)(t % COMPACT_LANES);
    if (st)
    {
        if (step_aborted(st))
            return;
        count = st->nManBp;
        if (t == 0)
        {
            st->nMan = count > 0 ? newIndex[count - 1] + (keep[count - 1] ? 1 : 0) : 0;
            if (flip)
                st->flips++;
        }
    }
    if (m >= count || !keep[m])
        return;
    const int d = newIndex[m];
    const int n = src.n[m];
    if (lane == 0)
    {
        dst.ab[d] = src.ab[m];
        dst.seq[d] = src.seq[m];
        dst.n[d] = n;
    }
    if (lane < 3)
        dst.basis[3 * d + lane] = src.basis[3 * m + lane];
    const float4 *s = src.contact + (size_t)m * 32;
    float4 *o = dst.contact + (size_t)d * 32;
    for (int k = lane; k < 4 * n; k += COMPACT_LANES)
        o[k] = s[k];
}

__global__ void k_joint_compact(int count, const unsigned char *keep, const int *newIndex, const int2 *abS,
                                const unsigned long long *seqS, const float4 *dS, int2 *abD,
                                unsigned long long *seqD, float4 *dD)
{
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= count || !keep[j])
        return;
    int d = newIndex[j];
    abD[d] = abS[j];
    seqD[d] = seqS[j];
    for (int k = 0; k < 8; ++k)
        dD[8 * (size_t)d + k] = dS[8 * (size_t)j + k];
}

// Joint edits between steps. Each device joint looks its sequence number up in the sorted
// edit list; a match records the joint index per edit (bodies must agree) and, for a
// removal, clears the joint's keep flag. matched[0] counts the matches.
__global__ void k_joint_match(int count, const unsigned long long *seq, const int2 *ab, int edits,
                              const unsigned long long *editSeq, const int2 *editAB, int *editJoint,
                              unsigned char *keep, int *matched)
{
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= count)
        return;
    unsigned long long s = seq[j];
    int lo = 0, hi = edits;
    while (lo < hi)
    {
        int mid = (lo + hi) >> 1;
        if (editSeq[mid] < s)
            lo = mid + 1;
        else
            hi = mid;
    }
    bool hit = lo < edits && editSeq[lo] == s;
    if (hit && editAB)
        hit = editAB[lo].x == ab[j].x && editAB[lo].y == ab[j].y;
    if (keep)
        keep[j] = hit ? 0 : 1;
    if (hit)
    {
        if (editJoint)
            editJoint[lo] = j;
        atomicAdd(matched, 1);
    }
}

__global__ void k_joint_write(int edits, const int *editJoint, const float4 *editData, float4 *joint, int count)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 8 * edits)
        return;
    int e = t >> 3, k = t & 7, j = editJoint[e];
    if (j >= 0 && j < count) // -1: the edit matched no joint
        joint[8 * (size_t)j + k] = editData[t];
}

// ---------------------------------------------------------------------------
// Adjacency (per-body force lists, newest first)
// ---------------------------------------------------------------------------

constexpr int KEY_SEQ_BITS = 40; // sequence numbers stay below 2^40
constexpr unsigned long long KEY_SEQ_MASK = (1ull << KEY_SEQ_BITS) - 1ull;
constexpr unsigned long long KEY_NO_BODY = 0xFFFFFFull; // body counts stay below this

// Incidence key: body, then newest force first. `shift` is the bit width of the sequence
// counter (every sequence number is below 2^shift), so the key spans shift + bits(n) bits
// and the sort passes only over those; the world side of an anchored joint takes body n,
// after every real body.
AVBD_DEV unsigned long long incidence_key(int body, unsigned long long seq, int shift, int n)
{
    unsigned long long b = body >= 0 ? (unsigned long long)body : (unsigned long long)n;
    unsigned long long cap = (1ull << shift) - 1ull;
    return (b << shift) | (cap - (seq & cap));
}

// Two incidences per force: manifolds [0, 2M), joints [2M, 2M+2J), springs, ignores. With a
// device step state M is the state's and the launch covers the buffers' capacity: slots
// past the live incidences get keys of all ones, which sort after every body.
__global__ void k_incidences(DevForces F, int shift, int n, unsigned long long *keys, unsigned *vals,
                             const StepState *st = nullptr, int capacity = 0)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    // A stopped step writes nothing from here on: the counts it would read are not the live
    // ones (its new manifolds were never committed).
    if (step_aborted(st))
        return;
    if (st)
        F.nMan = st->nMan;
    int total = 2 * (F.nMan + F.nJoint + F.nSpring + F.nIgnore);
    if (st && t >= total && t < capacity)
    {
        keys[t] = ~0ull;
        vals[t] = ADJ_NONE;
        return;
    }
    if (t >= total)
        return;
    int f = t >> 1;
    unsigned isA = (t & 1) ? 0u : 1u;
    int2 ab;
    unsigned long long seq;
    unsigned type;
    if (f < F.nMan)
    {
        ab = F.man.ab[f];
        seq = F.man.seq[f];
        type = ADJ_MANIFOLD;
    }
    else if ((f -= F.nMan) < F.nJoint)
    {
        ab = F.jointAB[f];
        seq = F.jointSeq[f];
        type = ADJ_JOINT;
    }
    else if ((f -= F.nJoint) < F.nSpring)
    {
        ab = F.springAB[f];
        seq = F.springSeq[f];
        type = ADJ_SPRING;
    }
    else
    {
        f -= F.nSpring;
        ab = F.ignoreAB[f];
        seq = F.ignoreSeq[f];
        type = ADJ_IGNORE;
    }
    keys[t] = incidence_key(isA ? ab.x : ab.y, seq, shift, n);
    vals[t] = make_adj(type, isA, (unsigned)f);
}

// Number of entries of an ascending sequence list above s.
AVBD_DEV int count_above(const unsigned long long *seq, int count, unsigned long long s)
{
    int lo = 0, hi = count;
    while (lo < hi)
    {
        int mid = (lo + hi) >> 1;
        if (seq[mid] <= s)
            lo = mid + 1;
        else
            hi = mid;
    }
    return count - lo;
}

// Incidences written in the global newest-first order of their forces, when each force
// list (manifolds, joints, springs, ignore pairs) is stored in ascending sequence order: a
// force's place is the number of forces with a larger sequence number, found by binary
// search in the other lists. A stable sort by body alone then gives every body's force list
// newest first. Keys are the body (n for the world side of an anchored joint); with a device
// step state the launch covers the capacity and unused slots get keys of all ones.
__global__ void k_incidences_ranked(DevForces F, int n, unsigned *keys, unsigned *vals, const StepState *st = nullptr,
                                    int capacityForces = 0)
{
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (step_aborted(st))
        return;
    if (st)
        F.nMan = st->nMan;
    const int total = F.nMan + F.nJoint + F.nSpring + F.nIgnore;
    if (f >= total)
    {
        if (st && f < capacityForces)
        {
            keys[2 * f] = keys[2 * f + 1] = 0xFFFFFFFFu;
            vals[2 * f] = vals[2 * f + 1] = ADJ_NONE;
        }
        return;
    }
    int2 ab;
    unsigned type;
    int idx = f;
    unsigned long long s;
    int rank;
    if (idx < F.nMan)
    {
        ab = F.man.ab[idx];
        s = F.man.seq[idx];
        type = ADJ_MANIFOLD;
        rank = F.nMan - 1 - idx + count_above(F.jointSeq, F.nJoint, s) + count_above(F.springSeq, F.nSpring, s) +
               count_above(F.ignoreSeq, F.nIgnore, s);
    }
    else if ((idx -= F.nMan) < F.nJoint)
    {
        ab = F.jointAB[idx];
        s = F.jointSeq[idx];
        type = ADJ_JOINT;
        rank = F.nJoint - 1 - idx + count_above(F.man.seq, F.nMan, s) + count_above(F.springSeq, F.nSpring, s) +
               count_above(F.ignoreSeq, F.nIgnore, s);
    }
    else if ((idx -= F.nJoint) < F.nSpring)
    {
        ab = F.springAB[idx];
        s = F.springSeq[idx];
        type = ADJ_SPRING;
        rank = F.nSpring - 1 - idx + count_above(F.man.seq, F.nMan, s) + count_above(F.jointSeq, F.nJoint, s) +
               count_above(F.ignoreSeq, F.nIgnore, s);
    }
    else
    {
        idx -= F.nSpring;
        ab = F.ignoreAB[idx];
        s = F.ignoreSeq[idx];
        type = ADJ_IGNORE;
        rank = F.nIgnore - 1 - idx + count_above(F.man.seq, F.nMan, s) + count_above(F.jointSeq, F.nJoint, s) +
               count_above(F.springSeq, F.nSpring, s);
    }
    keys[2 * rank] = ab.x >= 0 ? (unsigned)ab.x : (unsigned)n;
    vals[2 * rank] = make_adj(type, 1u, (unsigned)idx);
    keys[2 * rank + 1] = (unsigned)ab.y;
    vals[2 * rank + 1] = make_adj(type, 0u, (unsigned)idx);
}

// Segment starts of a sorted key array whose top bits are the segment id (0..n-1, or
// larger for "no segment"); start[s] for s in [0, n] with gaps filled.
template <class Key>
__global__ void k_segment_starts(const Key *keys, int total, int shift, int n, int *start,
                                 const StepState *st = nullptr)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= total || step_aborted(st))
        return;
    long long cur = (long long)(keys[k] >> shift);
    if (cur > n)
        cur = n;
    long long prev = -1;
    if (k > 0)
    {
        prev = (long long)(keys[k - 1] >> shift);
        if (prev > n)
            prev = n;
    }
    for (long long s = prev + 1; s <= cur; ++s)
        start[s] = k;
    if (k == total - 1)
        for (long long s = cur + 1; s <= n; ++s)
            start[s] = total;
}

__global__ void k_copy_adj(const unsigned *vals, unsigned *adj, int total, const StepState *st = nullptr)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < total && !step_aborted(st))
        adj[k] = vals[k];
}

// ---------------------------------------------------------------------------
// Step admission (device-resident steps): nothing of the world has changed yet, so a step
// that cannot run as issued stops here and the host redoes it.
// ---------------------------------------------------------------------------

AVBD_DEV bool finite4(float4 v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z) && isfinite(v.w); }

// Every body's pose and velocities must be finite (the reference propagates NaN silently;
// this step refuses it before touching anything); a joint broken in an earlier step must
// first leave the joint list (Joint::initialize returns false, solver.cpp:1085-1132), which
// the host's compaction does. With a step state the kernel stops the step; `seen` (either
// path) collects STEP_SEEN_* bits for the host.
constexpr int STEP_SEEN_NONFINITE = 1, STEP_SEEN_BROKEN_JOINT = 2;

__global__ void k_step_begin(DevBodies B, const float4 *joint, int nJoint, StepState *st, int *seen)
{
    if (step_aborted(st))
        return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    bool bad = false, broke = false;
    if (t < B.n)
        bad = !finite4(B.pos[t]) || !finite4(B.quat[t]) || !finite4(B.vel[t]) || !finite4(B.angvel[t]);
    if (t < nJoint)
        broke = joint[8 * (size_t)t + 4].w != 0.0f;
    const bool lead = (threadIdx.x & 31) == 0;
    if (__any_sync(0xFFFFFFFFu, bad) && lead)
    {
        if (st)
            step_abort(st, ABORT_NONFINITE);
        if (seen)
            atomicOr(seen, STEP_SEEN_NONFINITE);
    }
    if (__any_sync(0xFFFFFFFFu, broke) && lead)
    {
        if (st)
            step_abort(st, ABORT_JOINTS);
        if (seen)
            atomicOr(seen, STEP_SEEN_BROKEN_JOINT);
    }
}

// ---------------------------------------------------------------------------
// Body warm start (solver.cpp:1134-1169)
// ---------------------------------------------------------------------------

__global__ void k_warm_start(DevBodies B, const int *adjStart, Params P, const StepState *st = nullptr)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B.n || step_aborted(st))
        return;
    float dt = P.dt, g = P.gravity;
    float3 pos = xyz(B.pos[b]);
    float4 q = B.quat[b];
    float3 vel = xyz(B.vel[b]);
    float3 w = xyz(B.angvel[b]);
    float3 pv = xyz(B.prevVel[b]);
    float mass = B.massMoment[b].x;
    float3 inertLin = add(pos, mul(vel, dt));
    if (mass > 0)
        inertLin = add(inertLin, mul(f3(0, 0, g), dt * dt));
    float4 inertAng = qstep(q, mul(w, dt));
    float3 accel = divs(sub(vel, pv), dt);
    float accelExt = accel.z * rsign(g);
    float accelWeight = rclamp(accelExt / fabsf(g), 0.0f, 1.0f);
    if (!isfinite(accelWeight))
        accelWeight = 0.0f;
    const float3 pos0 = pos;
    const float4 q0 = q;
    B.initLin[b] = f4(pos, 0.0f);
    B.initAng[b] = q;
    if (mass > 0)
    {
        pos = add(add(pos, mul(vel, dt)), mul(f3(0, 0, g), accelWeight * dt * dt));
        q = qstep(q, mul(w, dt));
    }
    if (mass > 0 && adjStart[b + 1] == adjStart[b])
    {
        pos = inertLin;
        q = inertAng;
    }
    B.pos[b] = f4(pos, 0.0f);
    B.quat[b] = q;
    B.inertLin[b] = f4(inertLin, 0.0f);
    B.inertAng[b] = inertAng;
    B.initAngInv[b] = qinverse(q0);
    B.inertAngInv[b] = qinverse(inertAng);
    B.dqLin[b] = f4(sub(pos, pos0), 0.0f);
    B.dqAng[b] = f4(qdiff(q, q0), 0.0f);
}

// finishStep velocities (solver.cpp:1275-1287); rolling friction is sphere-only
__global__ void k_finish(DevBodies B, Params P, const StepState *st = nullptr)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B.n || step_aborted(st))
        return;
    float4 v = B.vel[b];
    B.prevVel[b] = v;
    if (B.massMoment[b].x > 0)
    {
        B.vel[b] = f4(divs(sub(xyz(B.pos[b]), xyz(B.initLin[b])), P.dt), 0.0f);
        B.angvel[b] = f4(divs(qdiff(B.quat[b], B.initAng[b]), P.dt), 0.0f);
    }
}

// ---------------------------------------------------------------------------
// Jones-Plassmann colouring of the dynamic-body constraint graph. In round r an
// uncoloured vertex whose (priority, index) beats every uncoloured neighbour takes the
// smallest colour unused by neighbours coloured in earlier rounds. The result depends
// only on the graph, so the CPU oracle reproduces it exactly.
// state: -2 not a vertex, -1 uncoloured, else round << 16 | colour
// ---------------------------------------------------------------------------

// All Jones-Plassmann rounds in one cooperative launch. Priority mode 0: lower list index
// first, which reproduces the sequential greedy colouring in list order; mode 1: hashed.
__global__ void k_colour_all(DevBodies B, DevForces F, int n, int mode, int *state, ColourControl *ctl,
                             StepCounters *cnt, unsigned spinLimit, const StepState *st)
{
    if (step_aborted(st)) // uniform: every block leaves before the first barrier
        return;
    const int stride = gridDim.x * blockDim.x;
    int mine = 0;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < n; b += stride)
    {
        bool vertex = B.massMoment[b].x > 0 && F.adjStart[b + 1] > F.adjStart[b];
        __stcg(&state[b], vertex ? -1 : -2);
        mine += vertex ? 1 : 0;
    }
    int bs = block_sum(mine);
    if (threadIdx.x == 0 && bs)
        atomicAdd(&ctl->vertices, bs);
    unsigned target = 0;
    if (!grid_barrier(ctl, target, spinLimit))
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
            for (int k = F.adjStart[v]; k < F.adjStart[v + 1]; ++k)
            {
                unsigned e = F.adj[k];
                if (adj_type(e) == ADJ_IGNORE)
                    continue;
                int2 ab = force_bodies(F, e);
                int u = ab.x == v ? ab.y : ab.x;
                if (u < 0)
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
                cnt->error = DERR_TOO_MANY_COLOURS;
                c = 255;
            }
            __stcg(&state[v], (round << 16) | c);
            atomicMax(&ctl->maxColour, c);
            mine++;
        }
        bs = block_sum(mine);
        if (threadIdx.x == 0 && bs)
            atomicAdd(&ctl->coloured[round], bs);
        if (!grid_barrier(ctl, target, spinLimit))
            return;
        done += ((volatile int *)ctl->coloured)[round];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
    {
        ctl->rounds = round;
        if (done < total)
            ctl->error = 2;
    }
}

// Solve-list keys: colour in the top 8 bits, body index (< 2^24) below; non-vertices last.
__global__ void k_colour_keys(const int *state, int n, int *colour, unsigned *keys)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n)
        return;
    int s = state[b];
    int c = s >= 0 ? (s & 0xFFFF) : -1;
    colour[b] = c;
    keys[b] = c >= 0 ? (((unsigned)c << 24) | (unsigned)b) : 0xFFFFFFFFu;
}

// ---------------------------------------------------------------------------
// Primal: one group of G lanes per body of the current colour (solver.cpp:1177-1242).
// Each lane evaluates one constraint row (a manifold contact, a joint part or a spring)
// into its 27-entry contribution; lanes that own an entry then add the rows in the
// body's force order (newest force first, contacts in manifold order), so every sum has
// the reference's order and the result is bit-identical. One lane factors the 6x6 LDL.
// ---------------------------------------------------------------------------

constexpr unsigned KIND_NONE = 0u;
constexpr unsigned KIND_FULL = (1u << 27) - 1u;
constexpr unsigned KIND_LHSANG = 0x3Fu << 6;
constexpr unsigned KIND_ANG = (0x3Fu << 6) | (0x7u << 24);

struct Pose
{
    float3 p, ip;
    float4 q, iq;
};

// What a contact row reads of a body: its orientation and its pose difference from the
// step start, dLin = p - p0 and dAng = qdiff(q, q0) (manifold.cpp:185-188). The differences
// are stored with the pose (k_warm_start, k_primal) instead of being recomputed by every row;
// they are the same functions of the same floats, so every row sees the same bits.
struct Motion
{
    float4 q;
    float3 dLin, dAng;
};

AVBD_DEV Motion motion_of(const Pose &s)
{
    Motion m;
    m.q = s.q;
    m.dLin = sub(s.p, s.ip);
    m.dAng = qdiff(s.q, s.iq);
    return m;
}

template <bool COH = false>
AVBD_DEV Motion load_motion(const DevBodies &B, int b)
{
    Motion m;
    m.q = ld_state<COH>(B.quat + b);
    m.dLin = xyz(ld_state<COH>(B.dqLin + b));
    m.dAng = xyz(ld_state<COH>(B.dqAng + b));
    return m;
}

// a * diag(k): column j of a scaled by k[j]. The reference forms this product with full
// row-by-column dots (jLinT * K, jAngT * K in manifold.cpp:218-221 and joint.cpp:89-95); the
// two products with K's zero entries add +-0, which leaves every nonzero entry unchanged
// and can only change the sign of an exact zero. These matrices feed only the left-hand
// side, whose accumulators start at +0 or a positive mass term and so never hold -0: the
// sums, and the step, are bit-identical.
AVBD_DEV M3 times_diag(const M3 &a, float3 k)
{
    return rows(f3(a.r0.x * k.x, a.r0.y * k.y, a.r0.z * k.z), f3(a.r1.x * k.x, a.r1.y * k.y, a.r1.z * k.z),
                f3(a.r2.x * k.x, a.r2.y * k.y, a.r2.z * k.z));
}

AVBD_DEV void store_terms(float *t, const M3 &LL, const M3 &LA, const M3 &LC, float3 RL, float3 RA)
{
    t[E_LL00] = LL.r0.x;
    t[E_LL10] = LL.r1.x;
    t[E_LL11] = LL.r1.y;
    t[E_LL20] = LL.r2.x;
    t[E_LL21] = LL.r2.y;
    t[E_LL22] = LL.r2.z;
    t[E_LA00] = LA.r0.x;
    t[E_LA10] = LA.r1.x;
    t[E_LA11] = LA.r1.y;
    t[E_LA20] = LA.r2.x;
    t[E_LA21] = LA.r2.y;
    t[E_LA22] = LA.r2.z;
    t[E_LC00] = LC.r0.x;
    t[E_LC01] = LC.r0.y;
    t[E_LC02] = LC.r0.z;
    t[E_LC10] = LC.r1.x;
    t[E_LC11] = LC.r1.y;
    t[E_LC12] = LC.r1.z;
    t[E_LC20] = LC.r2.x;
    t[E_LC21] = LC.r2.y;
    t[E_LC22] = LC.r2.z;
    t[E_RL0] = RL.x;
    t[E_RL1] = RL.y;
    t[E_RL2] = RL.z;
    t[E_RA0] = RA.x;
    t[E_RA1] = RA.y;
    t[E_RA2] = RA.z;
}

// Contact row: C, F with normal clamp and friction cone (manifold.cpp:183-212)
struct ContactEval
{
    M3 jALin, jBLin, jAAng, jBAng;
    float3 C, F;
    float fs, bounds;
};

// F from C with the contact's penalty and multiplier: normal clamp and friction cone
// (manifold.cpp:199-212).
AVBD_DEV void contact_force(ContactEval &e, const ContactRec &c, float friction)
{
    M3 K = diag(c.pen.x, c.pen.y, c.pen.z);
    float3 F = add(mv(K, e.C), c.lam);
    F.x = rmin(F.x, 0.0f);
    e.bounds = fabsf(F.x) * friction;
    e.fs = sqrtf(F.y * F.y + F.z * F.z);
    if (e.fs > e.bounds && e.fs > 0)
    {
        F.y *= e.bounds / e.fs;
        F.z *= e.bounds / e.fs;
    }
    e.F = F;
}

// Manifold::updateDual for one contact (manifold.cpp:231-280), on the evaluation at the
// current poses: lambda takes F, the penalties ramp, the stick flag follows.
AVBD_DEV void contact_dual(ContactRec &c, const ContactEval &e, float betaLin)
{
    c.lam = e.F;
    if (e.F.x < 0)
        c.pen.x = rmin(c.pen.x + betaLin * fabsf(e.C.x), PENALTY_MAX);
    if (e.fs <= e.bounds)
    {
        c.pen.y = rmin(c.pen.y + betaLin * fabsf(e.C.y), PENALTY_MAX);
        c.pen.z = rmin(c.pen.z + betaLin * fabsf(e.C.z), PENALTY_MAX);
        c.stick = sqrtf(e.C.y * e.C.y + e.C.z * e.C.z) < STICK_THRESH;
    }
}

AVBD_DEV void store_contact_state(float4 *cp, const ContactRec &c)
{
    cp[2] = make_float4(c.C0.z, c.pen.x, c.pen.y, c.pen.z);
    cp[3] = make_float4(c.lam.x, c.lam.y, c.lam.z, __uint_as_float((unsigned)c.key | (c.stick ? 0x80000000u : 0u)));
}

// The same two words into a taped step's record of contact slot `slot` (lp: one iteration's
// slice of the adjoint's multiplier and penalty tape, two float4s per slot; null: no tape).
AVBD_DEV void tape_contact_state(float4 *lp, long long slot, const ContactRec &c)
{
    if (!lp)
        return;
    lp[2 * slot] = make_float4(c.C0.z, c.pen.x, c.pen.y, c.pen.z);
    lp[2 * slot + 1] =
        make_float4(c.lam.x, c.lam.y, c.lam.z, __uint_as_float((unsigned)c.key | (c.stick ? 0x80000000u : 0u)));
}

// rAW, rBW: the contact's world offsets from the two bodies' centres (rotate(q, r) for boxes,
// contactOffsetWorld for round bodies).
AVBD_DEV ContactEval eval_contact_arms(const Motion &A, const Motion &Bp, const M3 &basis, float friction,
                                       const ContactRec &c, float alpha, float3 rAW, float3 rBW)
{
    ContactEval e;
    const float3 &dqALin = A.dLin;
    const float3 &dqAAng = A.dAng;
    const float3 &dqBLin = Bp.dLin;
    const float3 &dqBAng = Bp.dAng;
    e.jALin = basis;
    e.jBLin = mneg(basis);
    e.jAAng = rows(cross(rAW, e.jALin.r0), cross(rAW, e.jALin.r1), cross(rAW, e.jALin.r2));
    e.jBAng = rows(cross(rBW, e.jBLin.r0), cross(rBW, e.jBLin.r1), cross(rBW, e.jBLin.r2));
    e.C = add(add(add(add(mul(c.C0, 1.0f - alpha), mv(e.jALin, dqALin)), mv(e.jBLin, dqBLin)), mv(e.jAAng, dqAAng)),
              mv(e.jBAng, dqBAng));
    contact_force(e, c, friction);
    return e;
}

AVBD_DEV ContactEval eval_contact(const Motion &A, const Motion &Bp, const M3 &basis, float friction,
                                  const ContactRec &c, float alpha)
{
    return eval_contact_arms(A, Bp, basis, friction, c, alpha, rotate(A.q, c.rA), rotate(Bp.q, c.rB));
}

AVBD_DEV ContactEval eval_contact(const Pose &A, const Pose &Bp, const M3 &basis, float friction,
                                  const ContactRec &c, float alpha)
{
    return eval_contact(motion_of(A), motion_of(Bp), basis, friction, c, alpha);
}

AVBD_DEV M3 gs_ball_socket(int k, float3 v)
{
    float vk = comp(v, k);
    float3 r0 = f3(-vk, 0, 0), r1 = f3(0, -vk, 0), r2 = f3(0, 0, -vk);
    if (k == 0)
    {
        r0.x += v.x;
        r1.x += v.y;
        r2.x += v.z;
    }
    else if (k == 1)
    {
        r0.y += v.x;
        r1.y += v.y;
        r2.y += v.z;
    }
    else
    {
        r0.z += v.x;
        r1.z += v.y;
        r2.z += v.z;
    }
    return rows(r0, r1, r2);
}

// Joint rows (joint.cpp:56-123): part 0 = linear stamp, 1 = diagonalised geometric
// stiffness added to lhsAng, 2 = angular stamp.
template <bool COH = false>
AVBD_DEV unsigned joint_term(const DevBodies &B, const DevForces &F, unsigned j, int part, bool isA, float alpha,
                             float *t)
{
    const float4 *d = F.joint + 8 * (size_t)j;
    int2 ab = F.jointAB[j];
    float4 d0 = d[0], d1 = d[1];
    float3 pB = xyz(ld_state<COH>(B.pos + ab.y));
    float4 qB = ld_state<COH>(B.quat + ab.y);
    const M3 I = rows(f3(1, 0, 0), f3(0, 1, 0), f3(0, 0, 1));
    const M3 NI = rows(f3(-1, 0, 0), f3(0, -1, 0), f3(0, 0, -1));
    if (part < 2)
    {
        float3 rA = xyz(d0), rB = xyz(d1);
        float3 penLin = xyz(ld_state<COH>(d + 4));
        float3 rAW = ab.x >= 0 ? rotate(ld_state<COH>(B.quat + ab.x), rA) : f3(0, 0, 0);
        float3 rBW = rotate(qB, rB);
        M3 K = diag(penLin.x, penLin.y, penLin.z);
        float3 C = sub(ab.x >= 0 ? add(xyz(ld_state<COH>(B.pos + ab.x)), rAW) : rA, add(pB, rBW));
        if (isinf(d0.w))
            C = sub(C, mul(xyz(d[2]), alpha));
        float3 Fv = add(mv(K, C), xyz(ld_state<COH>(d + 6)));
        if (part == 0)
        {
            M3 jLin = isA ? I : NI;
            M3 jAng = isA ? skew(neg(rAW)) : skew(rBW);
            M3 jLinT = trans(jLin), jAngT = trans(jAng);
            M3 jAngTk = times_diag(jAngT, penLin);
            store_terms(t, mm(times_diag(jLinT, penLin), jLin), mm(jAngTk, jAng), mm(jAngTk, jLin), mv(jLinT, Fv),
                        mv(jAngT, Fv));
            return KIND_FULL;
        }
        float3 r = isA ? rAW : neg(rBW);
        M3 H = madd(madd(mscale(gs_ball_socket(0, r), Fv.x), mscale(gs_ball_socket(1, r), Fv.y)),
                    mscale(gs_ball_socket(2, r), Fv.z));
        M3 D = diagonalize(H);
        t[E_LA00] = D.r0.x;
        t[E_LA10] = D.r1.x;
        t[E_LA11] = D.r1.y;
        t[E_LA20] = D.r2.x;
        t[E_LA21] = D.r2.y;
        t[E_LA22] = D.r2.z;
        return KIND_LHSANG;
    }
    float3 penAng = xyz(ld_state<COH>(d + 5));
    float torqueArm = d[3].w;
    M3 K = diag(penAng.x, penAng.y, penAng.z);
    float4 qa = ab.x >= 0 ? ld_state<COH>(B.quat + ab.x) : make_float4(0, 0, 0, 1);
    float3 C = mul(qdiff(qa, qB), torqueArm);
    if (isinf(d1.w))
        C = sub(C, mul(xyz(d[3]), alpha));
    float3 Fv = add(mv(K, C), xyz(ld_state<COH>(d + 7)));
    M3 jAng = mscale(isA ? I : NI, torqueArm);
    M3 LA = mm(mm(trans(jAng), K), jAng);
    float3 RA = mv(trans(jAng), Fv);
    t[E_LA00] = LA.r0.x;
    t[E_LA10] = LA.r1.x;
    t[E_LA11] = LA.r1.y;
    t[E_LA20] = LA.r2.x;
    t[E_LA21] = LA.r2.y;
    t[E_LA22] = LA.r2.z;
    t[E_RA0] = RA.x;
    t[E_RA1] = RA.y;
    t[E_RA2] = RA.z;
    return KIND_ANG;
}

// Spring row (spring.cpp:27-69)
template <bool COH = false>
AVBD_DEV unsigned spring_term(const DevBodies &B, const DevForces &F, unsigned s, bool isA, float *t)
{
    const float4 *d = F.spring + 2 * (size_t)s;
    int2 ab = F.springAB[s];
    float4 d0 = d[0], d1 = d[1];
    float3 rA = xyz(d0), rB = xyz(d1);
    float rest = d0.w, stiffness = d1.w;
    float4 qA = ld_state<COH>(B.quat + ab.x), qB = ld_state<COH>(B.quat + ab.y);
    float3 pA = xform(xyz(ld_state<COH>(B.pos + ab.x)), qA, rA);
    float3 pB = xform(xyz(ld_state<COH>(B.pos + ab.y)), qB, rB);
    float3 dd = sub(pA, pB);
    float dLen = len(dd);
    if (dLen <= 1.0e-6f)
        return KIND_NONE;
    float3 n = divs(dd, dLen);
    float C = dLen - rest;
    float f = stiffness * C;
    float3 jLin, jAng;
    if (isA)
    {
        float3 rW = rotate(qA, rA);
        jLin = n;
        jAng = cross(rW, n);
    }
    else
    {
        float3 rW = rotate(qB, rB);
        jLin = neg(n);
        jAng = neg(cross(rW, n));
    }
    store_terms(t, mscale(outer(jLin, jLin), stiffness), mscale(outer(jAng, jAng), stiffness),
                mscale(outer(jAng, jLin), stiffness), mul(jLin, f), mul(jAng, f));
    return KIND_FULL;
}

// Rows a force can stamp during one step, in the order the primal adds them: the contacts
// of a manifold (fixed once Manifold::initialize ran), a joint's linear stamp, its
// geometric stiffness and its angular stamp (each present while its penalty is nonzero,
// joint.cpp:60, 103), a spring. Listed once per step; joint parts that are off (a
// fractured joint, a zero stiffness) stamp nothing, exactly as if they were not listed.
AVBD_DEV int rows_listed(const DevForces &F, unsigned e)
{
    switch (adj_type(e))
    {
    case ADJ_MANIFOLD:
        return F.man.n[adj_index(e)];
    case ADJ_JOINT:
        return 3;
    case ADJ_SPRING:
        return 1;
    default:
        return 0;
    }
}

// Row list, built in parallel over the force-list entries (sorted incidence keys carry the
// body): entry k contributes rows_listed rows unless its body is static (never solved).
// Incidences without a body (the world side of an anchored joint) sort after the last body
// and contribute none.
template <class Key>
__global__ void k_entry_rows(DevForces F, DevBodies B, const Key *sortedKeys, int total, int shift,
                             int *count, const StepState *st = nullptr)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k > total || step_aborted(st))
        return;
    int r = 0;
    if (k < total)
    {
        unsigned long long b = sortedKeys[k] >> shift;
        if (b < (unsigned long long)B.n && B.massMoment[b].x > 0)
            r = rows_listed(F, F.adj[k]);
    }
    count[k] = r; // count[total] = 0, so the exclusive scan ends with the row total
}

__global__ void k_row_starts(const int *adjStart, const int *entryRow, int n, int *rowStart,
                             const StepState *st = nullptr)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b <= n && !step_aborted(st))
        rowStart[b] = entryRow[adjStart[b]];
}

// The other body of a force-list entry (-1: the world side of an anchored joint).
AVBD_DEV int entry_partner(const DevForces &F, unsigned e)
{
    unsigned i = adj_index(e);
    bool isA = adj_isA(e) != 0;
    int2 ab = make_int2(-1, -1);
    switch (adj_type(e))
    {
    case ADJ_MANIFOLD:
        ab = F.man.ab[i];
        break;
    case ADJ_JOINT:
        ab = F.jointAB[i];
        break;
    case ADJ_SPRING:
        ab = F.springAB[i];
        break;
    default:
        break;
    }
    return isA ? ab.y : ab.x;
}

// Row entries carry the partner body next to the row index (bodies < 2^24, rows < 8), so
// a contact row's partner pose is fetched together with its contact data.
// Bit 30 marks the rows whose contact this body updates in a fused dual pass: the body
// with the lower colour, or the only dynamic one (set after colouring).
constexpr int ROW_OWNS_DUAL = 1 << 30;
// Bit 31: the partner is dynamic with a higher colour (so with ROW_OWNS_DUAL clear, the
// partner is dynamic with a lower colour; with both clear, it is static or absent).
constexpr int ROW_PARTNER_LATER = (int)0x80000000u;
AVBD_DEV int row_sub(int2 row) { return row.y & 7; }
AVBD_DEV int row_partner(int2 row) { return ((row.y & (ROW_OWNS_DUAL - 1)) >> 3) - 1; }

__global__ void k_entry_fill(DevForces F, const int *entryRow, const int *count, int total,
                             const StepState *st = nullptr)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= total || step_aborted(st))
        return;
    int out = entryRow[k];
    unsigned e = F.adj[k];
    int n = count[k];
    if (n == 0)
        return;
    int code = (entry_partner(F, e) + 1) << 3;
    for (int sub = 0; sub < n; ++sub)
        F.rows[out + sub] = make_int2((int)e, code | sub);
}

// Contact row of body `self` against its partner (Manifold::updatePrimal,
// manifold.cpp:183-228); the partner comes from the row entry.
template <bool COH = false, bool ROUND = false>
AVBD_DEV unsigned contact_term_self(const DevBodies &B, const DevForces &F, unsigned m, int ci, bool isA, int self,
                                    int partner, bool dual, const Params &P, float *t, float4 *lpTape = nullptr)
{
    const float4 *bs = F.man.basis + 3 * (size_t)m;
    float4 b0 = bs[0], b1 = bs[1];
    M3 basis = rows(xyz(b0), xyz(b1), xyz(bs[2]));
    float4 *cp = F.man.contact + (size_t)m * 32 + 4 * ci;
    ContactRec c = load_contact<COH>(cp);
    const int ia = isA ? self : partner, ib = isA ? partner : self;
    Motion A = load_motion<COH>(B, ia), Bm = load_motion<COH>(B, ib);
    // the contact's world arms (ROUND: the world has round bodies, whose manifolds are
    // flagged in basis row 1)
    const bool round = ROUND && b1.w != 0.0f;
    const float3 rAW = round ? contact_offset(body_shape(B, ia), A.q, c.rA, basis, true, c.key) : rotate(A.q, c.rA);
    const float3 rBW = round ? contact_offset(body_shape(B, ib), Bm.q, c.rB, basis, false, c.key) : rotate(Bm.q, c.rB);
    const float3 rW = isA ? rAW : rBW;
    ContactEval e = eval_contact_arms(A, Bm, basis, b0.w, c, P.alpha, rAW, rBW);
    if (dual)
    {
        // the previous iteration's dual update of this contact, at the same poses, then
        // this row's force from the same C with the updated penalty and multiplier
        contact_dual(c, e, P.betaLin);
        store_contact_state(cp, c);
        tape_contact_state(lpTape, 8ll * m + ci, c);
        contact_force(e, c, b0.w);
    }
    // this body's Jacobian rows, formed again from the basis and its arm as
    // eval_contact_arms forms them (fewer values live across the dual update)
    const M3 jLin = isA ? basis : mneg(basis);
    const M3 jAng = rows(cross(rW, jLin.r0), cross(rW, jLin.r1), cross(rW, jLin.r2));
    M3 jLinT = trans(jLin), jAngT = trans(jAng);
    M3 jAngTk = times_diag(jAngT, c.pen);
    store_terms(t, mm(times_diag(jLinT, c.pen), jLin), mm(jAngTk, jAng), mm(jAngTk, jLin), mv(jLinT, e.F),
                mv(jAngT, e.F));
    return KIND_FULL;
}

// One listed row's contribution (Manifold/Joint/Spring::updatePrimal).
// `fusedDual`: this launch also performs the previous iteration's contact dual updates,
// each by the row of the body that owns it.
template <bool COH = false, bool ROUND = false>
AVBD_DEV unsigned listed_row_term(const DevBodies &B, const DevForces &F, int2 row, int self, bool fusedDual,
                                  const Params &P, float *t, float4 *lpTape = nullptr)
{
    unsigned e = (unsigned)row.x;
    unsigned i = adj_index(e);
    bool isA = adj_isA(e) != 0;
    int sub = row_sub(row);
    switch (adj_type(e))
    {
    case ADJ_MANIFOLD:
        return contact_term_self<COH, ROUND>(B, F, i, sub, isA, self, row_partner(row),
                                      fusedDual && (row.y & ROW_OWNS_DUAL) != 0, P, t, lpTape);
    case ADJ_JOINT:
    {
        const float4 *d = F.joint + 8 * (size_t)i;
        bool on = sub < 2 ? lensq(xyz(ld_state<COH>(d + 4))) > 0 : lensq(xyz(ld_state<COH>(d + 5))) > 0;
        return on ? joint_term<COH>(B, F, i, sub, isA, P.alpha, t) : KIND_NONE;
    }
    case ADJ_SPRING:
        return spring_term<COH>(B, F, i, isA, t);
    default:
        return KIND_NONE;
    }
}

// Initial system M/dt^2 (solver.cpp:1189-1198) as 27 entries
template <bool COH = false>
AVBD_DEV void initial_system(const DevBodies &B, int b, float dt, float *t)
{
    float4 mm4 = B.massMoment[b];
    float dt2 = dt * dt;
    // diag(m) / dt2 entry by entry, as the reference divides the whole matrix: the
    // diagonal divided, the off-diagonal zeros' quotient 0 / dt2 formed once
    const float z = zero_over(dt2), ml = fdiv(mm4.x, dt2);
    M3 lhsLin = rows(f3(ml, z, z), f3(z, ml, z), f3(z, z, ml));
    M3 lhsAng = rows(f3(fdiv(mm4.y, dt2), z, z), f3(z, fdiv(mm4.z, dt2), z), f3(z, z, fdiv(mm4.w, dt2)));
    M3 lhsCross = diag(0, 0, 0);
    float3 rhsLin = mv(lhsLin, sub(xyz(ld_state<COH>(B.pos + b)), xyz(B.inertLin[b])));
    float3 rhsAng = mv(lhsAng, qdiff_inv(ld_state<COH>(B.quat + b), B.inertAngInv[b]));
    store_terms(t, lhsLin, lhsAng, lhsCross, rhsLin, rhsAng);
}

// Shared memory of one primal batch: GPB bodies, G lanes each.
template <int G, int BLOCK>
struct PrimalShared
{
    static constexpr int GPB = BLOCK / G;
    float term[GPB][G][E_COUNT];
    float sys[GPB][E_COUNT]; // odd stride: one system per thread without bank conflicts
    float4 start[4][GPB];    // position, orientation, step-start position, inverse step-start orientation
    unsigned kind[GPB][G];
    int body[GPB];
};

// Barrier of one SUB-thread unit of the block (SUB = BLOCK: the whole block). Units use
// named barriers 1..BLOCK/SUB, so they never wait for each other.
template <int SUB, int BLOCK>
AVBD_DEV void unit_sync()
{
    static_assert(BLOCK % SUB == 0 && SUB % 32 == 0 && BLOCK / SUB <= 15, "barrier units");
    if constexpr (SUB == BLOCK)
        __syncthreads();
    else
        asm volatile("bar.sync %0, %1;" ::"r"(1 + (int)threadIdx.x / SUB), "n"(SUB) : "memory");
}

// Per-body progress of the iteration kernel when it runs without per-colour grid barriers:
// done[b] = the iterations body b has completed in this launch. `done` null: the
// barriers order the passes and nothing is waited for.
struct IterFlow
{
    int *done = nullptr;
    int it = 0;
    int *error = nullptr;
    unsigned spinLimit = 1u << 22; // polls before a partner wait gives up
    // a taped step (the adjoint's forward): slice k of each tape holds the state after
    // iteration k - 1 (slice 0 the state before the first); null: no tape
    float4 *poseTape = nullptr; // per slice: n positions, then n orientations
    float4 *lpTape = nullptr;   // per slice: two float4s per contact slot (8 per manifold)
    int tapeN = 0, tapeM = 0;
    AVBD_DEV float4 *lp_slice(int k) const { return lpTape ? lpTape + (size_t)k * 16 * tapeM : nullptr; }
};

AVBD_DEV int ld_acquire(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

AVBD_DEV void st_release(int *p, int v)
{
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

constexpr unsigned FLOW_SPIN_LIMIT = 1u << 22; // default poll limit of a partner wait

// A row reads its partner's pose (and, for a contact the partner owns, the contact's
// multipliers) as the colour-ordered sweep leaves them: a partner of an earlier colour
// must have finished this iteration, one of a later colour the previous iteration (so
// that it has read this body's previous pose, and made its own contact updates). Static
// partners never move. On expiry the wait records an error and gives up.
AVBD_DEV void wait_partner(const IterFlow &flow, int2 row)
{
    const int need = (row.y & ROW_OWNS_DUAL) == 0 ? flow.it + 1 : ((row.y & ROW_PARTNER_LATER) ? flow.it : 0);
    if (need == 0)
        return;
    const int *d = flow.done + row_partner(row);
    unsigned spins = 0;
    while (ld_acquire(d) < need)
    {
        if (++spins >= flow.spinLimit)
        {
            atomicExch(flow.error, 1);
            return;
        }
        if (spins > 64)
        {
            if (*(volatile int *)flow.error) // another wait expired: the launch is failing
                return;
            __nanosleep(64);
        }
    }
}

// `start`: the body's position, orientation, step-start position and the inverse of the
// step-start orientation, staged in shared memory by the gathering lanes, so that no
// register holds them across the factorisation.
template <bool COH, int GPB>
AVBD_DEV void solve_and_move(const DevBodies &B, int b, const float *sys, const float4 (*start)[GPB], int t,
                             const IterFlow &flow)
{
    float3 dxl, dxa;
    ldl_solve27(sys, dxl, dxa);
    const float4 p0 = start[0][t], q0 = start[1][t], i0 = start[2][t], a0inv = start[3][t];
    float3 p = add(xyz(p0), dxl);
    float4 q = qstep(q0, dxa);
    B.pos[b] = f4(p, 0.0f);
    B.quat[b] = q;
    B.dqLin[b] = f4(sub(p, xyz(i0)), 0.0f);
    B.dqAng[b] = f4(qdiff_inv(q, a0inv), 0.0f);
    if (flow.poseTape)
    {
        float4 *pt = flow.poseTape + (size_t)(flow.it + 1) * 2 * flow.tapeN;
        pt[b] = f4(p, 0.0f);
        pt[flow.tapeN + b] = q;
    }
    if (flow.done) // a release: the body's pose, and the contact updates its rows made before
        st_release(flow.done + b, flow.it + 1); // the block's barrier, are visible before the count
}

template <bool COH>
AVBD_DEV void dual_joint(const DevBodies &B, const DevForces &F, int j, const Params &P);
template <bool COH, bool ROUND>
AVBD_DEV void dual_contact_slot(const DevBodies &B, const DevManifolds &M, long long t, const Params &P,
                                float4 *lpTape = nullptr);

// One primal solve per body of a batch of one colour (solver.cpp:1186-1233). Rows: G lanes
// per body. The solve entries carry the body and its row range; every lane of a group
// builds the initial system M/dt^2 and keeps the entries it owns, then the rows are
// evaluated G at a time (lane j evaluates row base + j into shared memory) and every lane
// adds its entries row by row, so each sum keeps the reference's order. Solve: the batch's
// accumulated systems go to shared memory and one thread per body factors its 6x6 system
// and moves the body, so the factorisation runs with every lane of its warp busy. The
// block works in independent units of SUB threads (SUB / G bodies, which the unit's first
// SUB / G threads factorise); every thread of the block calls this (it holds the units'
// barriers).
template <int G, int BLOCK, int SUB, bool COH, bool ROUND>
AVBD_DEV void primal_batch(const DevBodies &B, const DevForces &F, const Params &P, const int4 *entries, int count,
                           bool fusedDual, PrimalShared<G, BLOCK> &sh, const IterFlow &flow = IterFlow{},
                           bool lastDual = false)
{
    static_assert(BLOCK % G == 0 && 32 % G == 0, "group size");
    constexpr int OWN = (E_COUNT + G - 1) / G;
    const int g = threadIdx.x / G;
    const int lane = threadIdx.x % G;
    if (g < count)
    {
        const unsigned gmask = (G == 32) ? 0xFFFFFFFFu : (((1u << G) - 1u) << ((threadIdx.x & 31) / G * G));
        const int4 ent = entries[g];
        const int b = ent.x, r0 = ent.y, r1 = ent.z;
        for (int j = lane; j < 4; j += G) // stage the solve's poses while the rows are gathered
            sh.start[j][g] = j == 0   ? ld_state<COH>(B.pos + b)
                             : j == 1 ? ld_state<COH>(B.quat + b)
                             : j == 2 ? B.initLin[b]
                                      : B.initAngInv[b];

        // Joints' dual updates of the previous iteration (Joint::updateDual, fracture
        // included), made by the body that owns them before any of its rows reads them, as
        // the contact rows do for their contacts: the lower colour (or the only dynamic body)
        // owns the joint, its partner has finished the previous iteration and neither has
        // moved in this one, so the poses are the ones the reference's dual sweep reads.
        if (fusedDual && F.nJoint > 0)
        {
            for (int r = r0 + lane; r < r1; r += G)
            {
                const int2 row = F.rows[r];
                const unsigned e = (unsigned)row.x;
                if (adj_type(e) == ADJ_JOINT && row_sub(row) == 0 && (row.y & ROW_OWNS_DUAL) != 0)
                {
                    if (flow.done)
                        wait_partner(flow, row);
                    dual_joint<COH>(B, F, (int)adj_index(e), P);
                }
            }
            __syncwarp(gmask);
        }
        float acc[OWN];
        {
            float t0[E_COUNT];
            initial_system<COH>(B, b, P.dt, t0);
#pragma unroll
            for (int k = 0; k < OWN; ++k) // acc[k] = t0[lane + k G], with constant indices only
            {
                float v = 0.0f;
#pragma unroll
                for (int j = 0; j < G; ++j)
                    if (j + k * G < E_COUNT && lane == j)
                        v = t0[j + k * G];
                acc[k] = v;
            }
        }

        for (int base = r0; base < r1; base += G)
        {
            int r = base + lane;
            if (r < r1)
            {
                const int2 row = F.rows[r];
                if (flow.done)
                    wait_partner(flow, row);
                sh.kind[g][lane] =
                    listed_row_term<COH, ROUND>(B, F, row, b, fusedDual, P, sh.term[g][lane], flow.lp_slice(flow.it));
            }
            __syncwarp(gmask);
            int nrows = min(G, r1 - base);
            for (int rr = 0; rr < nrows; ++rr)
            {
                unsigned kind = sh.kind[g][rr];
                if (kind == KIND_FULL)
                {
#pragma unroll
                    for (int kk = 0; kk < OWN; ++kk)
                    {
                        int e = lane + kk * G;
                        if (e < E_COUNT)
                            acc[kk] = acc[kk] + sh.term[g][rr][e];
                    }
                }
                else
                {
#pragma unroll
                    for (int kk = 0; kk < OWN; ++kk)
                    {
                        int e = lane + kk * G;
                        if (e < E_COUNT && ((kind >> e) & 1u))
                            acc[kk] = acc[kk] + sh.term[g][rr][e];
                    }
                }
            }
            __syncwarp(gmask);
        }
#pragma unroll
        for (int k = 0; k < OWN; ++k)
        {
            int e = lane + k * G;
            if (e < E_COUNT)
                sh.sys[g][e] = acc[k];
        }
        if (lane == 0)
            sh.body[g] = b;
    }
    unit_sync<SUB, BLOCK>();
    const int lt = threadIdx.x % SUB;
    const int t = (threadIdx.x / SUB) * (SUB / G) + lt; // the unit's body this thread factorises
    if (lt < SUB / G && t < count)
        solve_and_move<COH, BLOCK / G>(B, sh.body[t], sh.sys[t], sh.start, t, flow);
    if (lastDual)
    {
        // Last iteration: the body that moves last in each of its contacts and joints (the
        // later colour, or the only dynamic body) makes that force's final dual update right
        // after its solve, on both bodies' final poses (its earlier partners finished before
        // its rows were read), which the closing pass would otherwise do.
        unit_sync<SUB, BLOCK>();
        if (g < count)
        {
            const int4 ent = entries[g];
            for (int r = ent.y + lane; r < ent.z; r += G)
            {
                const int2 row = F.rows[r];
                if (row.y & ROW_PARTNER_LATER)
                    continue;
                const unsigned e = (unsigned)row.x;
                if (adj_type(e) == ADJ_MANIFOLD)
                    dual_contact_slot<COH, ROUND>(B, F.man, 8ll * adj_index(e) + row_sub(row), P,
                                                  flow.lp_slice(flow.it + 1));
                else if (adj_type(e) == ADJ_JOINT && row_sub(row) == 0)
                    dual_joint<COH>(B, F, (int)adj_index(e), P);
            }
        }
    }
}

// One launch per colour: block k takes the colour's bodies [k GPB, (k+1) GPB).
template <int G, int BLOCK, int MINB, bool ROUND = false>
__global__ void __launch_bounds__(BLOCK, MINB) k_primal(DevBodies B, DevForces F, Params P, const int4 *entries,
                                                        int first, int count)
{
    __shared__ PrimalShared<G, BLOCK> sh;
    constexpr int GPB = BLOCK / G;
    const int base = blockIdx.x * GPB;
    primal_batch<G, BLOCK, BLOCK, false, ROUND>(B, F, P, entries + first + base, min(GPB, count - base), false, sh);
}

// ---------------------------------------------------------------------------
// Dual (solver.cpp:1244-1271)
// ---------------------------------------------------------------------------

// Manifold::updateDual per contact slot (manifold.cpp:231-280); t = manifold * 8 + slot.
template <bool COH, bool ROUND>
AVBD_DEV void dual_contact_slot(const DevBodies &B, const DevManifolds &M, long long t, const Params &P,
                                float4 *lpTape)
{
    int m = (int)(t >> 3), ci = (int)(t & 7);
    if (ci >= M.n[m])
        return;
    int2 ab = M.ab[m];
    Motion A = load_motion<COH>(B, ab.x), Bp = load_motion<COH>(B, ab.y);
    const float4 *bs = M.basis + 3 * (size_t)m;
    float4 b0 = bs[0], b1 = bs[1];
    M3 basis = rows(xyz(b0), xyz(b1), xyz(bs[2]));
    float4 *cp = M.contact + (size_t)m * 32 + 4 * ci;
    ContactRec c = load_contact<COH>(cp);
    ContactEval e = ROUND && b1.w != 0.0f
                        ? eval_contact_arms(A, Bp, basis, b0.w, c, P.alpha,
                                            contact_offset(body_shape(B, ab.x), A.q, c.rA, basis, true, c.key),
                                            contact_offset(body_shape(B, ab.y), Bp.q, c.rB, basis, false, c.key))
                        : eval_contact(A, Bp, basis, b0.w, c, P.alpha);
    contact_dual(c, e, P.betaLin);
    store_contact_state(cp, c);
    tape_contact_state(lpTape, t, c);
}

template <bool ROUND = false>
__global__ void k_dual_contacts(DevBodies B, DevManifolds M, int nMan, Params P)
{
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < 8ll * nMan)
        dual_contact_slot<false, ROUND>(B, M, t, P);
}

// Joint::updateDual with fracture (joint.cpp:125-182)
template <bool COH>
AVBD_DEV void dual_joint(const DevBodies &B, const DevForces &F, int j, const Params &P)
{
    float4 *d = F.joint + 8 * (size_t)j;
    int2 ab = F.jointAB[j];
    float4 d0 = d[0], d1 = d[1];
    float4 d4 = ld_state<COH>(d + 4);
    float3 penLin = xyz(d4), penAng = xyz(ld_state<COH>(d + 5));
    float3 lamLin = xyz(ld_state<COH>(d + 6)), lamAng = xyz(ld_state<COH>(d + 7));
    float brokenFlag = d4.w;
    float3 pB = xyz(ld_state<COH>(B.pos + ab.y));
    float4 qB = ld_state<COH>(B.quat + ab.y);
    if (lensq(penLin) > 0)
    {
        M3 K = diag(penLin.x, penLin.y, penLin.z);
        float3 pa = ab.x >= 0 ? xform(xyz(ld_state<COH>(B.pos + ab.x)), ld_state<COH>(B.quat + ab.x), xyz(d0))
                              : xyz(d0);
        float3 C = sub(pa, xform(pB, qB, xyz(d1)));
        if (isinf(d0.w))
        {
            C = sub(C, mul(xyz(d[2]), P.alpha));
            lamLin = add(mv(K, C), lamLin);
        }
        penLin = minv(add(penLin, mul(absv(C), P.betaLin)), rmin(d0.w, PENALTY_MAX));
    }
    if (lensq(penAng) > 0)
    {
        M3 K = diag(penAng.x, penAng.y, penAng.z);
        float4 qa = ab.x >= 0 ? ld_state<COH>(B.quat + ab.x) : make_float4(0, 0, 0, 1);
        float3 C = mul(qdiff(qa, qB), d[3].w);
        if (isinf(d1.w))
        {
            C = sub(C, mul(xyz(d[3]), P.alpha));
            lamAng = add(mv(K, C), lamAng);
        }
        penAng = minv(add(penAng, mul(absv(C), P.betaAng)), rmin(d1.w, PENALTY_MAX));
    }
    float fracture = d[2].w;
    if (lensq(lamAng) > fracture * fracture)
    {
        penLin = f3(0, 0, 0);
        penAng = f3(0, 0, 0);
        lamLin = f3(0, 0, 0);
        lamAng = f3(0, 0, 0);
        brokenFlag = 1.0f;
    }
    d[4] = f4(penLin, brokenFlag);
    d[5] = f4(penAng, 0.0f);
    d[6] = f4(lamLin, 0.0f);
    d[7] = f4(lamAng, 0.0f);
}

__global__ void k_dual_joints(DevBodies B, DevForces F, Params P)
{
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < F.nJoint)
        dual_joint<false>(B, F, j, P);
}

// ---------------------------------------------------------------------------
// All iterations of a step in one cooperative launch
// ---------------------------------------------------------------------------

// Bounded grid-wide barrier of the iteration kernel: on expiry the kernel records an
// error and every block leaves.
constexpr unsigned ITER_SPIN_LIMIT = 1u << 22;

struct IterSync
{
    unsigned arrive; // barrier arrivals so far in this launch
    int error;
    int pad[2];
};

// Arrivals count up through the launch (the counter starts at zero): barrier k of the
// launch releases every block once k x gridDim.x blocks have arrived, so the last block's
// arrival alone opens it.
AVBD_DEV bool iter_barrier(IterSync *s, unsigned &target, unsigned spinLimit = ITER_SPIN_LIMIT)
{
    __shared__ int ok;
    __syncthreads();
    target += gridDim.x;
    if (threadIdx.x == 0)
    {
        __threadfence();
        atomicAdd(&s->arrive, 1u);
        volatile unsigned *arrive = &s->arrive;
        unsigned spins = 0;
        while (*arrive < target && ++spins < spinLimit)
            if (spins > 256)
                __nanosleep(32);
        ok = spins < spinLimit;
        if (!ok)
            atomicExch(&s->error, 1);
        __threadfence();
    }
    __syncthreads();
    return ok && ((volatile int *)&s->error)[0] == 0;
}

// Solver::iteratePrimalDualCpu (solver.cpp:1177-1271) for every iteration of a step, one
// block per SM, mutable state read at L2. Per iteration: each colour's bodies in batches of
// at most GPB per block, spread evenly over the blocks; the block works in independent
// units of SUB threads. With joints, a grid barrier follows each colour and the joints'
// dual update each iteration; without, each row waits for its partner's iteration count
// instead (wait_partner), so blocks and units run ahead of one another. The contacts' dual
// update of iteration k is done in iteration k + 1 by the row of the body that owns the
// contact, before that row uses it: the owner is the contact's body with the lower colour
// (or its only dynamic body), which has not moved yet in iteration k + 1, and neither has
// the other body, so both poses are those the dual sweep of iteration k reads and every
// contact's update is the same. After one closing grid barrier, the last iteration's
// contact updates end the launch.
// The adjoint's per-iteration record of a taped step (IterFlow's tape fields).
struct IterTape
{
    float4 *pose = nullptr;
    float4 *lp = nullptr;
    int n = 0, nMan = 0;
};

// TAPE: the instance that fills a taped step's records (the others compile without them).
template <int G, int BLOCK, int SUB, bool ROUND = false, bool TAPE = false>
__global__ void __launch_bounds__(BLOCK, 1) k_iterations(DevBodies B, DevForces F, Params P, const int4 *entries,
                                                         const int *colourStart, int nColours, int iterations,
                                                         IterSync *sync, int *done, unsigned spinLimit,
                                                         const StepState *st, const int *orphanFlag,
                                                         IterTape tape)
{
    if (st)
    {
        if (step_aborted(st)) // uniform: every block leaves before the first barrier
            return;
        nColours = st->nColours;
        F.nMan = st->nMan;
    }
    extern __shared__ __align__(16) unsigned char smemRaw[];
    PrimalShared<G, BLOCK> &sh = *reinterpret_cast<PrimalShared<G, BLOCK> *>(smemRaw);
    constexpr int GPB = BLOCK / G;
    const long long stride = (long long)gridDim.x * BLOCK;
    const long long tid = (long long)blockIdx.x * BLOCK + threadIdx.x;
    unsigned target = 0;
    // rows wait for their partners instead of every colour for the grid; joints' dual
    // updates are fused into their owners' rows like the contacts'; the last iteration's
    // dual updates follow each force's last solve, so only forces without a dynamic body
    // (flagged by the initialisation) need the closing pass
    const bool barriers = done == nullptr;
    const bool orphans = barriers || (orphanFlag && *orphanFlag != 0);
    IterFlow flow;
    flow.done = barriers ? nullptr : done;
    flow.error = &sync->error;
    flow.spinLimit = spinLimit;
    if constexpr (TAPE)
    {
        flow.poseTape = tape.pose;
        flow.lpTape = tape.lp;
        flow.tapeN = tape.n;
        flow.tapeM = tape.nMan;
    }
    for (int it = 0; it < iterations; ++it)
    {
        flow.it = it;
        const bool last = !barriers && it == iterations - 1;
        for (int c = 0; c < nColours; ++c)
        {
            // the colour's bodies in equal contiguous batches over every block, as few
            // rounds of at most GPB bodies per block as the colour needs
            const int first = colourStart[c], cnt = colourStart[c + 1] - first;
            const int rounds = (cnt + gridDim.x * GPB - 1) / (gridDim.x * GPB);
            const int per = rounds > 0 ? (cnt + gridDim.x * rounds - 1) / (gridDim.x * rounds) : 0;
            for (int r = 0; r < rounds; ++r)
            {
                const int base = (r * gridDim.x + blockIdx.x) * per;
                if (base >= cnt)
                    break;
                primal_batch<G, BLOCK, SUB, true, ROUND>(B, F, P, entries + first + base, min(per, cnt - base),
                                                         it > 0, sh, flow, last);
                unit_sync<SUB, BLOCK>(); // the unit's solve threads are done with the shared systems
            }
            if (barriers && !iter_barrier(sync, target, spinLimit))
                return;
        }
        if (barriers && F.nJoint > 0)
        {
            for (long long j = tid; j < F.nJoint; j += stride)
                dual_joint<true>(B, F, (int)j, P);
            if (!iter_barrier(sync, target, spinLimit))
                return;
        }
    }
    if (iterations <= 0 || !orphans)
        return;
    if (!barriers && !iter_barrier(sync, target, spinLimit)) // every body has finished every iteration
        return;
    // Contacts between two static bodies have no owning row: nothing moves them, so their
    // update of every iteration runs here, one after the other on the same poses. (With
    // barriers, every contact's last update runs here.)
    for (long long t = tid; t < 8ll * F.nMan; t += stride)
    {
        if ((int)(t & 7) >= F.man.n[t >> 3]) // an empty slot: nothing to load
            continue;
        int2 ab = F.man.ab[t >> 3];
        bool orphan = B.massMoment[ab.x].x <= 0 && B.massMoment[ab.y].x <= 0;
        if (!orphan && !barriers)
            continue;
        for (int r = orphan ? iterations : 1; r > 0; --r) // update r from the end: iteration iterations - r
            dual_contact_slot<true, ROUND>(B, F.man, t, P, flow.lp_slice(iterations - r + 1));
    }
    // joints without a dynamic body likewise
    if (!barriers)
        for (long long j = tid; j < F.nJoint; j += stride)
        {
            int2 ab = F.jointAB[j];
            bool orphan = (ab.x < 0 || B.massMoment[ab.x].x <= 0) && B.massMoment[ab.y].x <= 0;
            for (int r = orphan ? iterations : 0; r > 0; --r)
                dual_joint<true>(B, F, (int)j, P);
        }
}

// ---------------------------------------------------------------------------
// Greedy colouring in list order as one dataflow pass (the default colouring mode)
// ---------------------------------------------------------------------------

AVBD_DEV unsigned long long ld_acquire_u64(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

AVBD_DEV void st_release_u64(unsigned long long *p, unsigned long long v)
{
    asm volatile("st.release.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// With list-index priority the Jones-Plassmann rounds colour a vertex once every
// lower-index neighbour has its colour, with the smallest colour none of them uses (the
// sequential greedy colouring in list order, which the oracle restates); its round is one
// more than the largest round among those neighbours. So each vertex simply waits for its
// lower-index neighbours: the smallest uncoloured vertex can always proceed (its thread has
// finished every smaller vertex of its grid-stride sequence and all blocks are resident),
// so the waits cannot cycle; each is bounded and on expiry records ctl->error and gives up.
// `state` holds (epoch << 32 | round << 16 | colour) of the vertices coloured in the launch
// with that epoch, so nothing needs clearing between launches.
//
// The same cooperative launch then places the vertices in colour order, ascending body
// index inside each colour (what sorting (colour, body) keys gives): block b counts the
// colours of its contiguous share of the bodies, and after a grid barrier every block
// derives its colours' write positions from all blocks' counts and writes the solve list,
// the solve entries (body, row range) and each row's dual-owner / later-partner bits.
constexpr int COLOUR_FLOW_BLOCK = 256;

__global__ void __launch_bounds__(COLOUR_FLOW_BLOCK) k_colour_greedy(
    DevBodies B, DevForces F, int n, unsigned long long *state, unsigned epoch, int *colour, ColourControl *ctl,
    StepCounters *cnt, unsigned spinLimit, int *blockCounts, int *colourStart, int *solveList, int4 *entries,
    const int *rowStart, StepState *st)
{
    if (step_aborted(st)) // uniform: every block leaves before the first barrier
        return;
    __shared__ int hist[256];
    __shared__ int running[256];
    __shared__ int shTotal[256];
    __shared__ int shC, shVertices;
    const int stride = gridDim.x * blockDim.x;
    const int G = gridDim.x;
    const int lane = threadIdx.x & 31;
    int mine = 0, maxC = -1, maxR = -1;
    bool failed = false;
    // Warps take 32 consecutive bodies at a time and colour them in rounds. A lower-index
    // neighbour inside the warp is read from its lane by shuffles, so a chain of neighbours
    // inside the warp advances one link per shuffle pass, all in registers; a neighbour in
    // another warp is polled (without blocking) in memory once per round. A warp that makes
    // no progress in a round backs off, and after spinLimit such rounds the wait has expired.
    constexpr int NB = 8; // lower-index neighbours kept in registers (more: rescanned per round)
    for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n && !failed; base += stride)
    {
        const int v = base + lane;
        bool pending = false, many = false;
        int nb[NB];
        int nnb = 0;
        unsigned seen = 0;  // bit k: nb[k]'s colour is in `used`
        unsigned intra = 0; // bit k: nb[k] is a lane of this warp
        unsigned long long used[4] = {0ull, 0ull, 0ull, 0ull};
        int round = 0;
        unsigned mine_cr = ~0u; // round << 16 | colour once taken (read by the warp's shuffles)
        bool publish = false;  // taken in this round, not yet in `state`
        if (v < n)
        {
            pending = B.massMoment[v].x > 0 && F.adjStart[v + 1] > F.adjStart[v];
            if (!pending)
                __stcg(&colour[v], -1);
            else
                for (int k = F.adjStart[v]; k < F.adjStart[v + 1]; ++k)
                {
                    unsigned e = F.adj[k];
                    if (adj_type(e) == ADJ_IGNORE)
                        continue;
                    int2 ab = force_bodies(F, e);
                    int u = ab.x == v ? ab.y : ab.x;
                    // static bodies are not vertices; a dynamic neighbour shares this force
                    if (u < 0 || u >= v || B.massMoment[u].x <= 0)
                        continue;
                    if (nnb < NB)
                    {
                        if (u >= base)
                            intra |= 1u << nnb;
                        nb[nnb++] = u;
                    }
                    else
                        many = true;
                }
        }
        const unsigned all = (1u << nnb) - 1u;
        // shuffle passes look at the first kIntra neighbours (the warp's largest in-warp one)
        const int kIntra = __reduce_max_sync(0xFFFFFFFFu, 32 - __clz((int)intra));
        // takes the smallest colour no lower neighbour uses; `state` is written at the end of
        // the round, by all lanes that took one together (one release for the warp)
        auto take = [&]() {
            int c = 0;
            while (c < 256 && ((used[c >> 6] >> (c & 63)) & 1ull))
                c++;
            if (c >= 256)
            {
                cnt->error = DERR_TOO_MANY_COLOURS;
                c = 255;
            }
            __stcg(&colour[v], c);
            mine++;
            maxC = max(maxC, c);
            maxR = max(maxR, round);
            mine_cr = ((unsigned)min(round, 0xFFFF) << 16) | (unsigned)c;
            publish = true;
            pending = false;
        };
        unsigned idle = 0;
        while (__any_sync(0xFFFFFFFFu, pending))
        {
            bool progressed = false;
            if (pending && !many)
            {
                // neighbours in other warps
#pragma unroll
                for (int k = 0; k < NB; ++k)
                {
                    if (k >= nnb || (((seen | intra) >> k) & 1u))
                        continue;
                    const unsigned long long su = ld_acquire_u64(&state[nb[k]]);
                    if ((su >> 32) != (unsigned long long)epoch)
                        continue;
                    const int cu = (int)(su & 0xFFFFu), ru = (int)((su >> 16) & 0xFFFFu);
                    if (cu < 256)
                        used[cu >> 6] |= 1ull << (cu & 63);
                    round = max(round, ru + 1);
                    seen |= 1u << k;
                }
            }
            else if (pending)
            {
                // more than NB lower neighbours: look at all of them again each round
                bool ready = true;
                used[0] = used[1] = used[2] = used[3] = 0ull;
                round = 0;
                for (int k = F.adjStart[v]; k < F.adjStart[v + 1] && ready; ++k)
                {
                    unsigned e = F.adj[k];
                    if (adj_type(e) == ADJ_IGNORE)
                        continue;
                    int2 ab = force_bodies(F, e);
                    int u = ab.x == v ? ab.y : ab.x;
                    if (u < 0 || u >= v || B.massMoment[u].x <= 0)
                        continue;
                    const unsigned long long su = ld_acquire_u64(&state[u]);
                    if ((su >> 32) != (unsigned long long)epoch)
                    {
                        ready = false;
                        break;
                    }
                    const int cu = (int)(su & 0xFFFFu), ru = (int)((su >> 16) & 0xFFFFu);
                    if (cu < 256)
                        used[cu >> 6] |= 1ull << (cu & 63);
                    round = max(round, ru + 1);
                }
                if (ready)
                {
                    take();
                    progressed = true;
                }
            }
            // neighbours inside the warp: shuffle passes while any lane takes a colour
            for (;;)
            {
                bool took = false;
#pragma unroll
                for (int k = 0; k < NB; ++k)
                {
                    if (k >= kIntra) // warp-uniform
                        break;
                    const bool in = (intra >> k) & 1u;
                    const int src = in ? nb[k] - base : lane;
                    const unsigned cr = __shfl_sync(0xFFFFFFFFu, mine_cr, src);
                    if (pending && !many && in && !((seen >> k) & 1u) && cr != ~0u)
                    {
                        const int cu = (int)(cr & 0xFFFFu);
                        used[cu >> 6] |= 1ull << (cu & 63);
                        round = max(round, (int)(cr >> 16) + 1);
                        seen |= 1u << k;
                    }
                }
                if (pending && !many && seen == all)
                {
                    take();
                    took = true;
                    progressed = true;
                }
                if (!__any_sync(0xFFFFFFFFu, took))
                    break;
            }
            if (publish)
            {
                st_release_u64(&state[v], ((unsigned long long)epoch << 32) | (unsigned long long)mine_cr);
                publish = false;
            }
            if (__any_sync(0xFFFFFFFFu, progressed))
            {
                idle = 0;
                continue;
            }
            // no lane of the warp could move: its neighbours belong to other warps
            if (++idle >= spinLimit)
            {
                if (lane == 0)
                    atomicExch(&ctl->error, 1);
                failed = true;
                break;
            }
            if (idle > 16)
            {
                if (((volatile int *)&ctl->error)[0])
                {
                    failed = true;
                    break;
                }
                __nanosleep(32);
            }
        }
    }
    // vertices, largest colour and round of the launch
    {
        int s = block_sum(mine);
        if (threadIdx.x == 0 && s)
            atomicAdd(&ctl->vertices, s);
        int wc = __reduce_max_sync(0xFFFFFFFFu, maxC + 1) - 1;
        int wr = __reduce_max_sync(0xFFFFFFFFu, maxR + 1) - 1;
        if ((threadIdx.x & 31) == 0 && wc >= 0)
        {
            atomicMax(&ctl->maxColour, wc);
            atomicMax(&ctl->rounds, wr + 1);
        }
    }
    unsigned target = 0;
    auto failing = [&]() {
        if (blockIdx.x == 0 && threadIdx.x == 0 && st)
        {
            st->error = STEP_ERR_COLOURING;
            st->abort = ABORT_ERROR;
        }
    };
    if (!grid_barrier(ctl, target, spinLimit))
        return failing();
    // counts per colour of this block's share of the bodies
    const int chunk = (n + G - 1) / G;
    const int b0 = min(n, blockIdx.x * chunk), b1 = min(n, b0 + chunk);
    if (threadIdx.x == 0)
    {
        shVertices = ((volatile int *)&ctl->vertices)[0];
        shC = shVertices > 0 ? ((volatile int *)&ctl->maxColour)[0] + 1 : 0;
    }
    for (int c = threadIdx.x; c < 256; c += blockDim.x)
        hist[c] = 0;
    __syncthreads();
    const int C = shC;
    for (int v = b0 + threadIdx.x; v < b1; v += blockDim.x)
    {
        int c = __ldcg(&colour[v]);
        if (c >= 0)
            atomicAdd(&hist[c], 1);
    }
    __syncthreads();
    for (int c = threadIdx.x; c < C; c += blockDim.x)
        __stcg(&blockCounts[(size_t)c * G + blockIdx.x], hist[c]);
    if (!grid_barrier(ctl, target, spinLimit))
        return failing();
    // each colour's total and this block's first position inside the colour: the block
    // sums all blocks' counts of the colour together (G <= blockDim x a few)
    for (int c = 0; c < C; ++c)
    {
        int before = 0, total = 0;
        for (int b = threadIdx.x; b < G; b += blockDim.x)
        {
            int k = __ldcg(&blockCounts[(size_t)c * G + b]);
            total += k;
            before += b < (int)blockIdx.x ? k : 0;
        }
        total = block_sum(total);
        before = block_sum(before);
        if (threadIdx.x == 0)
        {
            shTotal[c] = total;
            running[c] = before;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        int acc = 0;
        for (int c = 0; c < C; ++c)
        {
            int t = shTotal[c];
            shTotal[c] = acc; // now the colour's start
            acc += t;
        }
    }
    __syncthreads();
    for (int c = threadIdx.x; c < C; c += blockDim.x)
        running[c] += shTotal[c];
    if (blockIdx.x == 0)
    {
        for (int c = threadIdx.x; c < C; c += blockDim.x)
            colourStart[c] = shTotal[c];
        if (threadIdx.x == 0)
            colourStart[C] = shVertices;
    }
    __syncthreads();
    // stable placement: tiles of the block's share, warps in order inside a tile
    const int warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    for (int base = b0; base < b1; base += blockDim.x)
    {
        const int v = base + threadIdx.x;
        const int c = v < b1 ? __ldcg(&colour[v]) : -1;
        const unsigned same = __match_any_sync(0xFFFFFFFFu, c);
        const int rank = __popc(same & lt);
        const bool leader = (same & lt) == 0;
        // only the positions need the warps in turn; the writes follow in parallel
        int pos = -1;
        for (int w = 0; w < COLOUR_FLOW_BLOCK / 32; ++w)
        {
            if (warp == w && c >= 0)
            {
                pos = running[c] + rank;
                __syncwarp(same);
                if (leader)
                    running[c] += __popc(same);
            }
            __syncthreads();
        }
        if (pos >= 0)
        {
            solveList[pos] = v;
            const int r0 = rowStart[v], r1 = rowStart[v + 1];
            entries[pos] = make_int4(v, r0, r1, 0);
            // the rows whose contact or joint dual update this body owns in the fused pass
            for (int r = r0; r < r1; ++r)
            {
                int2 row = F.rows[r];
                const int p = row_partner(row);
                const int cp = p >= 0 ? __ldcg(&colour[p]) : -1;
                const bool own = p < 0 || cp < 0 || c < cp;
                const bool later = p >= 0 && cp >= 0 && c < cp;
                row.y = own ? (row.y | ROW_OWNS_DUAL) : (row.y & ~ROW_OWNS_DUAL);
                row.y = later ? (row.y | ROW_PARTNER_LATER) : (row.y & ~ROW_PARTNER_LATER);
                F.rows[r] = row;
            }
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && st)
    {
        int err = ctl->error ? STEP_ERR_COLOURING
                             : (cnt->error == DERR_TOO_MANY_COLOURS ? STEP_ERR_COLOURS : STEP_ERR_NONE);
        st->nColours = C;
        st->nSolve = shVertices;
        st->rounds = ctl->rounds;
        if (err != STEP_ERR_NONE)
        {
            st->error = err;
            st->abort = ABORT_ERROR;
        }
    }
}

} // namespace avbd
