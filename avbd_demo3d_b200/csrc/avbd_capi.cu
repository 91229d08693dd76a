// Host side of the B200 AVBD step: context, device memory, launch orchestration and
// the C ABI declared in include/avbd_cuda.h.
//
// One avbd_step() runs what Solver::stepCpuReference does (solver.cpp:1036-1041) as a
// sequence of kernels on the context stream:
//   broadphase (grid or all pairs) -> new manifolds in the reference's creation order
//   -> manifold/joint initialisation -> compaction -> per-body force lists (CSR, newest
//   first) -> body warm start -> Jones-Plassmann colouring -> iterations x (per-colour
//   primal, dual) -> velocities.
// The host reads a handful of counts per step (new pairs, surviving forces, colouring
// progress, colour ranges) to size launches and buffers.
#include "../../include/avbd_cuda.h"
#include "avbd_kernels.cuh"

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <iomanip>
#include <sstream>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace avbd;

namespace
{

template <class T>
struct DArr
{
    T *p = nullptr;
    size_t cap = 0;
};

struct ManBuf
{
    DArr<int2> ab;
    DArr<unsigned long long> seq;
    DArr<int> n;
    DArr<float4> basis;
    DArr<float4> contact;
};

constexpr int PRIMAL_BLOCK = 128;
// iteration kernel: lanes per body, threads per block (one block per SM), threads per
// independently synchronised unit. Four units of 64 bodies: without grid barriers between
// colours the units drift apart, so one unit's factorisation (a few warps, latency-bound)
// overlaps the others' row gathering (every warp, issue-bound). The batch fills the units
// in order, which leaves the last one short and the units out of phase: measured 302 us
// per step's iterations on the 65,536-box scene, against 322 us for one unit per block and
// 316 us for four equal shares (in phase, their factorisations coincide).
constexpr int ITER_G = 4, ITER_BLOCK = 1024, ITER_SUB = 256;

// Primal kernel variants: lanes per body (G) and the occupancy target given to the
// compiler (resident blocks per SM; 1 = no register cap).
struct PrimalVariant
{
    int group, minBlocks;
    void (*kernel)(DevBodies, DevForces, Params, const int4 *, int, int);
};

const PrimalVariant kPrimalVariants[] = {
    {8, 1, k_primal<8, PRIMAL_BLOCK, 1>},   {8, 6, k_primal<8, PRIMAL_BLOCK, 6>},
    {8, 8, k_primal<8, PRIMAL_BLOCK, 8>},   {4, 1, k_primal<4, PRIMAL_BLOCK, 1>},
    {4, 6, k_primal<4, PRIMAL_BLOCK, 6>},   {16, 1, k_primal<16, PRIMAL_BLOCK, 1>},
    {16, 6, k_primal<16, PRIMAL_BLOCK, 6>}, {32, 1, k_primal<32, PRIMAL_BLOCK, 1>},
    {4, 8, k_primal<4, PRIMAL_BLOCK, 8>},   {2, 8, k_primal<2, PRIMAL_BLOCK, 8>},
};
constexpr int kNumPrimalVariants = (int)(sizeof(kPrimalVariants) / sizeof(kPrimalVariants[0]));
const PrimalVariant kRoundPrimal = {4, 1, k_primal<4, PRIMAL_BLOCK, 1, true>}; // worlds with round bodies

} // namespace

struct AdjointState; // avbd_adjoint.cuh

struct AvbdContext
{
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaMemPool_t pool = nullptr; // stream-ordered device allocations of this context
    bool ownStream = false;
    std::string err;
    int errCode = 0;
    AvbdParams params{};
    bool loaded = false;

    int n = 0;
    DArr<float4> pos, quat, initLin, initAng, inertLin, inertAng, vel, angvel, prevVel, massMoment, sizeRad;
    DArr<float4> dqLin, dqAng; // pose - initial pose (linear, qdiff), refreshed wherever the pose is written
    DArr<float4> initAngInv, inertAngInv; // inverses of the step's initial and inertial orientations
    DArr<float> friction;

    // worlds: static per-world classification, per-step grids (one grid per world)
    int W = 1;
    std::vector<int> hWorldStart;      // W + 1 body ranges
    std::vector<int> hBinned, hLarge;  // world by world, body order
    std::vector<int> hWorldLargeStart; // W + 1 ranges in hLarge
    std::vector<int4> hLLItems;        // large-large work items
    DArr<int> bodyWorld, worldStart, worldLargeStart, worldBinned;
    DArr<float> binnedRadiusW;
    DArr<int4> llItems;
    DArr<int> binned, large;
    DArr<float4> largeLo, largeHi, largeSphere;
    DArr<int> llCount, llOffset;
    DArr<uint4> llChunkLo, llChunkHi; // bounds of each large-list chunk's spheres (ordered ints)
    DArr<int> llRecorded;               // LL_SLOTS partners per large-large work item
    DArr<unsigned long long> pairSetKeys; // body pairs linked by a force, for the broadphase
    DArr<unsigned long long> largeKeys, largeKeysAlt;
    const unsigned long long *largeSorted = nullptr;
    DArr<unsigned> bounds;  // 8 words per world
    DArr<GridParams> grid;  // per world
    DArr<int> cappedAny;
    DArr<unsigned long long> cellHashKeys, largeHashKeys;
    DArr<unsigned> cellHashVals, largeHashVals;
    unsigned cellHashMask = 0, largeHashMask = 0;
    DArr<unsigned long long> bpKeys, bpKeysAlt;
    DArr<int> pairCount, pairOffset;
    DArr<int> pairRecorded; // BP_SLOTS new partners per grid entry lane from the counting pass
    DArr<int> pairLaneCount; // new partners per grid entry lane
    // LBVH broadphase mode: Morton-sorted binned bodies, tree nodes, grid position per body
    DArr<unsigned long long> lbvhCodes, lbvhCodesAlt;
    DArr<int> lbvhBodies, lbvhBodiesAlt, lbvhChild, lbvhParent, entryOf, worldBinnedStart;
    DArr<float4> lbvhLo, lbvhHi;
    DArr<unsigned> lbvhArrivals;
    DArr<int> sapVals, sapValsAlt, sapAxis; // sweep and prune: sorted bodies, axis per world

    ManBuf man[2];
    int cur = 0;
    int nMan = 0;
    DArr<unsigned char> keep;
    DArr<int> keepIdx;

    int nJoint = 0, nSpring = 0, nIgnore = 0;
    DArr<int2> jointAB[2];
    DArr<unsigned long long> jointSeq[2];
    DArr<float4> joint[2];
    int jcur = 0;
    DArr<unsigned long long> editSeq; // joint edits between steps: sorted sequence numbers,
    DArr<int2> editAB;                // their bodies, packed states (8 float4 each),
    DArr<float4> editData;            // matched joint per edit, then the match count
    DArr<int> editJoint;
    DArr<unsigned> snapIds, snapIdsAlt; // snapshot records: caller ids sorted with their bodies
    DArr<int> snapOrder, snapOrderAlt;
    DArr<uint4> snapRecords;
    DArr<int2> springAB, ignoreAB;
    DArr<unsigned long long> springSeq, ignoreSeq;
    DArr<float4> spring;

    DArr<int> adjStart;
    DArr<unsigned> adj, incVals, incValsAlt;
    DArr<int> rowCount, entryRow, rowStart; // rows per force-list entry, their offsets, ranges per body
    DArr<int2> rows;
    DArr<unsigned long long> incKeys, incKeysAlt;
    int incShift = 1; // sequence bits of the incidence keys of the current adjacency
    bool seqRanked = false; // force lists in ascending, distinct sequence order (incidences by rank)
    DArr<unsigned> incKeys32, incKeys32Alt; // body keys of the ranked incidences

    DArr<int> colourState, colour, solveList, colourStart;
    DArr<int4> solveEntry; // solve list with each body's row range, for the primal
    DArr<unsigned> colKeys, colKeysAlt;
    DArr<ColourControl> colourCtl;
    int colourBlocks = 148;   // co-resident blocks for the cooperative colouring launch
    int colourFlowBlocks = 148; // blocks of the greedy colouring's cooperative launch
    DArr<unsigned long long> colourFlow; // per body: (epoch, round, colour) of the greedy colouring
    DArr<int> colourBlockCounts;          // 256 colours x blocks
    unsigned colourEpoch = 0;
    int iterationMode = AVBD_ITERATIONS_PERSISTENT;
    DArr<float4> shape;      // (type, radius, half length, 0) per body when any body is round
    bool hasShapes = false;  // some body is not a box
    bool hasSpheres = false; // rolling friction pass after the velocity update
    int iterBlocks = 0;       // co-resident blocks of the iteration kernel (0: not launchable)
    DArr<IterSync> iterSync;
    DArr<int> iterDone; // per body: iterations completed in the running iteration launch
    int *hIterError = nullptr; // pinned: barrier expiry of the last iteration kernel
    int colourMode = 0;       // 0 greedy (list-index priority), 1 hashed priority
    int *hColourSummary = nullptr; // pinned: vertices, rounds, max colour, error
    int *hColourStarts = nullptr;  // pinned: 257 colour range starts
    std::vector<int> hColourStart;
    int nColours = 0, nSolve = 0;

    DArr<char> cubTemp;
    // Side streams of a device step: side[0] builds the pair set, the large bodies' boxes and
    // the large-large pass, side[1] the large bodies' cell lists, side[3] the LBVH mode's tree,
    // while the context stream bins and sorts the grid entries; side[2] initialises the
    // manifolds that existed before the step meanwhile. Events fork and join them (sideEv; 6
    // and 7 for side[2], 8 for the tree) and the broadphase's side streams have their own cub
    // scratch.
    cudaStream_t side[4] = {nullptr, nullptr, nullptr, nullptr};
    // a synchronous step's non-finite check (k_step_begin's flags, copied to hStepFlags) waits
    // to be read at the broadphase's first wait for the device, before anything changes
    bool flagsPending = false;
    cudaEvent_t sideEv[9] = {};
    DArr<char> cubTempSide[3];
    Lbvh lbvhTree{}; // the LBVH mode's tree of this step (built on side[3])
    DArr<StepCounters> counters;
    StepCounters *hCounters = nullptr;
    long long *hScalars = nullptr; // pinned scratch for small readbacks
    GridParams *hGrid = nullptr;   // pinned copy of the per-world grid parameters
    size_t hGridCap = 0;
    int *hCapped = nullptr;        // pinned: any world over the cell cap
    float4 *hStage = nullptr;      // pinned staging for body state transfers
    DArr<float> stateStage;        // the same on the device: body state in the callers' packed layout
    size_t hStageCap = 0;
    cudaEvent_t stageDone = nullptr; // staging copies issued before this event are complete

    long long nextSeq = 0;
    AvbdStats stats{};
    cudaEvent_t evStart = nullptr, evStop = nullptr;

    // profiling: events around each phase, summed per phase after the step
    int primalVariant = 4; // G = 4 lanes per body, 6 resident blocks per SM (autotuned on stacks)
    bool profiling = false;
    std::vector<cudaEvent_t> evPool;
    size_t evUsed = 0;
    std::vector<std::pair<int, std::pair<size_t, size_t>>> marks;
    double phaseMs[AVBD_PHASE_COUNT] = {0};
    long long phaseLaunches[AVBD_PHASE_COUNT] = {0};
    long long launches = 0;
    long long stepsProfiled = 0;

    // adjoint: checkpoints, tape and adjoint buffers; `recording` while a step is taped
    AdjointState *adjoint = nullptr;
    bool recording = false;

    // Device-resident steps (grid broadphase, single-launch iterations): the counts live in
    // a device StepState and a step issues all its launches without waiting for the device.
    // pendingFast steps have been issued since the host last read that state; until then the
    // host's nMan / nextSeq / cur are the values at that read (the *AtConfirm fields).
    DArr<StepState> stepState;
    StepState *hState = nullptr; // pinned copy of the state, written by every device step
    DArr<int> stepFlags;          // STEP_SEEN_* bits of the synchronous step's admission check
    int *hStepFlags = nullptr;    // pinned copy
    int stepMode = AVBD_STEP_DEVICE;
    int pendingFast = 0;
    int doneAtConfirm = 0, flipsAtConfirm = 0, curAtConfirm = 0;
    bool stateDirty = true;        // the host changed counts: write them to the device state
    unsigned long long seqBound = 0; // above every sequence number a pending step can create
    long long manifoldSpare = 0;   // manifold room beyond the live count (0: the default policy)
    long long deviceSteps = 0, redoneSteps = 0;
    unsigned waitColour = 0, waitIteration = 0; // poll limits of the bounded waits (0: default)

    // One step with caller-given pairs (and contacts) in place of the broadphase
    // (stepCpuReferenceWithExternalBroadphase): set by avbd_step_external for that step only.
    bool external = false;
    std::vector<int2> hExtPairs, hExtEntryPairs; // valid pairs; contact entries that may create
    DArr<int2> extPairs;
    DArr<unsigned char> extFlags;
    DArr<unsigned long long> extKeys;
    DArr<int> extEntry, extNum;
    DArr<float4> extBasis, extContact;
    int extKeyCount = 0;
};

namespace
{

int settle(AvbdContext *ctx);

int fail(AvbdContext *ctx, int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (ctx)
    {
        ctx->err = buf;
        ctx->errCode = code;
    }
    return code;
}

#define CU(call)                                                                                                   \
    do                                                                                                             \
    {                                                                                                              \
        cudaError_t e_ = (call);                                                                                   \
        if (e_ != cudaSuccess)                                                                                     \
            return fail(ctx, AVBD_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__,      \
                        __LINE__);                                                                                 \
    } while (0)

#define CHECK(expr)                                                                                                \
    do                                                                                                             \
    {                                                                                                              \
        int r_ = (expr);                                                                                           \
        if (r_ != AVBD_OK)                                                                                         \
            return r_;                                                                                             \
    } while (0)

// Entry points that read or change device state first wait for the device-resident steps
// issued so far (redoing any that stopped on the device), so calls act in issue order.
#define SETTLED()                                                                                                  \
    do                                                                                                             \
    {                                                                                                              \
        if (ctx && ctx->pendingFast)                                                                               \
            CHECK(settle(ctx));                                                                                    \
    } while (0)

#define LAUNCHED()                                                                                                 \
    do                                                                                                             \
    {                                                                                                              \
        ctx->launches++;                                                                                           \
        cudaError_t e_ = cudaGetLastError();                                                                       \
        if (e_ != cudaSuccess)                                                                                     \
            return fail(ctx, AVBD_ERR_CUDA, "kernel launch failed: %s (%s:%d)", cudaGetErrorString(e_), __FILE__,  \
                        __LINE__);                                                                                 \
    } while (0)

// Growth is stream-ordered (the context's memory pool keeps freed blocks cached), so a
// buffer that grows mid-run never synchronises the device.
template <class T>
int reserve(AvbdContext *ctx, DArr<T> &a, size_t count, bool preserve, size_t used = 0)
{
    if (count <= a.cap && a.p)
        return AVBD_OK;
    size_t cap = std::max(count, a.cap + a.cap / 2);
    cap = std::max<size_t>(cap, 16);
    T *p = nullptr;
    CU(cudaMallocFromPoolAsync((void **)&p, cap * sizeof(T), ctx->pool, ctx->stream));
    if (a.p)
    {
        if (preserve && used)
            CU(cudaMemcpyAsync(p, a.p, std::min(used, a.cap) * sizeof(T), cudaMemcpyDeviceToDevice, ctx->stream));
        CU(cudaFreeAsync(a.p, ctx->stream));
    }
    a.p = p;
    a.cap = cap;
    return AVBD_OK;
}

template <class T>
void release(DArr<T> &a)
{
    if (a.p)
        cudaFree(a.p); // only at destruction, after the stream has drained
    a.p = nullptr;
    a.cap = 0;
}

int grid_for(long long n, int block) { return (int)std::max<long long>(1, (n + block - 1) / block); }

int ensure_temp(AvbdContext *ctx, size_t bytes) { return reserve(ctx, ctx->cubTemp, bytes, false); }

// Phase timing with CUDA events on the context stream (enabled by avbd_set_profiling).
int prof_event(AvbdContext *ctx, size_t &idx)
{
    if (ctx->evUsed == ctx->evPool.size())
    {
        cudaEvent_t e;
        CU(cudaEventCreate(&e));
        ctx->evPool.push_back(e);
    }
    idx = ctx->evUsed++;
    CU(cudaEventRecord(ctx->evPool[idx], ctx->stream));
    return AVBD_OK;
}

struct PhaseScope
{
    AvbdContext *ctx;
    int phase;
    size_t begin = 0;
    bool on;
    PhaseScope(AvbdContext *c, int p) : ctx(c), phase(p), on(c->profiling)
    {
        if (on && prof_event(ctx, begin) != AVBD_OK)
            on = false;
    }
    ~PhaseScope()
    {
        size_t end;
        if (on && prof_event(ctx, end) == AVBD_OK)
            ctx->marks.push_back({phase, {begin, end}});
    }
};

int prof_collect(AvbdContext *ctx)
{
    if (ctx->marks.empty())
        return AVBD_OK;
    CU(cudaStreamSynchronize(ctx->stream));
    for (auto &m : ctx->marks)
    {
        float ms = 0.0f;
        CU(cudaEventElapsedTime(&ms, ctx->evPool[m.second.first], ctx->evPool[m.second.second]));
        ctx->phaseMs[m.first] += ms;
        ctx->phaseLaunches[m.first]++;
    }
    ctx->marks.clear();
    ctx->evUsed = 0;
    return AVBD_OK;
}

int reserve_manifolds(AvbdContext *ctx, ManBuf &b, size_t count, size_t used)
{
    CHECK(reserve(ctx, b.ab, count, true, used));
    CHECK(reserve(ctx, b.seq, count, true, used));
    CHECK(reserve(ctx, b.n, count, true, used));
    CHECK(reserve(ctx, b.basis, 3 * count, true, 3 * used));
    CHECK(reserve(ctx, b.contact, 32 * count, true, 32 * used));
    return AVBD_OK;
}

DevBodies dev_bodies(AvbdContext *ctx)
{
    DevBodies B;
    B.n = ctx->n;
    B.pos = ctx->pos.p;
    B.quat = ctx->quat.p;
    B.initLin = ctx->initLin.p;
    B.initAng = ctx->initAng.p;
    B.dqLin = ctx->dqLin.p;
    B.dqAng = ctx->dqAng.p;
    B.initAngInv = ctx->initAngInv.p;
    B.inertAngInv = ctx->inertAngInv.p;
    B.inertLin = ctx->inertLin.p;
    B.inertAng = ctx->inertAng.p;
    B.vel = ctx->vel.p;
    B.angvel = ctx->angvel.p;
    B.prevVel = ctx->prevVel.p;
    B.massMoment = ctx->massMoment.p;
    B.sizeRad = ctx->sizeRad.p;
    B.shape = ctx->hasShapes ? ctx->shape.p : nullptr;
    B.friction = ctx->friction.p;
    return B;
}

DevManifolds dev_man(ManBuf &b)
{
    DevManifolds M;
    M.ab = b.ab.p;
    M.seq = b.seq.p;
    M.n = b.n.p;
    M.basis = b.basis.p;
    M.contact = b.contact.p;
    return M;
}

DevForces dev_forces(AvbdContext *ctx)
{
    DevForces F;
    F.nMan = ctx->nMan;
    F.man = dev_man(ctx->man[ctx->cur]);
    F.nJoint = ctx->nJoint;
    F.jointAB = ctx->jointAB[ctx->jcur].p;
    F.jointSeq = ctx->jointSeq[ctx->jcur].p;
    F.joint = ctx->joint[ctx->jcur].p;
    F.nSpring = ctx->nSpring;
    F.springAB = ctx->springAB.p;
    F.springSeq = ctx->springSeq.p;
    F.spring = ctx->spring.p;
    F.nIgnore = ctx->nIgnore;
    F.ignoreAB = ctx->ignoreAB.p;
    F.ignoreSeq = ctx->ignoreSeq.p;
    F.adjStart = ctx->adjStart.p;
    F.adj = ctx->adj.p;
    F.rowStart = ctx->rowStart.p;
    F.rows = ctx->rows.p;
    return F;
}

DevGrid dev_grid(AvbdContext *ctx)
{
    DevGrid G;
    G.W = ctx->W;
    G.bodyWorld = ctx->bodyWorld.p;
    G.worldStart = ctx->worldStart.p;
    G.binnedRadius = ctx->binnedRadiusW.p;
    G.worldLargeStart = ctx->worldLargeStart.p;
    G.bounds = ctx->bounds.p;
    G.grid = ctx->grid.p;
    G.cappedAny = ctx->cappedAny.p;
    return G;
}

HashTable cell_hash(AvbdContext *ctx)
{
    return HashTable{ctx->cellHashKeys.p, ctx->cellHashVals.p, ctx->cellHashMask};
}

HashTable large_hash(AvbdContext *ctx)
{
    return HashTable{ctx->largeHashKeys.p, ctx->largeHashVals.p, ctx->largeHashMask};
}

Params dev_params(const AvbdParams &p)
{
    Params P;
    P.dt = p.dt;
    P.gravity = p.gravity;
    P.iterations = p.iterations;
    P.alpha = p.alpha;
    P.betaLin = p.betaLin;
    P.betaAng = p.betaAng;
    P.gamma = p.gamma;
    return P;
}

// Exclusive scan of n ints into out; total (out[n-1] + in[n-1]) lands in hScalars[slot].
int scan_counts(AvbdContext *ctx, const int *in, int *out, int n, int slot)
{
    size_t bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, ctx->stream);
    CHECK(ensure_temp(ctx, bytes));
    CU(cub::DeviceScan::ExclusiveSum(ctx->cubTemp.p, bytes, in, out, n, ctx->stream));
    return AVBD_OK;
}

__global__ void k_total(const int *scan, const int *in, int n, long long *out)
{
    *out = (long long)scan[n - 1] + (long long)in[n - 1];
}

// Colouring summary into pinned host memory: vertices, rounds, max colour, error.
__global__ void k_colour_count(const ColourControl *ctl, int *unused, int *summary)
{
    summary[0] = ctl->vertices;
    summary[1] = ctl->rounds;
    summary[2] = ctl->maxColour;
    summary[3] = ctl->error;
}

__global__ void k_solve_list_all(const unsigned *keys, int n, int *list, int *colourStart, const ColourControl *ctl,
                                 const int *rowStart, int4 *entries, const int *colour, int2 *rows,
                                 StepState *st = nullptr, const StepCounters *cnt = nullptr)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    int count = ctl->vertices;
    int nColours = count > 0 ? ctl->maxColour + 1 : 0;
    if (st)
    {
        if (step_aborted(st))
            return;
        if (k == 0)
        {
            // a failed colouring stops this step and every later one
            int err = ctl->error ? STEP_ERR_COLOURING
                                 : (cnt->error == DERR_TOO_MANY_COLOURS ? STEP_ERR_COLOURS : STEP_ERR_NONE);
            st->nColours = nColours;
            st->nSolve = count;
            st->rounds = ctl->rounds;
            if (err != STEP_ERR_NONE)
            {
                st->error = err;
                st->abort = ABORT_ERROR;
            }
        }
    }
    if (k >= count)
        return;
    unsigned key = keys[k];
    int b = (int)(key & 0xFFFFFFu);
    list[k] = b;
    int r0 = rowStart[b], r1 = rowStart[b + 1];
    entries[k] = make_int4(b, r0, r1, 0);
    // the contact rows whose dual update this body owns in a fused pass
    int cb = colour[b];
    for (int r = r0; r < r1; ++r)
    {
        int2 row = rows[r];
        int p = row_partner(row);
        bool own = p < 0 || colour[p] < 0 || cb < colour[p];
        bool later = p >= 0 && colour[p] >= 0 && cb < colour[p];
        row.y = own ? (row.y | ROW_OWNS_DUAL) : (row.y & ~ROW_OWNS_DUAL);
        row.y = later ? (row.y | ROW_PARTNER_LATER) : (row.y & ~ROW_PARTNER_LATER);
        rows[r] = row;
    }
    int c = (int)(key >> 24);
    int prev = k > 0 ? (int)(keys[k - 1] >> 24) : -1;
    for (int x = prev + 1; x <= c; ++x)
        colourStart[x] = k;
    if (k == count - 1)
        for (int x = c + 1; x <= nColours; ++x)
            colourStart[x] = count;
}

__global__ void k_u8_to_int(const unsigned char *in, int *out, int n, const StepState *st = nullptr)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    // device-resident steps: the launch covers the capacity, the live count is the state's
    out[k] = (!st || k < st->nManBp) ? in[k] : 0;
}

// Host counts into the device step state (after a load, an edit or a synchronous step).
__global__ void k_state_set(StepState *st, int nMan, unsigned long long nextSeq)
{
    StepState s = {};
    s.nMan = nMan;
    s.nManBp = nMan;
    s.nextSeq = nextSeq;
    *st = s;
}

// After the counting passes of the grid broadphase: the new pairs' total, their place
// after the live manifolds and their sequence numbers, or a stop when they do not fit or
// the grid needs the host's cell-count cap.
__global__ void k_bp_commit(StepState *st, const int *offset, const int *count, int nB, const int *llOffset,
                            const int *llCount, int nItems, const int *cappedAny, const StepCounters *cnt,
                            long long capacity)
{
    if (st->abort)
        return;
    if ((cappedAny && *cappedAny) || cnt->error)
    {
        st->abort = ABORT_GRID;
        return;
    }
    long long p1 = nB > 0 ? (long long)offset[nB - 1] + count[nB - 1] : 0;
    long long p2 = nItems > 0 ? (long long)llOffset[nItems - 1] + llCount[nItems - 1] : 0;
    if ((long long)st->nMan + p1 + p2 > capacity)
    {
        st->abort = ABORT_MANIFOLDS;
        return;
    }
    st->manBase = st->nMan;
    st->newBinned = (int)p1;
    st->seqBase = st->nextSeq;
    st->nManBp = st->nMan + (int)(p1 + p2);
    st->nextSeq += (unsigned long long)(p1 + p2);
    st->created = (int)(p1 + p2);
}

// End of a device-resident step: an expired iteration wait stops every later step.
__global__ void k_step_end(StepState *st, const IterSync *sync)
{
    if (st->abort)
        return;
    if (sync->error)
    {
        st->error = STEP_ERR_ITERATION;
        st->abort = ABORT_ERROR;
        return;
    }
    st->stepsDone++;
}

// Per-body force lists (CSR) sorted newest first.
template <class Key>
int build_rows(AvbdContext *ctx, const Key *sortedKeys, int total, size_t manifolds, const StepState *st = nullptr);

// Bits needed to write v (0 for v = 0).
int bit_width(unsigned long long v) { return v ? 64 - __builtin_clzll(v) : 0; }

// Manifolds both buffers can hold.
size_t man_capacity(const AvbdContext *ctx)
{
    size_t c = ~(size_t)0;
    for (const ManBuf &b : ctx->man)
        c = std::min({c, b.ab.cap, b.seq.cap, b.n.cap, b.basis.cap / 3, b.contact.cap / 32});
    return c == ~(size_t)0 ? 0 : c;
}

// `deviceCounts`: a device-resident step; the manifold count is the step state's, so the
// incidences cover the manifold buffers' capacity and the unused slots sort last.
int build_adjacency(AvbdContext *ctx, bool deviceCounts = false)
{
    int n = ctx->n;
    CHECK(reserve(ctx, ctx->adjStart, (size_t)n + 1, false));
    const size_t mans = deviceCounts ? man_capacity(ctx) : (size_t)ctx->nMan;
    long long T = 2ll * ((long long)mans + ctx->nJoint + ctx->nSpring + ctx->nIgnore);
    if (T == 0)
    {
        CU(cudaMemsetAsync(ctx->adjStart.p, 0, sizeof(int) * ((size_t)n + 1), ctx->stream));
        return build_rows<unsigned>(ctx, nullptr, 0, 0);
    }
    if (T > (long long)ADJ_INDEX_MASK)
        return fail(ctx, AVBD_ERR_CAPACITY, "too many force incidences (%lld)", T);
    CHECK(reserve(ctx, ctx->incVals, T, false));
    CHECK(reserve(ctx, ctx->incValsAlt, T, false));
    CHECK(reserve(ctx, ctx->adj, T, false));
    DevForces F = dev_forces(ctx);
    const StepState *st = deviceCounts ? ctx->stepState.p : nullptr;
    if (ctx->seqRanked)
    {
        // incidences in newest-first order of their forces, then a stable sort by body
        CHECK(reserve(ctx, ctx->incKeys32, T, false));
        CHECK(reserve(ctx, ctx->incKeys32Alt, T, false));
        const int forces = (int)(T / 2);
        k_incidences_ranked<<<grid_for(forces, 256), 256, 0, ctx->stream>>>(F, n, ctx->incKeys32.p, ctx->incVals.p,
                                                                            st, forces);
        LAUNCHED();
        cub::DoubleBuffer<unsigned> dk(ctx->incKeys32.p, ctx->incKeys32Alt.p);
        cub::DoubleBuffer<unsigned> dv(ctx->incVals.p, ctx->incValsAlt.p);
        const int endBit = std::max(1, bit_width((unsigned long long)n));
        size_t bytes = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, bytes, dk, dv, (int)T, 0, endBit, ctx->stream);
        CHECK(ensure_temp(ctx, bytes));
        CU(cub::DeviceRadixSort::SortPairs(ctx->cubTemp.p, bytes, dk, dv, (int)T, 0, endBit, ctx->stream));
        ctx->launches++;
        ctx->incShift = 0;
        k_segment_starts<<<grid_for(T, 256), 256, 0, ctx->stream>>>(dk.Current(), (int)T, 0, n, ctx->adjStart.p, st);
        LAUNCHED();
        k_copy_adj<<<grid_for(T, 256), 256, 0, ctx->stream>>>(dv.Current(), ctx->adj.p, (int)T, st);
        LAUNCHED();
        return build_rows(ctx, dk.Current(), (int)T, mans, st);
    }
    CHECK(reserve(ctx, ctx->incKeys, T, false));
    CHECK(reserve(ctx, ctx->incKeysAlt, T, false));
    // every sequence number is below nextSeq (below seqBound while steps are pending on the
    // device): the key needs bit_width(that) + bit_width(n) bits
    const unsigned long long seqTop = deviceCounts ? ctx->seqBound : (unsigned long long)ctx->nextSeq;
    int shift = std::max(1, bit_width(std::max<unsigned long long>(seqTop, 1)));
    int endBit = shift + bit_width((unsigned long long)n);
    if (shift > KEY_SEQ_BITS || endBit > 64)
        return fail(ctx, AVBD_ERR_CAPACITY, "sequence numbers (%llu) too large for the incidence keys", seqTop);
    ctx->incShift = shift;
    k_incidences<<<grid_for(T, 256), 256, 0, ctx->stream>>>(F, shift, n, ctx->incKeys.p, ctx->incVals.p,
                                                            deviceCounts ? ctx->stepState.p : nullptr, (int)T);
    LAUNCHED();
    cub::DoubleBuffer<unsigned long long> dk(ctx->incKeys.p, ctx->incKeysAlt.p);
    cub::DoubleBuffer<unsigned> dv(ctx->incVals.p, ctx->incValsAlt.p);
    size_t bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, dk, dv, (int)T, 0, endBit, ctx->stream);
    CHECK(ensure_temp(ctx, bytes));
    CU(cub::DeviceRadixSort::SortPairs(ctx->cubTemp.p, bytes, dk, dv, (int)T, 0, endBit, ctx->stream));
    ctx->launches++;
    k_segment_starts<<<grid_for(T, 256), 256, 0, ctx->stream>>>(dk.Current(), (int)T, shift, n, ctx->adjStart.p, st);
    LAUNCHED();
    k_copy_adj<<<grid_for(T, 256), 256, 0, ctx->stream>>>(dv.Current(), ctx->adj.p, (int)T, st);
    LAUNCHED();
    return build_rows(ctx, dk.Current(), (int)T, mans, st);
}

// The primal's row list, one (entry, row) pair per constraint row in force order, for the
// dynamic bodies (no host read: sized by an upper bound, ranges from a device scan).
template <class Key>
int build_rows(AvbdContext *ctx, const Key *sortedKeys, int total, size_t manifolds, const StepState *st)
{
    int n = ctx->n;
    CHECK(reserve(ctx, ctx->rowStart, (size_t)n + 1, false));
    if (total == 0)
    {
        CU(cudaMemsetAsync(ctx->rowStart.p, 0, sizeof(int) * ((size_t)n + 1), ctx->stream));
        return AVBD_OK;
    }
    CHECK(reserve(ctx, ctx->rowCount, (size_t)total + 1, false));
    CHECK(reserve(ctx, ctx->entryRow, (size_t)total + 1, false));
    size_t bound = 16 * manifolds + 6 * (size_t)ctx->nJoint + 2 * (size_t)ctx->nSpring;
    CHECK(reserve(ctx, ctx->rows, std::max<size_t>(bound, 1), false));
    DevForces F = dev_forces(ctx);
    k_entry_rows<<<grid_for((long long)total + 1, 256), 256, 0, ctx->stream>>>(F, dev_bodies(ctx), sortedKeys, total,
                                                                               ctx->incShift, ctx->rowCount.p, st);
    LAUNCHED();
    CHECK(scan_counts(ctx, ctx->rowCount.p, ctx->entryRow.p, total + 1, 0));
    ctx->launches++;
    k_row_starts<<<grid_for((long long)n + 1, 256), 256, 0, ctx->stream>>>(ctx->adjStart.p, ctx->entryRow.p, n,
                                                                           ctx->rowStart.p, st);
    LAUNCHED();
    F = dev_forces(ctx);
    k_entry_fill<<<grid_for(total, 256), 256, 0, ctx->stream>>>(F, ctx->entryRow.p, ctx->rowCount.p, total, st);
    LAUNCHED();
    return AVBD_OK;
}

// The reference's cell-count cap (solver.cpp:341-357) with the host C library's cbrtf, the
// function the reference itself calls, so the rescaled grid matches bit for bit.
void host_grid_cap(GridParams &g)
{
    const unsigned long long maxCells = 1ull << 22;
    float cellSize = g.cellSize0;
    int nx, ny, nz;
    auto dims = [&](float cs) -> unsigned long long {
        nx = (int)(g.extx / cs) + 1;
        ny = (int)(g.exty / cs) + 1;
        nz = (int)(g.extz / cs) + 1;
        return (unsigned long long)nx * (unsigned long long)ny * (unsigned long long)nz;
    };
    unsigned long long numCells = dims(cellSize);
    while (numCells > maxCells)
    {
        float f = cbrtf((float)numCells / (float)maxCells);
        cellSize *= f > 1.1f ? f : 1.1f;
        numCells = dims(cellSize);
    }
    g.cellSize = cellSize;
    g.nx = nx;
    g.ny = ny;
    g.nz = nz;
    g.numCells = numCells;
    g.capped = 0;
}

// Large bodies binned into the grid cells of their world that their inflated AABB touches:
// sorted (world, cell, index) keys and a hash table of run starts, including each world's
// global run for bodies spanning too many cells.
// keys: world | global (1) | cell (22) | large index (24), written large body by large body:
// the stable sort orders (world, global, cell) only and keeps each run in large-index order.
// Unused slots (all ones) still sort last.
int large_sort_end(const AvbdContext *ctx) { return 47 + std::max(1, bit_width((unsigned long long)(ctx->W - 1))); }

// cub scratch the large bodies' cell-list sort needs (reserved before the lists are built
// on a side stream)
size_t large_sort_bytes(AvbdContext *ctx, int nL)
{
    if (!nL)
        return 0;
    cub::DoubleBuffer<unsigned long long> lk(ctx->largeKeys.p, ctx->largeKeysAlt.p);
    size_t bytes = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, bytes, lk, nL * LARGE_MAX_CELLS, 24, large_sort_end(ctx));
    return bytes;
}

// The large bodies' cell lists on stream s, with scratch `temp` already reserved for
// large_sort_bytes (no allocation here: s may be a side stream).
int large_cell_lists(AvbdContext *ctx, int nL, cudaStream_t s, DArr<char> &temp)
{
    ctx->largeSorted = ctx->largeKeys.p;
    if (!nL)
        return AVBD_OK;
    int total = nL * LARGE_MAX_CELLS;
    k_bp_large_cells<<<grid_for(nL, 128), 128, 0, s>>>(dev_grid(ctx), ctx->large.p, ctx->largeLo.p, ctx->largeHi.p,
                                                       nL, ctx->largeKeys.p);
    LAUNCHED();
    cub::DoubleBuffer<unsigned long long> lk(ctx->largeKeys.p, ctx->largeKeysAlt.p);
    size_t bytes = temp.cap;
    CU(cub::DeviceRadixSort::SortKeys(temp.p, bytes, lk, total, 24, large_sort_end(ctx), s));
    ctx->launches++;
    ctx->largeSorted = lk.Current();
    // sentinel after the sorted keys: candidate walks stop at it
    CU(cudaMemsetAsync(lk.Current() + total, 0xFF, sizeof(unsigned long long), s));
    CU(cudaMemsetAsync(ctx->largeHashKeys.p, 0xFF, sizeof(unsigned long long) * ((size_t)ctx->largeHashMask + 1), s));
    k_bp_hash_large_runs<<<grid_for(total, 256), 256, 0, s>>>(lk.Current(), total, large_hash(ctx));
    LAUNCHED();
    return AVBD_OK;
}

// The LBVH part of the grid's counting pass: each world's tree over its binned bodies
// (lbvh_build, which needs only the grid parameters and the bodies, so it runs beside the
// grid entries' sort), then every grid entry's binned partners through it (lbvh_count, which
// writes the entry totals). lbvh_reserve sizes every buffer first, on the context stream.
int lbvh_reserve(AvbdContext *ctx, int nB)
{
    CHECK(reserve(ctx, ctx->lbvhCodes, (size_t)nB, false));
    CHECK(reserve(ctx, ctx->lbvhCodesAlt, (size_t)nB, false));
    CHECK(reserve(ctx, ctx->lbvhBodies, (size_t)nB, false));
    CHECK(reserve(ctx, ctx->lbvhBodiesAlt, (size_t)nB, false));
    CHECK(reserve(ctx, ctx->lbvhChild, 2 * (size_t)nB, false));
    CHECK(reserve(ctx, ctx->lbvhParent, 2 * (size_t)nB, false));
    CHECK(reserve(ctx, ctx->lbvhLo, 2 * (size_t)nB, false));
    CHECK(reserve(ctx, ctx->lbvhHi, 2 * (size_t)nB, false));
    CHECK(reserve(ctx, ctx->lbvhArrivals, (size_t)nB, false));
    CHECK(reserve(ctx, ctx->entryOf, (size_t)ctx->n, false));
    cub::DoubleBuffer<unsigned long long> dk(ctx->lbvhCodes.p, ctx->lbvhCodesAlt.p);
    cub::DoubleBuffer<int> dv(ctx->lbvhBodies.p, ctx->lbvhBodiesAlt.p);
    size_t bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, dk, dv, nB, 0, 32 + bit_width((unsigned long long)(ctx->W - 1)));
    return reserve(ctx, ctx->cubTempSide[2], std::max<size_t>(bytes, 16), false);
}

// Morton codes, their sort, the Karras build and the bottom-up refit, on stream s.
int lbvh_build(AvbdContext *ctx, int nB, cudaStream_t s)
{
    const int W = ctx->W;
    DevBodies B = dev_bodies(ctx);
    DevGrid G = dev_grid(ctx);
    k_lbvh_codes<<<grid_for(nB, 256), 256, 0, s>>>(B, G, ctx->binned.p, nB, ctx->lbvhCodes.p, ctx->lbvhBodies.p);
    LAUNCHED();
    cub::DoubleBuffer<unsigned long long> dk(ctx->lbvhCodes.p, ctx->lbvhCodesAlt.p);
    cub::DoubleBuffer<int> dv(ctx->lbvhBodies.p, ctx->lbvhBodiesAlt.p);
    const int endBit = 32 + bit_width((unsigned long long)(W - 1));
    size_t bytes = ctx->cubTempSide[2].cap;
    CU(cub::DeviceRadixSort::SortPairs(ctx->cubTempSide[2].p, bytes, dk, dv, nB, 0, endBit, s));
    ctx->launches++;
    CU(cudaMemsetAsync(ctx->lbvhParent.p, 0xFF, sizeof(int) * 2 * (size_t)nB, s));
    CU(cudaMemsetAsync(ctx->lbvhArrivals.p, 0, sizeof(unsigned) * (size_t)nB, s));
    Lbvh &T = ctx->lbvhTree;
    T.codes = dk.Current();
    T.bodies = dv.Current();
    T.segStart = ctx->worldBinnedStart.p;
    T.W = W;
    T.n = nB;
    T.child = ctx->lbvhChild.p;
    T.parent = ctx->lbvhParent.p;
    T.lo = ctx->lbvhLo.p;
    T.hi = ctx->lbvhHi.p;
    T.arrivals = ctx->lbvhArrivals.p;
    k_lbvh_build<<<grid_for(nB, 128), 128, 0, s>>>(T);
    LAUNCHED();
    k_lbvh_refit<<<grid_for(nB, 128), 128, 0, s>>>(T, B);
    LAUNCHED();
    return AVBD_OK;
}

// The grid entries' partners through the tree, on the context stream (after the build).
int lbvh_count(AvbdContext *ctx, const unsigned long long *gridKeys, int nB, const PairSet &S)
{
    k_grid_entry_of<<<grid_for(nB, 256), 256, 0, ctx->stream>>>(gridKeys, nB, ctx->entryOf.p);
    LAUNCHED();
    k_lbvh_count<<<grid_for(nB, 128), 128, 0, ctx->stream>>>(dev_bodies(ctx), dev_forces(ctx), dev_grid(ctx),
                                                             ctx->lbvhTree, gridKeys, nB, ctx->entryOf.p,
                                                             ctx->pairCount.p, ctx->pairLaneCount.p,
                                                             ctx->pairRecorded.p, ctx->counters.p, S);
    LAUNCHED();
    return AVBD_OK;
}

// Broadphase of every world: appends new manifolds after the existing ones. `deviceCounts`
// (grid mode only): no host read; k_bp_commit places the new pairs from the device counts
// and the emitting passes take their base from the step state.
// The non-finite check of a synchronous step, read after the first wait of its broadphase
// (which has changed nothing yet): the step is refused before its new pairs are written.
int nonfinite_checked(AvbdContext *ctx)
{
    if (!ctx->flagsPending)
        return AVBD_OK;
    ctx->flagsPending = false;
    if (*ctx->hStepFlags & STEP_SEEN_NONFINITE)
        return fail(ctx, AVBD_ERR_STATE,
                    "non-finite body position, orientation or velocity at the start of a step (the step was not run)");
    return AVBD_OK;
}

int broadphase(AvbdContext *ctx, bool deviceCounts = false)
{
    int n = ctx->n;
    if (deviceCounts && n < 2)
    {
        // still commit (no new pairs), so the step state carries this step's counts
        k_bp_commit<<<1, 1, 0, ctx->stream>>>(ctx->stepState.p, nullptr, nullptr, 0, nullptr, nullptr, 0,
                                              nullptr, ctx->counters.p, (long long)man_capacity(ctx));
        LAUNCHED();
        return AVBD_OK;
    }
    if (n < 2)
        return AVBD_OK;
    DevBodies B = dev_bodies(ctx);
    DevGrid G = dev_grid(ctx);
    float dt = ctx->params.dt;
    StepCounters *cnt = ctx->counters.p;
    int M0 = ctx->nMan;
    long long P1 = 0, P2 = 0;
    const int mode = ctx->params.broadphase;
    if (mode == AVBD_BROADPHASE_ALL_PAIRS)
    {
        CHECK(reserve(ctx, ctx->pairCount, n, false));
        CHECK(reserve(ctx, ctx->pairOffset, n, false));
        DevForces F = dev_forces(ctx);
        k_bp_all_pairs<false><<<grid_for(n, 128), 128, 0, ctx->stream>>>(B, F, G, n, ctx->pairCount.p, nullptr, 0, 0,
                                                                          cnt);
        LAUNCHED();
        CHECK(scan_counts(ctx, ctx->pairCount.p, ctx->pairOffset.p, n, 0));
        ctx->launches++;
        k_total<<<1, 1, 0, ctx->stream>>>(ctx->pairOffset.p, ctx->pairCount.p, n, ctx->hScalars);
        LAUNCHED();
        CU(cudaStreamSynchronize(ctx->stream));
        CHECK(nonfinite_checked(ctx));
        P1 = ctx->hScalars[0];
        if (P1 > 0)
        {
            CHECK(reserve_manifolds(ctx, ctx->man[ctx->cur], (size_t)(M0 + P1), (size_t)M0));
            DevForces F2 = dev_forces(ctx);
            k_bp_all_pairs<true><<<grid_for(n, 128), 128, 0, ctx->stream>>>(
                B, F2, G, n, nullptr, ctx->pairOffset.p, M0, (unsigned long long)ctx->nextSeq, cnt);
            LAUNCHED();
        }
    }
    else if (mode == AVBD_BROADPHASE_SAP)
    {
        // axis per world -> interval keys -> stable sort -> counted sweep -> emitted pairs
        const int W = ctx->W;
        CHECK(reserve(ctx, ctx->sapAxis, (size_t)W, false));
        CHECK(reserve(ctx, ctx->bpKeys, n, false));
        CHECK(reserve(ctx, ctx->bpKeysAlt, n, false));
        CHECK(reserve(ctx, ctx->sapVals, n, false));
        CHECK(reserve(ctx, ctx->sapValsAlt, n, false));
        CHECK(reserve(ctx, ctx->pairCount, n, false));
        CHECK(reserve(ctx, ctx->pairOffset, n, false));
        k_sap_axis<<<W, SAP_TILE, 0, ctx->stream>>>(B, ctx->worldStart.p, ctx->sapAxis.p);
        LAUNCHED();
        k_sap_keys<<<grid_for(n, 256), 256, 0, ctx->stream>>>(B, ctx->bodyWorld.p, ctx->sapAxis.p, ctx->bpKeys.p,
                                                              ctx->sapVals.p);
        LAUNCHED();
        cub::DoubleBuffer<unsigned long long> dk(ctx->bpKeys.p, ctx->bpKeysAlt.p);
        cub::DoubleBuffer<int> dv(ctx->sapVals.p, ctx->sapValsAlt.p);
        int endBit = 32;
        while ((1 << (endBit - 32)) < W)
            ++endBit;
        size_t bytes = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, bytes, dk, dv, n, 0, endBit, ctx->stream);
        CHECK(ensure_temp(ctx, bytes));
        CU(cub::DeviceRadixSort::SortPairs(ctx->cubTemp.p, bytes, dk, dv, n, 0, endBit, ctx->stream));
        ctx->launches++;
        DevForces F = dev_forces(ctx);
        k_sap_sweep<false><<<grid_for(n, 128), 128, 0, ctx->stream>>>(B, F, ctx->sapAxis.p, dk.Current(),
                                                                       dv.Current(), n, ctx->pairCount.p, nullptr, 0,
                                                                       0, cnt);
        LAUNCHED();
        CHECK(scan_counts(ctx, ctx->pairCount.p, ctx->pairOffset.p, n, 0));
        ctx->launches++;
        k_total<<<1, 1, 0, ctx->stream>>>(ctx->pairOffset.p, ctx->pairCount.p, n, ctx->hScalars);
        LAUNCHED();
        CU(cudaStreamSynchronize(ctx->stream));
        CHECK(nonfinite_checked(ctx));
        P1 = ctx->hScalars[0];
        if (P1 > 0)
        {
            CHECK(reserve_manifolds(ctx, ctx->man[ctx->cur], (size_t)(M0 + P1), (size_t)M0));
            DevForces F2 = dev_forces(ctx);
            k_sap_sweep<true><<<grid_for(n, 128), 128, 0, ctx->stream>>>(B, F2, ctx->sapAxis.p, dk.Current(),
                                                                          dv.Current(), n, nullptr,
                                                                          ctx->pairOffset.p, M0,
                                                                          (unsigned long long)ctx->nextSeq, cnt);
            LAUNCHED();
        }
    }
    else
    {
        if (mode != AVBD_BROADPHASE_GRID && mode != AVBD_BROADPHASE_LBVH)
            return fail(ctx, AVBD_ERR_ARGUMENT, "broadphase mode %d is not implemented on the GPU", mode);
        const bool lbvh = mode == AVBD_BROADPHASE_LBVH;
        const int nB = (int)ctx->hBinned.size(), nL = (int)ctx->hLarge.size();
        const int nItems = (int)ctx->hLLItems.size();
        // Three streams: the context stream bins and sorts the grid entries and counts their
        // pairs; side[0] builds the pair set, the large bodies' boxes and the large-large
        // pass; side[1] the large bodies' cell lists (after the grid parameters and the
        // boxes). Every buffer the side streams touch is reserved before they fork, since
        // growth is ordered on the context stream.
        cudaStream_t M = ctx->stream, S1 = ctx->side[0], S2 = ctx->side[1];
        cudaEvent_t evFork = ctx->sideEv[0], evPairSet = ctx->sideEv[1], evLarge = ctx->sideEv[2],
                    evParams = ctx->sideEv[3], evLists = ctx->sideEv[4], evLL = ctx->sideEv[5];
        StepState *stp = deviceCounts ? ctx->stepState.p : nullptr;
        // the body pairs the existing forces link (constrainedTo by one hash probe run)
        PairSet S;
        const long long forces = (long long)(deviceCounts ? man_capacity(ctx) : (size_t)ctx->nMan) + ctx->nJoint +
                                 ctx->nSpring + ctx->nIgnore;
        unsigned long long slots = 1024;
        while (slots < 2ull * (unsigned long long)forces)
            slots <<= 1;
        CHECK(reserve(ctx, ctx->pairSetKeys, (size_t)slots, false));
        S.keys = ctx->pairSetKeys.p;
        S.mask = (unsigned)(slots - 1);
        if (nItems > 0)
        {
            CHECK(reserve(ctx, ctx->llChunkLo, (size_t)nL, false));
            CHECK(reserve(ctx, ctx->llChunkHi, (size_t)nL, false));
            CHECK(reserve(ctx, ctx->llRecorded, (size_t)nItems * LL_SLOTS, false));
            size_t bytes = 0;
            cub::DeviceScan::ExclusiveSum(nullptr, bytes, ctx->llCount.p, ctx->llOffset.p, nItems);
            CHECK(reserve(ctx, ctx->cubTempSide[0], std::max<size_t>(bytes, 16), false));
        }
        if (nB && nL)
            CHECK(reserve(ctx, ctx->cubTempSide[1], std::max<size_t>(large_sort_bytes(ctx, nL), 16), false));
        if (nB && lbvh)
            CHECK(lbvh_reserve(ctx, nB));
        cudaStream_t S3 = ctx->side[3];
        cudaEvent_t evTree = ctx->sideEv[8];
        cub::DoubleBuffer<unsigned long long> dk(ctx->bpKeys.p, ctx->bpKeysAlt.p);
        ctx->hScalars[0] = 0;
        ctx->hScalars[1] = 0;
        DevForces F = dev_forces(ctx);
        // the large-large pass on stream s: chunk bounds, counts (and records), offsets
        auto large_large_count = [&](cudaStream_t s) -> int {
            if (nItems > 0)
            {
                k_ll_chunk_init<<<grid_for(nL, 256), 256, 0, s>>>(ctx->llChunkLo.p, ctx->llChunkHi.p, nL);
                LAUNCHED();
                k_ll_chunk_bounds<<<grid_for(nL, 128), 128, 0, s>>>(G, ctx->large.p, ctx->largeSphere.p, nL,
                                                                    ctx->llChunkLo.p, ctx->llChunkHi.p);
                LAUNCHED();
                k_bp_large_large<BP_COUNT><<<grid_for(nItems, 128), 128, 0, s>>>(
                    F, ctx->large.p, ctx->largeSphere.p, ctx->llItems.p, nItems, ctx->llCount.p, nullptr, 0, 0, cnt,
                    nullptr, ctx->llChunkLo.p, ctx->llChunkHi.p, ctx->llRecorded.p, S);
                LAUNCHED();
                size_t bytes = ctx->cubTempSide[0].cap;
                CU(cub::DeviceScan::ExclusiveSum(ctx->cubTempSide[0].p, bytes, ctx->llCount.p, ctx->llOffset.p, nItems,
                                                 s));
                ctx->launches++;
                if (!deviceCounts)
                {
                    k_total<<<1, 1, 0, s>>>(ctx->llOffset.p, ctx->llCount.p, nItems, ctx->hScalars + 1);
                    LAUNCHED();
                }
            }
            return AVBD_OK;
        };
        // keys -> sorted entries -> cell runs -> counted new pairs, on the context stream;
        // the pair set and (waitLists) the large bodies' cell lists are waited for first
        auto counting_pass = [&](bool waitLists) -> int {
            k_bp_keys<<<grid_for(nB, 256), 256, 0, M>>>(B, G, ctx->binned.p, nB, ctx->bpKeys.p);
            LAUNCHED();
            dk = cub::DoubleBuffer<unsigned long long>(ctx->bpKeys.p, ctx->bpKeysAlt.p);
            size_t bytes = 0;
            // grid keys: world (below W) | cell (22 bits) | body (24 bits). The keys are
            // written in the binned list's order (world by world, ascending body index) and the
            // radix sort is stable, so ordering the (world, cell) bits alone leaves every cell's
            // entries in body order: 3 passes for one world instead of 6.
            int gridEnd = 46 + bit_width((unsigned long long)(ctx->W - 1));
            cub::DeviceRadixSort::SortKeys(nullptr, bytes, dk, nB, 24, gridEnd, M);
            CHECK(ensure_temp(ctx, bytes));
            CU(cub::DeviceRadixSort::SortKeys(ctx->cubTemp.p, bytes, dk, nB, 24, gridEnd, M));
            ctx->launches++;
            CU(cudaMemsetAsync(ctx->cellHashKeys.p, 0xFF,
                               sizeof(unsigned long long) * ((size_t)ctx->cellHashMask + 1), M));
            k_bp_hash_runs<<<grid_for(nB, 256), 256, 0, M>>>(dk.Current(), nB, cell_hash(ctx));
            LAUNCHED();
            CHECK(reserve(ctx, ctx->pairRecorded, (size_t)nB * BP_LANES * BP_SLOTS, false));
            CHECK(reserve(ctx, ctx->pairLaneCount, (size_t)nB * BP_LANES, false));
            if (waitLists)
                CU(cudaStreamWaitEvent(M, evLists, 0));
            CU(cudaStreamWaitEvent(M, evPairSet, 0));
            // LBVH mode: the grid pass counts the large-body part only; the tree finds the rest
            k_bp_pairs<BP_COUNT><<<grid_for((long long)nB * BP_LANES, 128), 128, 0, M>>>(
                B, F, G, dk.Current(), nB, cell_hash(ctx), ctx->large.p, ctx->largeLo.p, ctx->largeHi.p,
                ctx->largeSorted, large_hash(ctx), dt, ctx->pairCount.p, nullptr, 0, 0, cnt, ctx->pairRecorded.p,
                ctx->pairLaneCount.p, nullptr, S, lbvh ? (1u << 14) : 0x7FFFu);
            LAUNCHED();
            if (lbvh)
            {
                CU(cudaStreamWaitEvent(M, evTree, 0)); // the tree, built on side[3]
                CHECK(lbvh_count(ctx, dk.Current(), nB, S));
            }
            CHECK(scan_counts(ctx, ctx->pairCount.p, ctx->pairOffset.p, nB, 0));
            ctx->launches++;
            if (!deviceCounts)
            {
                k_total<<<1, 1, 0, M>>>(ctx->pairOffset.p, ctx->pairCount.p, nB, ctx->hScalars);
                LAUNCHED();
            }
            return AVBD_OK;
        };
        // side[0]: pair set, large boxes, large-large pass
        CU(cudaEventRecord(evFork, M));
        CU(cudaStreamWaitEvent(S1, evFork, 0));
        CU(cudaMemsetAsync(ctx->pairSetKeys.p, 0xFF, sizeof(unsigned long long) * slots, S1));
        k_pair_set<<<grid_for(std::max(forces, 1ll), 256), 256, 0, S1>>>(dev_forces(ctx), S, stp);
        LAUNCHED();
        CU(cudaEventRecord(evPairSet, S1));
        if (nL)
        {
            k_bp_large<<<grid_for(nL, 64), 64, 0, S1>>>(B, ctx->large.p, nL, dt, ctx->largeLo.p, ctx->largeHi.p,
                                                        ctx->largeSphere.p);
            LAUNCHED();
        }
        CU(cudaEventRecord(evLarge, S1));
        CHECK(large_large_count(S1));
        CU(cudaEventRecord(evLL, S1));
        // context stream: bounds and grid parameters, then (side[1]) the large cell lists
        // beside the grid entries' sort
        CU(cudaMemsetAsync(ctx->cappedAny.p, 0, sizeof(int), M));
        ctx->largeSorted = ctx->largeKeys.p;
        if (nB)
        {
            k_bp_bounds_init<<<grid_for(8ll * ctx->W, 256), 256, 0, M>>>(ctx->bounds.p, ctx->W);
            LAUNCHED();
            k_bp_bounds<<<std::min(grid_for(nB, 256), 148 * 2), 256, 0, M>>>(B, G, ctx->binned.p, nB, dt);
            LAUNCHED();
            k_bp_params<<<grid_for(ctx->W, 128), 128, 0, M>>>(G, ctx->worldBinned.p);
            LAUNCHED();
            if (nL || lbvh)
                CU(cudaEventRecord(evParams, M));
            if (nL)
            {
                CU(cudaStreamWaitEvent(S2, evParams, 0));
                CU(cudaStreamWaitEvent(S2, evLarge, 0));
                CHECK(large_cell_lists(ctx, nL, S2, ctx->cubTempSide[1]));
                CU(cudaEventRecord(evLists, S2));
            }
            if (lbvh) // the tree needs only the grid parameters and the bodies
            {
                CU(cudaStreamWaitEvent(S3, evParams, 0));
                CHECK(lbvh_build(ctx, nB, S3));
                CU(cudaEventRecord(evTree, S3));
            }
            CHECK(counting_pass(nL > 0));
        }
        CU(cudaStreamWaitEvent(M, evLL, 0)); // join: everything side[0] made
        if (deviceCounts)
        {
            StepState *st = ctx->stepState.p;
            k_bp_commit<<<1, 1, 0, ctx->stream>>>(st, ctx->pairOffset.p, ctx->pairCount.p, nB, ctx->llOffset.p,
                                                  ctx->llCount.p, nItems, ctx->cappedAny.p, cnt,
                                                  (long long)man_capacity(ctx));
            LAUNCHED();
            F = dev_forces(ctx);
            if (nB)
            {
                k_bp_pairs<BP_EMIT_RECORDED><<<grid_for((long long)nB * BP_LANES, 128), 128, 0, ctx->stream>>>(
                    B, F, G, dk.Current(), nB, cell_hash(ctx), ctx->large.p, ctx->largeLo.p, ctx->largeHi.p,
                    ctx->largeSorted, large_hash(ctx), dt, ctx->pairCount.p, ctx->pairOffset.p, 0, 0, cnt,
                    ctx->pairRecorded.p, ctx->pairLaneCount.p, st, S);
                LAUNCHED();
            }
            if (nItems > 0)
            {
                k_bp_large_large<BP_EMIT_RECORDED><<<grid_for(nItems, 128), 128, 0, ctx->stream>>>(
                    F, ctx->large.p, ctx->largeSphere.p, ctx->llItems.p, nItems, ctx->llCount.p, ctx->llOffset.p, 0, 0,
                    cnt, st, ctx->llChunkLo.p, ctx->llChunkHi.p, ctx->llRecorded.p, S);
                LAUNCHED();
            }
            return AVBD_OK;
        }
        CU(cudaMemcpyAsync(ctx->hCapped, ctx->cappedAny.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        CU(cudaMemcpyAsync(ctx->hCounters, cnt, sizeof(StepCounters), cudaMemcpyDeviceToHost, ctx->stream));
        CU(cudaStreamSynchronize(ctx->stream));
        CHECK(nonfinite_checked(ctx));
        if (nB && *ctx->hCapped)
        {
            // rare path: rescale the capped worlds' cells exactly as the reference does, recount
            CU(cudaMemcpyAsync(ctx->hGrid, ctx->grid.p, sizeof(GridParams) * ctx->W, cudaMemcpyDeviceToHost,
                               ctx->stream));
            CU(cudaStreamSynchronize(ctx->stream));
            for (int w = 0; w < ctx->W; ++w)
                if (ctx->hGrid[w].capped)
                    host_grid_cap(ctx->hGrid[w]);
            CU(cudaMemcpyAsync(ctx->grid.p, ctx->hGrid, sizeof(GridParams) * ctx->W, cudaMemcpyHostToDevice,
                               ctx->stream));
            CU(cudaMemsetAsync(cnt, 0, sizeof(StepCounters), ctx->stream));
            // the recount runs on the context stream alone (every side stream has joined)
            if (nL)
                CHECK(large_cell_lists(ctx, nL, M, ctx->cubTempSide[1]));
            CHECK(counting_pass(false));
            CHECK(large_large_count(M));
            CU(cudaMemcpyAsync(ctx->hCounters, cnt, sizeof(StepCounters), cudaMemcpyDeviceToHost, ctx->stream));
            CU(cudaStreamSynchronize(ctx->stream));
            ctx->stats.grid_rescaled = 1;
        }
        if (ctx->hCounters->error)
            return fail(ctx, AVBD_ERR_CAPACITY, "broadphase grid exceeds the cell cap");
        P1 = ctx->hScalars[0];
        P2 = ctx->hScalars[1];
        if (P1 + P2 > 0)
            CHECK(reserve_manifolds(ctx, ctx->man[ctx->cur], (size_t)(M0 + P1 + P2), (size_t)M0));
        F = dev_forces(ctx);
        if (P1 > 0)
        {
            // the pairs each entry recorded while counting; entries that found more search again
            k_bp_pairs<BP_EMIT_RECORDED><<<grid_for((long long)nB * BP_LANES, 128), 128, 0, ctx->stream>>>(
                B, F, G, dk.Current(), nB, cell_hash(ctx), ctx->large.p, ctx->largeLo.p, ctx->largeHi.p,
                ctx->largeSorted, large_hash(ctx), dt, ctx->pairCount.p, ctx->pairOffset.p, M0,
                (unsigned long long)ctx->nextSeq, cnt, ctx->pairRecorded.p, ctx->pairLaneCount.p, nullptr, S);
            LAUNCHED();
        }
        if (P2 > 0)
        {
            k_bp_large_large<BP_EMIT_RECORDED><<<grid_for(nItems, 128), 128, 0, ctx->stream>>>(
                F, ctx->large.p, ctx->largeSphere.p, ctx->llItems.p, nItems, ctx->llCount.p, ctx->llOffset.p,
                (int)(M0 + P1), (unsigned long long)(ctx->nextSeq + P1), cnt, nullptr, ctx->llChunkLo.p,
                ctx->llChunkHi.p, ctx->llRecorded.p, S);
            LAUNCHED();
        }
    }
    ctx->stats.manifolds_created = P1 + P2;
    ctx->nMan = (int)(M0 + P1 + P2);
    ctx->nextSeq += P1 + P2;
    return AVBD_OK;
}

// Force initialisation of a device-resident step: the launches cover the manifold
// capacity, the live count comes from the step state, and the compaction records the
// surviving count there. Joints need no compaction here: a step starts only when none is
// broken (k_step_begin), and a joint breaks only in the iterations.
// Manifold::initialize of the manifolds that existed before a device step needs nothing
// from the step's broadphase: it runs on side[2] beside it, reading the live buffer and
// writing the updated records into the other one, so a step that stops at its commit leaves
// the live buffer as it was. init_forces_device joins it, initialises the new pairs the same
// way and compacts the kept manifolds back into the live buffer.
int init_old_manifolds(AvbdContext *ctx)
{
    const int M = (int)man_capacity(ctx), J = ctx->nJoint;
    const int need = std::max(std::max(M, J), 1);
    CHECK(reserve(ctx, ctx->keep, (size_t)need, false));
    CHECK(reserve(ctx, ctx->keepIdx, (size_t)need * 2, false));
    if (!M)
        return AVBD_OK;
    cudaStream_t s = ctx->side[2];
    CU(cudaEventRecord(ctx->sideEv[6], ctx->stream));
    CU(cudaStreamWaitEvent(s, ctx->sideEv[6], 0));
    DevBodies B = dev_bodies(ctx);
    Params P = dev_params(ctx->params);
    DevManifolds Md = dev_man(ctx->man[ctx->cur]), Mo = dev_man(ctx->man[ctx->cur ^ 1]);
    int *orphans = &ctx->counters.p->orphans;
    if (ctx->hasShapes)
        k_manifold_init<true><<<grid_for(M, 128), 128, 0, s>>>(B, Md, M, P, ctx->keep.p, ctx->stepState.p,
                                                               ExternalContacts(), orphans, Mo, INIT_OLD);
    else
        k_manifold_init<false><<<grid_for(M, 128), 128, 0, s>>>(B, Md, M, P, ctx->keep.p, ctx->stepState.p,
                                                                ExternalContacts(), orphans, Mo, INIT_OLD);
    LAUNCHED();
    CU(cudaEventRecord(ctx->sideEv[7], s));
    return AVBD_OK;
}

int init_forces_device(AvbdContext *ctx)
{
    DevBodies B = dev_bodies(ctx);
    Params P = dev_params(ctx->params);
    StepState *st = ctx->stepState.p;
    const int M = (int)man_capacity(ctx), J = ctx->nJoint;
    const int need = std::max(std::max(M, J), 1);
    int *idx = ctx->keepIdx.p;
    int *cnt32 = ctx->keepIdx.p + need;
    if (M)
    {
        DevManifolds Md = dev_man(ctx->man[ctx->cur]), Mo = dev_man(ctx->man[ctx->cur ^ 1]);
        int *orphans = &ctx->counters.p->orphans;
        CU(cudaStreamWaitEvent(ctx->stream, ctx->sideEv[7], 0)); // the manifolds from before the step
        if (ctx->hasShapes)
            k_manifold_init<true><<<grid_for(M, 128), 128, 0, ctx->stream>>>(
                B, Md, M, P, ctx->keep.p, st, ExternalContacts(), orphans, Mo, INIT_NEW);
        else
            k_manifold_init<false><<<grid_for(M, 128), 128, 0, ctx->stream>>>(
                B, Md, M, P, ctx->keep.p, st, ExternalContacts(), orphans, Mo, INIT_NEW);
        LAUNCHED();
        k_u8_to_int<<<grid_for(M, 256), 256, 0, ctx->stream>>>(ctx->keep.p, cnt32, M, st);
        LAUNCHED();
        CHECK(scan_counts(ctx, cnt32, idx, M, 0));
        ctx->launches++;
        // back into the live buffer: no swap
        k_manifold_compact<<<grid_for((long long)M * COMPACT_LANES, 128), 128, 0, ctx->stream>>>(
            Mo, Md, M, ctx->keep.p, idx, st, false);
        LAUNCHED();
    }
    if (J)
    {
        DevForces F = dev_forces(ctx);
        k_joint_init<<<grid_for(J, 128), 128, 0, ctx->stream>>>(B, F, P, ctx->keep.p, st, &ctx->counters.p->orphans);
        LAUNCHED();
    }
    return AVBD_OK;
}

ExternalContacts external_contacts(AvbdContext *ctx)
{
    ExternalContacts E;
    if (ctx->external && ctx->extKeyCount > 0)
    {
        E.count = ctx->extKeyCount;
        E.keys = ctx->extKeys.p;
        E.entry = ctx->extEntry.p;
        E.num = ctx->extNum.p;
        E.basis = ctx->extBasis.p;
        E.contact = ctx->extContact.p;
    }
    return E;
}

// broadphaseExternalPairs (solver.cpp:579-626) for the step avbd_step_external issues: the
// device tests each given pair's bounding spheres and existing forces; the host walks the
// pairs, then the contact entries, in the caller's order (a pair made earlier in the list
// constrains a later duplicate) and the kept ones become new manifolds in that order.
int external_broadphase(AvbdContext *ctx)
{
    const int np = (int)ctx->hExtPairs.size(), ne = (int)ctx->hExtEntryPairs.size();
    const int total = np + ne;
    StepCounters c{};
    std::vector<int2> made;
    if (total > 0)
    {
        std::vector<int2> all(ctx->hExtPairs);
        all.insert(all.end(), ctx->hExtEntryPairs.begin(), ctx->hExtEntryPairs.end());
        CHECK(reserve(ctx, ctx->extPairs, (size_t)total, false));
        CHECK(reserve(ctx, ctx->extFlags, (size_t)total, false));
        CU(cudaMemcpyAsync(ctx->extPairs.p, all.data(), sizeof(int2) * total, cudaMemcpyHostToDevice, ctx->stream));
        DevBodies B = dev_bodies(ctx);
        DevForces F = dev_forces(ctx);
        if (np)
        {
            k_external_classify<<<grid_for(np, 128), 128, 0, ctx->stream>>>(B, F, ctx->extPairs.p, np, 1,
                                                                             ctx->extFlags.p);
            LAUNCHED();
        }
        if (ne)
        {
            k_external_classify<<<grid_for(ne, 128), 128, 0, ctx->stream>>>(B, F, ctx->extPairs.p + np, ne, 0,
                                                                             ctx->extFlags.p + np);
            LAUNCHED();
        }
        std::vector<unsigned char> flags((size_t)total);
        CU(cudaMemcpyAsync(flags.data(), ctx->extFlags.p, (size_t)total, cudaMemcpyDeviceToHost, ctx->stream));
        CU(cudaStreamSynchronize(ctx->stream));
        CHECK(nonfinite_checked(ctx));
        std::vector<unsigned long long> linked; // unordered pairs given a manifold in this pass
        auto key = [](int2 p) {
            unsigned lo = (unsigned)std::min(p.x, p.y), hi = (unsigned)std::max(p.x, p.y);
            return ((unsigned long long)lo << 32) | hi;
        };
        auto made_already = [&](unsigned long long k) {
            return std::find(linked.begin(), linked.end(), k) != linked.end();
        };
        for (int k = 0; k < total; ++k)
        {
            c.pairChecks++;
            if (!(flags[k] & 1))
                continue;
            c.sphereHits++;
            unsigned long long pk = key(all[k]);
            if ((flags[k] & 2) || made_already(pk))
            {
                c.constrainedHits++;
                continue;
            }
            made.push_back(all[k]);
            linked.push_back(pk);
        }
    }
    const int M0 = ctx->nMan, P = (int)made.size();
    if (P)
    {
        CHECK(reserve_manifolds(ctx, ctx->man[ctx->cur], (size_t)(M0 + P), (size_t)M0));
        CHECK(reserve(ctx, ctx->extPairs, (size_t)P, false));
        CU(cudaMemcpyAsync(ctx->extPairs.p, made.data(), sizeof(int2) * P, cudaMemcpyHostToDevice, ctx->stream));
        k_external_emit<<<grid_for(P, 128), 128, 0, ctx->stream>>>(dev_man(ctx->man[ctx->cur]), ctx->extPairs.p, P, M0,
                                                                   (unsigned long long)ctx->nextSeq);
        LAUNCHED();
    }
    // the step's counters, where the synchronous step reads them
    CU(cudaMemcpyAsync(ctx->counters.p, &c, sizeof(StepCounters), cudaMemcpyHostToDevice, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream)); // c and made live on this stack frame
    ctx->stats.manifolds_created = P;
    ctx->nMan = M0 + P;
    ctx->nextSeq += P;
    return AVBD_OK;
}

int init_forces(AvbdContext *ctx)
{
    DevBodies B = dev_bodies(ctx);
    Params P = dev_params(ctx->params);
    int M = ctx->nMan, J = ctx->nJoint;
    int need = std::max(M, J);
    CHECK(reserve(ctx, ctx->keep, (size_t)std::max(need, 1), false));
    CHECK(reserve(ctx, ctx->keepIdx, (size_t)std::max(need, 1) * 2, false));
    long long newM = 0, newJ = J;
    int *idx = ctx->keepIdx.p;
    int *cnt32 = ctx->keepIdx.p + std::max(need, 1);
    if (M)
    {
        DevManifolds Md = dev_man(ctx->man[ctx->cur]);
        const ExternalContacts E = external_contacts(ctx);
        if (ctx->hasShapes)
            k_manifold_init<true><<<grid_for(M, 128), 128, 0, ctx->stream>>>(B, Md, M, P, ctx->keep.p, nullptr, E,
                                                                            &ctx->counters.p->orphans);
        else
            k_manifold_init<false><<<grid_for(M, 128), 128, 0, ctx->stream>>>(B, Md, M, P, ctx->keep.p, nullptr, E,
                                                                             &ctx->counters.p->orphans);
        LAUNCHED();
        k_u8_to_int<<<grid_for(M, 256), 256, 0, ctx->stream>>>(ctx->keep.p, cnt32, M);
        LAUNCHED();
        CHECK(scan_counts(ctx, cnt32, idx, M, 0));
        ctx->launches++;
        k_total<<<1, 1, 0, ctx->stream>>>(idx, cnt32, M, ctx->hScalars);
        LAUNCHED();
        CU(cudaStreamSynchronize(ctx->stream));
        newM = ctx->hScalars[0];
        ManBuf &dst = ctx->man[ctx->cur ^ 1];
        CHECK(reserve_manifolds(ctx, dst, (size_t)std::max<long long>(newM, 1), 0));
        k_manifold_compact<<<grid_for((long long)M * COMPACT_LANES, 128), 128, 0, ctx->stream>>>(Md, dev_man(dst), M, ctx->keep.p, idx);
        LAUNCHED();
        ctx->cur ^= 1;
        ctx->nMan = (int)newM;
    }
    if (J)
    {
        DevForces F = dev_forces(ctx);
        k_joint_init<<<grid_for(J, 128), 128, 0, ctx->stream>>>(B, F, P, ctx->keep.p, nullptr,
                                                                 &ctx->counters.p->orphans);
        LAUNCHED();
        k_u8_to_int<<<grid_for(J, 256), 256, 0, ctx->stream>>>(ctx->keep.p, cnt32, J);
        LAUNCHED();
        CHECK(scan_counts(ctx, cnt32, idx, J, 0));
        ctx->launches++;
        k_total<<<1, 1, 0, ctx->stream>>>(idx, cnt32, J, ctx->hScalars + 1);
        LAUNCHED();
        CU(cudaStreamSynchronize(ctx->stream));
        newJ = ctx->hScalars[1];
        if (newJ != J)
        {
            int o = ctx->jcur ^ 1;
            CHECK(reserve(ctx, ctx->jointAB[o], (size_t)std::max<long long>(newJ, 1), false));
            CHECK(reserve(ctx, ctx->jointSeq[o], (size_t)std::max<long long>(newJ, 1), false));
            CHECK(reserve(ctx, ctx->joint[o], 8 * (size_t)std::max<long long>(newJ, 1), false));
            k_joint_compact<<<grid_for(J, 128), 128, 0, ctx->stream>>>(
                J, ctx->keep.p, idx, ctx->jointAB[ctx->jcur].p, ctx->jointSeq[ctx->jcur].p, ctx->joint[ctx->jcur].p,
                ctx->jointAB[o].p, ctx->jointSeq[o].p, ctx->joint[o].p);
            LAUNCHED();
            ctx->jcur = o;
            ctx->nJoint = (int)newJ;
        }
    }
    return AVBD_OK;
}

int colour_readback(AvbdContext *ctx);

// `deviceCounts`: the colouring summary and colour ranges stay on the device (the
// single-launch iteration kernel reads them there); errors go to the step state. Greedy
// mode (the default) colours in one dataflow launch (k_colour_greedy); hashed priorities
// run Jones-Plassmann rounds (k_colour_all) and sort (colour, body) keys.
int colour_bodies(AvbdContext *ctx, bool deviceCounts = false)
{
    int n = ctx->n;
    DevBodies B = dev_bodies(ctx);
    DevForces F = dev_forces(ctx);
    CHECK(reserve(ctx, ctx->colourState, n, false));
    CHECK(reserve(ctx, ctx->colour, n, false));
    CHECK(reserve(ctx, ctx->solveList, n, false));
    CHECK(reserve(ctx, ctx->solveEntry, n, false));
    CHECK(reserve(ctx, ctx->colKeys, n, false));
    CHECK(reserve(ctx, ctx->colKeysAlt, n, false));
    CHECK(reserve(ctx, ctx->colourStart, 257, false));
    CHECK(reserve(ctx, ctx->colourCtl, 1, false));
    if (n == 0 && !deviceCounts)
    {
        ctx->nColours = ctx->nSolve = 0;
        ctx->hColourStart.assign(1, 0);
        return AVBD_OK;
    }
    CU(cudaMemsetAsync(ctx->colourCtl.p, 0, sizeof(ColourControl), ctx->stream));
    int blocks = std::min(grid_for(std::max(n, 1), 256), ctx->colourBlocks);
    int mode = ctx->colourMode;
    unsigned spinLimit = ctx->waitColour ? ctx->waitColour : BARRIER_SPIN_LIMIT;
    StepState *st = deviceCounts ? ctx->stepState.p : nullptr;
    if (mode == AVBD_COLOUR_GREEDY)
    {
        // one cooperative launch: colours, ranges, solve list and entries, row bits
        const unsigned long long *oldFlow = ctx->colourFlow.p;
        CHECK(reserve(ctx, ctx->colourFlow, std::max(n, 1), false));
        if (ctx->colourFlow.p != oldFlow) // fresh memory: no epoch may match by accident
            CU(cudaMemsetAsync(ctx->colourFlow.p, 0, sizeof(unsigned long long) * ctx->colourFlow.cap, ctx->stream));
        int fb = std::min(grid_for(std::max(n, 1), COLOUR_FLOW_BLOCK), ctx->colourFlowBlocks);
        CHECK(reserve(ctx, ctx->colourBlockCounts, (size_t)256 * fb, false));
        unsigned epoch = ++ctx->colourEpoch;
        if (epoch == 0) // wrapped: clear every stored epoch and start again
        {
            CU(cudaMemsetAsync(ctx->colourFlow.p, 0, sizeof(unsigned long long) * ctx->colourFlow.cap, ctx->stream));
            epoch = ctx->colourEpoch = 1;
        }
        DevForces Fr = dev_forces(ctx);
        void *fargs[] = {&B, &Fr, &n, &ctx->colourFlow.p, &epoch, &ctx->colour.p, &ctx->colourCtl.p,
                         &ctx->counters.p, &spinLimit, &ctx->colourBlockCounts.p, &ctx->colourStart.p,
                         &ctx->solveList.p, &ctx->solveEntry.p, &ctx->rowStart.p, &st};
        CU(cudaLaunchCooperativeKernel((void *)k_colour_greedy, fb, COLOUR_FLOW_BLOCK, fargs, 0, ctx->stream));
        LAUNCHED();
        if (deviceCounts)
            return AVBD_OK;
        return colour_readback(ctx);
    }
    void *args[] = {&B, &F, &n, &mode, &ctx->colourState.p, &ctx->colourCtl.p, &ctx->counters.p, &spinLimit, &st};
    CU(cudaLaunchCooperativeKernel((void *)k_colour_all, blocks, 256, args, 0, ctx->stream));
    LAUNCHED();
    k_colour_keys<<<grid_for(n, 256), 256, 0, ctx->stream>>>(ctx->colourState.p, n, ctx->colour.p, ctx->colKeys.p);
    LAUNCHED();
    cub::DoubleBuffer<unsigned> dk(ctx->colKeys.p, ctx->colKeysAlt.p);
    size_t bytes = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, bytes, dk, n, 0, 32, ctx->stream);
    CHECK(ensure_temp(ctx, bytes));
    CU(cub::DeviceRadixSort::SortKeys(ctx->cubTemp.p, bytes, dk, n, 0, 32, ctx->stream));
    ctx->launches++;
    // colour ranges for up to 256 colours are written from the sorted keys; the host reads
    // them together with the colouring summary in one copy
    CU(cudaMemsetAsync(ctx->colourStart.p, 0, sizeof(int) * 257, ctx->stream));
    if (deviceCounts)
    {
        k_solve_list_all<<<grid_for(std::max(n, 1), 256), 256, 0, ctx->stream>>>(
            dk.Current(), n, ctx->solveList.p, ctx->colourStart.p, ctx->colourCtl.p, ctx->rowStart.p,
            ctx->solveEntry.p, ctx->colour.p, ctx->rows.p, st, ctx->counters.p);
        LAUNCHED();
        return AVBD_OK;
    }
    k_solve_list_all<<<grid_for(n, 256), 256, 0, ctx->stream>>>(dk.Current(), n, ctx->solveList.p, ctx->colourStart.p,
                                                                 ctx->colourCtl.p, ctx->rowStart.p,
                                                                 ctx->solveEntry.p, ctx->colour.p, ctx->rows.p);
    LAUNCHED();
    return colour_readback(ctx);
}

// The synchronous step reads the colouring's summary and colour ranges on the host.
int colour_readback(AvbdContext *ctx)
{
    k_colour_count<<<1, 1, 0, ctx->stream>>>(ctx->colourCtl.p, nullptr, ctx->hColourSummary);
    LAUNCHED();
    CU(cudaMemcpyAsync(ctx->hColourStarts, ctx->colourStart.p, sizeof(int) * 257, cudaMemcpyDeviceToHost,
                       ctx->stream));
    CU(cudaMemcpyAsync(ctx->hCounters, ctx->counters.p, sizeof(StepCounters), cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    if (*ctx->hIterError)
        return fail(ctx, AVBD_ERR_STATE, "iteration kernel wait expired (a grid barrier or a partner body's iteration count)");
    const int *sum = ctx->hColourSummary; // vertices, rounds, maxColour, error
    if (sum[3])
        return fail(ctx, AVBD_ERR_STATE, "colouring did not finish (barrier wait expired or round cap reached)");
    if (ctx->hCounters->error == DERR_TOO_MANY_COLOURS)
        return fail(ctx, AVBD_ERR_CAPACITY, "constraint graph needs more than 256 colours");
    int nVert = sum[0];
    int C = nVert > 0 ? sum[2] + 1 : 0;
    ctx->nColours = C;
    ctx->nSolve = nVert;
    ctx->stats.colour_rounds = sum[1];
    ctx->hColourStart.assign(ctx->hColourStarts, ctx->hColourStarts + C + 1);
    return AVBD_OK;
}

// recording hooks of the adjoint (avbd_adjoint.cuh)
int rec_step_begin(AvbdContext *ctx);
int rec_prepared(AvbdContext *ctx);
int rec_iteration(AvbdContext *ctx, int it);
int rec_tape(AvbdContext *ctx, IterTape *tape);
void adjoint_release(AvbdContext *ctx);
void adjoint_invalidate(AvbdContext *ctx); // the world changed: no backward for the last forward

// Every iteration in one cooperative launch (k_iterations), the contacts' dual updates
// fused into the next iteration's rows. A taped step (the adjoint's forward) passes its
// per-iteration records, which the kernel fills as each body and contact finishes an
// iteration.
int iterate_persistent(AvbdContext *ctx, bool deviceCounts = false, IterTape tape = IterTape())
{
    DevBodies B = dev_bodies(ctx);
    DevForces F = dev_forces(ctx);
    Params P = dev_params(ctx->params);
    CHECK(reserve(ctx, ctx->iterSync, 1, false));
    CU(cudaMemsetAsync(ctx->iterSync.p, 0, sizeof(IterSync), ctx->stream));
    int nColours = ctx->nColours, iterations = ctx->params.iterations;
    const int4 *entries = ctx->solveEntry.p;
    const int *colourStart = ctx->colourStart.p;
    IterSync *sync = ctx->iterSync.p;
    // per-body completed iterations, from zero in every launch
    CHECK(reserve(ctx, ctx->iterDone, std::max(ctx->n, 1), false));
    CU(cudaMemsetAsync(ctx->iterDone.p, 0, sizeof(int) * (size_t)ctx->n, ctx->stream));
    int *done = ctx->iterDone.p;
    unsigned spinLimit = ctx->waitIteration ? ctx->waitIteration : ITER_SPIN_LIMIT;
    const StepState *st = deviceCounts ? ctx->stepState.p : nullptr;
    const int *orphans = &ctx->counters.p->orphans;
    void *args[] = {&B, &F, &P, &entries, &colourStart, &nColours, &iterations, &sync, &done, &spinLimit, &st,
                    &orphans, &tape};
    {
        PhaseScope ps(ctx, AVBD_PHASE_PRIMAL);
        // worlds with round bodies run the instance that evaluates their contact offsets
        // (a taped step, boxes only, runs the instance that fills its records)
        void *kernel = ctx->hasShapes ? (void *)k_iterations<ITER_G, ITER_BLOCK, ITER_SUB, true>
                       : tape.pose    ? (void *)k_iterations<ITER_G, ITER_BLOCK, ITER_SUB, false, true>
                                      : (void *)k_iterations<ITER_G, ITER_BLOCK, ITER_SUB, false>;
        CU(cudaLaunchCooperativeKernel(kernel, ctx->iterBlocks, ITER_BLOCK, args,
                                       sizeof(PrimalShared<ITER_G, ITER_BLOCK>), ctx->stream));
        LAUNCHED();
    }
    if (!deviceCounts) // device-resident steps hand the error to the step state (k_step_end)
        CU(cudaMemcpyAsync(ctx->hIterError, &ctx->iterSync.p->error, sizeof(int), cudaMemcpyDeviceToHost,
                           ctx->stream));
    return AVBD_OK;
}

int iterate(AvbdContext *ctx)
{
    if (ctx->iterationMode == AVBD_ITERATIONS_PERSISTENT && ctx->iterBlocks > 0 && ctx->params.iterations > 0 &&
        ctx->nSolve > 0)
    {
        IterTape tape;
        if (ctx->recording)
            CHECK(rec_tape(ctx, &tape));
        return iterate_persistent(ctx, false, tape);
    }
    DevBodies B = dev_bodies(ctx);
    DevForces F = dev_forces(ctx);
    Params P = dev_params(ctx->params);
    // worlds with round bodies: the one instance that evaluates their contact offsets
    const PrimalVariant &pv = ctx->hasShapes ? kRoundPrimal : kPrimalVariants[ctx->primalVariant];
    const int GPB = PRIMAL_BLOCK / pv.group;
    for (int it = 0; it < ctx->params.iterations; ++it)
    {
        if (ctx->recording)
            CHECK(rec_iteration(ctx, it));
        for (int c = 0; c < ctx->nColours; ++c)
        {
            int first = ctx->hColourStart[c];
            int count = ctx->hColourStart[c + 1] - first;
            if (count <= 0)
                continue;
            PhaseScope ps(ctx, AVBD_PHASE_PRIMAL);
            pv.kernel<<<grid_for(count, GPB), PRIMAL_BLOCK, 0, ctx->stream>>>(B, F, P, ctx->solveEntry.p, first,
                                                                               count);
            LAUNCHED();
        }
        PhaseScope ps(ctx, AVBD_PHASE_DUAL);
        if (ctx->nMan)
        {
            if (ctx->hasShapes)
                k_dual_contacts<true><<<grid_for(8ll * ctx->nMan, 256), 256, 0, ctx->stream>>>(B, F.man, ctx->nMan, P);
            else
                k_dual_contacts<false><<<grid_for(8ll * ctx->nMan, 256), 256, 0, ctx->stream>>>(B, F.man, ctx->nMan, P);
            LAUNCHED();
        }
        if (ctx->nJoint)
        {
            k_dual_joints<<<grid_for(ctx->nJoint, 128), 128, 0, ctx->stream>>>(B, F, P);
            LAUNCHED();
        }
    }
    if (ctx->recording)
        CHECK(rec_iteration(ctx, ctx->params.iterations));
    return AVBD_OK;
}

int step_once(AvbdContext *ctx)
{
    // refuse non-finite body state before anything changes, like a device-resident step
    CU(cudaMemsetAsync(ctx->stepFlags.p, 0, sizeof(int), ctx->stream));
    k_step_begin<<<grid_for(std::max(ctx->n, 1), 256), 256, 0, ctx->stream>>>(dev_bodies(ctx), nullptr, 0, nullptr,
                                                                               ctx->stepFlags.p);
    LAUNCHED();
    CU(cudaMemcpyAsync(ctx->hStepFlags, ctx->stepFlags.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    ctx->flagsPending = true; // read by the broadphase at its wait for the pair counts
    if (ctx->recording)
    {
        int rc = rec_step_begin(ctx);
        if (rc != AVBD_OK)
        {
            ctx->flagsPending = false;
            return rc;
        }
    }
    CU(cudaMemsetAsync(ctx->counters.p, 0, sizeof(StepCounters), ctx->stream));
    ctx->stats.grid_rescaled = 0;
    {
        PhaseScope ps(ctx, AVBD_PHASE_BROADPHASE);
        int rc = ctx->external ? external_broadphase(ctx) : broadphase(ctx);
        if (rc == AVBD_OK && ctx->flagsPending) // a broadphase that never waited (fewer than two bodies)
        {
            CU(cudaStreamSynchronize(ctx->stream));
            rc = nonfinite_checked(ctx);
        }
        ctx->flagsPending = false;
        CHECK(rc);
    }
    {
        PhaseScope ps(ctx, AVBD_PHASE_FORCE_INIT);
        CHECK(init_forces(ctx));
    }
    {
        PhaseScope ps(ctx, AVBD_PHASE_ADJACENCY);
        CHECK(build_adjacency(ctx));
    }
    DevBodies B = dev_bodies(ctx);
    Params P = dev_params(ctx->params);
    if (ctx->n)
    {
        PhaseScope ps(ctx, AVBD_PHASE_BODY_INIT);
        k_warm_start<<<grid_for(ctx->n, 256), 256, 0, ctx->stream>>>(B, ctx->adjStart.p, P);
        LAUNCHED();
    }
    {
        PhaseScope ps(ctx, AVBD_PHASE_COLOURING);
        CHECK(colour_bodies(ctx));
    }
    if (ctx->recording)
        CHECK(rec_prepared(ctx));
    CHECK(iterate(ctx));
    if (ctx->n)
    {
        PhaseScope ps(ctx, AVBD_PHASE_VELOCITY);
        k_finish<<<grid_for(ctx->n, 256), 256, 0, ctx->stream>>>(B, P);
        LAUNCHED();
        if (ctx->hasSpheres)
        {
            k_rolling_friction<<<grid_for(ctx->n, 128), 128, 0, ctx->stream>>>(B, dev_forces(ctx), ctx->adjStart.p);
            LAUNCHED();
        }
    }
    ctx->stats.body_count = ctx->n;
    ctx->stats.manifold_count = ctx->nMan;
    ctx->stats.joint_count = ctx->nJoint;
    ctx->stats.spring_count = ctx->nSpring;
    ctx->stats.solved_bodies = ctx->nSolve;
    ctx->stats.colours = ctx->nColours;
    ctx->stats.pair_checks = (int64_t)ctx->hCounters->pairChecks;
    ctx->stats.sphere_hits = (int64_t)ctx->hCounters->sphereHits;
    ctx->stats.constrained_hits = (int64_t)ctx->hCounters->constrainedHits;
    if (ctx->profiling)
        ctx->stepsProfiled++;
    return AVBD_OK;
}

// ---------------------------------------------------------------------------
// Device-resident steps
// ---------------------------------------------------------------------------

// The host's counts become the device state's (no step is pending).
int push_state(AvbdContext *ctx)
{
    k_state_set<<<1, 1, 0, ctx->stream>>>(ctx->stepState.p, ctx->nMan, (unsigned long long)ctx->nextSeq);
    LAUNCHED();
    ctx->doneAtConfirm = 0;
    ctx->flipsAtConfirm = 0;
    ctx->curAtConfirm = ctx->cur;
    ctx->seqBound = (unsigned long long)ctx->nextSeq;
    ctx->stateDirty = false;
    return AVBD_OK;
}

// Steps that can keep their counts on the device: the grid broadphase, the single-launch
// iterations, not while the differentiable step records.
bool device_step_ok(const AvbdContext *ctx)
{
    return ctx->stepMode == AVBD_STEP_DEVICE &&
           (ctx->params.broadphase == AVBD_BROADPHASE_GRID || ctx->params.broadphase == AVBD_BROADPHASE_LBVH) &&
           ctx->iterationMode == AVBD_ITERATIONS_PERSISTENT && ctx->iterBlocks > 0 && !ctx->recording &&
           ctx->params.iterations > 0;
}

// Both manifold buffers with room for the live manifolds and a step's new pairs (grown
// only while no step is pending, when the live count is known).
int device_reserve(AvbdContext *ctx)
{
    size_t live = (size_t)ctx->nMan;
    size_t want = ctx->manifoldSpare > 0 ? live + (size_t)ctx->manifoldSpare
                                         : std::max(2 * live, live + 2 * (size_t)ctx->n) + 1024;
    if (ctx->pendingFast == 0 && man_capacity(ctx) < want)
    {
        CHECK(reserve_manifolds(ctx, ctx->man[ctx->cur], want, live));
        CHECK(reserve_manifolds(ctx, ctx->man[ctx->cur ^ 1], want, 0));
    }
    return AVBD_OK;
}

// One Solver::step with every count on the device: the same kernels as step_once, sized by
// capacity, with k_step_begin / k_bp_commit deciding on the device whether the step can run.
int step_device(AvbdContext *ctx)
{
    // with no step pending the host's counts are current (a settle, a synchronous step, a
    // load or an edit came last): they become the device state's
    if (ctx->stateDirty || ctx->pendingFast == 0)
        CHECK(push_state(ctx));
    CHECK(device_reserve(ctx));
    // this step's new manifolds take sequence numbers below nextSeq + capacity: the bound the
    // incidence keys of this step (and of later pending steps) are sized by
    ctx->seqBound += (unsigned long long)man_capacity(ctx);
    StepState *st = ctx->stepState.p;
    CU(cudaMemsetAsync(ctx->counters.p, 0, sizeof(StepCounters), ctx->stream));
    ctx->stats.grid_rescaled = 0;
    DevBodies B = dev_bodies(ctx);
    Params P = dev_params(ctx->params);
    {
        PhaseScope ps(ctx, AVBD_PHASE_BROADPHASE);
        const int J = ctx->nJoint;
        k_step_begin<<<grid_for(std::max(std::max(ctx->n, J), 1), 256), 256, 0, ctx->stream>>>(
            B, ctx->joint[ctx->jcur].p, J, st, nullptr);
        LAUNCHED();
        CHECK(init_old_manifolds(ctx));
        CHECK(broadphase(ctx, true));
    }
    {
        PhaseScope ps(ctx, AVBD_PHASE_FORCE_INIT);
        CHECK(init_forces_device(ctx));
    }
    {
        PhaseScope ps(ctx, AVBD_PHASE_ADJACENCY);
        CHECK(build_adjacency(ctx, true));
    }
    if (ctx->n)
    {
        PhaseScope ps(ctx, AVBD_PHASE_BODY_INIT);
        k_warm_start<<<grid_for(ctx->n, 256), 256, 0, ctx->stream>>>(B, ctx->adjStart.p, P, st);
        LAUNCHED();
    }
    {
        PhaseScope ps(ctx, AVBD_PHASE_COLOURING);
        CHECK(colour_bodies(ctx, true));
    }
    CHECK(iterate_persistent(ctx, true));
    if (ctx->n)
    {
        PhaseScope ps(ctx, AVBD_PHASE_VELOCITY);
        k_finish<<<grid_for(ctx->n, 256), 256, 0, ctx->stream>>>(B, P, st);
        LAUNCHED();
        if (ctx->hasSpheres)
        {
            k_rolling_friction<<<grid_for(ctx->n, 128), 128, 0, ctx->stream>>>(B, dev_forces(ctx), ctx->adjStart.p,
                                                                               st);
            LAUNCHED();
        }
    }
    k_step_end<<<1, 1, 0, ctx->stream>>>(st, ctx->iterSync.p);
    LAUNCHED();
    CU(cudaMemcpyAsync(ctx->hState, st, sizeof(StepState), cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaMemcpyAsync(ctx->hCounters, ctx->counters.p, sizeof(StepCounters), cudaMemcpyDeviceToHost, ctx->stream));
    // the colour ranges, for host-side users of the last colouring (per-colour launches)
    CU(cudaMemcpyAsync(ctx->hColourStarts, ctx->colourStart.p, sizeof(int) * 257, cudaMemcpyDeviceToHost,
                       ctx->stream));
    ctx->pendingFast++;
    ctx->deviceSteps++;
    if (ctx->profiling)
        ctx->stepsProfiled++;
    return AVBD_OK;
}

// Wait for the device-resident steps issued so far and take their counts. Steps that
// stopped on the device before changing anything (ABORT_JOINTS / GRID / MANIFOLDS, and
// every step issued after one) are redone synchronously by step_once, which compacts the
// broken joints, rescales the grid with the host's cbrtf or grows the buffers; errors
// latch. Afterwards the host's counts are current again.
int settle(AvbdContext *ctx)
{
    if (ctx->pendingFast == 0)
        return AVBD_OK;
    const int pending = ctx->pendingFast;
    ctx->pendingFast = 0;
    CU(cudaStreamSynchronize(ctx->stream));
    const StepState s = *ctx->hState;
    const int done = s.stepsDone - ctx->doneAtConfirm;
    const int flips = s.flips - ctx->flipsAtConfirm;
    ctx->cur = ctx->curAtConfirm ^ (flips & 1);
    ctx->nMan = s.nMan;
    ctx->nextSeq = (long long)s.nextSeq;
    ctx->nColours = s.nColours;
    ctx->nSolve = s.nSolve;
    ctx->doneAtConfirm = s.stepsDone;
    ctx->flipsAtConfirm = s.flips;
    ctx->curAtConfirm = ctx->cur;
    ctx->seqBound = s.nextSeq;
    if (done > 0)
    {
        ctx->hColourStart.assign(ctx->hColourStarts, ctx->hColourStarts + std::min(std::max(ctx->nColours, 0), 256) + 1);
        ctx->stats.body_count = ctx->n;
        ctx->stats.manifold_count = ctx->nMan;
        ctx->stats.joint_count = ctx->nJoint;
        ctx->stats.spring_count = ctx->nSpring;
        ctx->stats.solved_bodies = ctx->nSolve;
        ctx->stats.colours = ctx->nColours;
        ctx->stats.colour_rounds = s.rounds;
        ctx->stats.manifolds_created = s.created;
        ctx->stats.pair_checks = (int64_t)ctx->hCounters->pairChecks;
        ctx->stats.sphere_hits = (int64_t)ctx->hCounters->sphereHits;
        ctx->stats.constrained_hits = (int64_t)ctx->hCounters->constrainedHits;
    }
    if (s.abort == ABORT_NONE)
        return device_step_ok(ctx) ? device_reserve(ctx) : AVBD_OK; // room for the next steps, now
    ctx->stateDirty = true; // the device's stop word is cleared before the next device step
    // A step that stopped after building the per-body force lists (at the colouring or the
    // iterations) left them built for its own manifolds; the next broadphase reads those
    // lists, so rebuild them from the confirmed state.
    CHECK(build_adjacency(ctx));
    if (s.abort == ABORT_ERROR)
    {
        if (s.error == STEP_ERR_ITERATION)
            return fail(ctx, AVBD_ERR_STATE,
                        "iteration kernel wait expired (a grid barrier or a partner body's iteration count)");
        if (s.error == STEP_ERR_COLOURS)
            return fail(ctx, AVBD_ERR_CAPACITY, "constraint graph needs more than 256 colours");
        return fail(ctx, AVBD_ERR_STATE, "colouring did not finish (barrier wait expired or round cap reached)");
    }
    if (s.abort == ABORT_NONFINITE)
        return fail(ctx, AVBD_ERR_STATE,
                    "non-finite body position, orientation or velocity at the start of a step (the step was not run)");
    for (int r = done; r < pending; ++r)
    {
        CHECK(step_once(ctx));
        ctx->redoneSteps++;
    }
    return device_step_ok(ctx) ? device_reserve(ctx) : AVBD_OK;
}

int stage_reserve(AvbdContext *ctx, size_t count)
{
    if (!ctx->stageDone)
        CU(cudaEventCreateWithFlags(&ctx->stageDone, cudaEventDisableTiming));
    CU(cudaEventSynchronize(ctx->stageDone)); // earlier copies out of the staging buffer are done
    if (count <= ctx->hStageCap)
        return AVBD_OK;
    if (ctx->hStage)
    {
        CU(cudaStreamSynchronize(ctx->stream));
        CU(cudaFreeHost(ctx->hStage));
        ctx->hStage = nullptr;
        ctx->hStageCap = 0;
    }
    CU(cudaMallocHost((void **)&ctx->hStage, count * sizeof(float4)));
    ctx->hStageCap = count;
    return AVBD_OK;
}

// Body state fields in the callers' packed layout: per field n entries of `width` floats
// (3, or 4 for orientations), in a device-usable buffer (the device staging buffer, or the
// caller's page-locked array through its mapped address; null: field absent).
struct PackedField
{
    float4 *arr;
    float *buf;
    int width;
    int aligned; // buf is 16-byte aligned: whole float4 accesses
    float w;     // fourth component written for an absent field
};

constexpr int MAX_PACKED = 9;
constexpr int PACK_BLOCK = 256;
struct PackedFields
{
    PackedField f[MAX_PACKED];
    int count;
};

// Each block moves its bodies' contiguous stretch of a field (PACK_BLOCK entries of `width`
// floats) between the packed buffer and shared memory in whole, consecutive accesses,
// float4 when the buffer is aligned, so that a caller's page-locked array crosses the bus
// in full lines. A block's stretch starts at a multiple of 3,072 or 4,096 bytes.
AVBD_DEV void packed_load(const PackedField &f, int i0, int cnt, float *s)
{
    const float *src = f.buf + (size_t)f.width * i0;
    const int total = cnt * f.width;
    if (f.aligned && (total & 3) == 0)
        for (int t = threadIdx.x; t < total / 4; t += blockDim.x)
            reinterpret_cast<float4 *>(s)[t] = reinterpret_cast<const float4 *>(src)[t];
    else
        for (int t = threadIdx.x; t < total; t += blockDim.x)
            s[t] = src[t];
}

AVBD_DEV void packed_store(const PackedField &f, int i0, int cnt, const float *s)
{
    float *dst = f.buf + (size_t)f.width * i0;
    const int total = cnt * f.width;
    if (f.aligned && (total & 3) == 0)
        for (int t = threadIdx.x; t < total / 4; t += blockDim.x)
            reinterpret_cast<float4 *>(dst)[t] = reinterpret_cast<const float4 *>(s)[t];
    else
        for (int t = threadIdx.x; t < total; t += blockDim.x)
            dst[t] = s[t];
}

// Packed caller layout -> the device's float4 arrays (absent fields take (0, 0, 0, w)). Every
// field's stretch is requested before any is used (one shared buffer holds them all), so a
// block keeps all its reads across the bus in flight at once.
__global__ void __launch_bounds__(PACK_BLOCK) k_unpack_state(PackedFields P, int n)
{
    __shared__ __align__(16) float s[MAX_PACKED][PACK_BLOCK * 4];
    const int i0 = blockIdx.x * PACK_BLOCK;
    const int cnt = min(PACK_BLOCK, n - i0);
    const int t = threadIdx.x;
    for (int k = 0; k < P.count; ++k)
        if (P.f[k].buf)
            packed_load(P.f[k], i0, cnt, s[k]);
    __syncthreads();
    if (t >= cnt)
        return;
    for (int k = 0; k < P.count; ++k)
    {
        const PackedField f = P.f[k];
        float4 v = make_float4(0.0f, 0.0f, 0.0f, f.w);
        if (f.buf)
        {
            const float *e = s[k] + f.width * t;
            v = f.width == 4 ? make_float4(e[0], e[1], e[2], e[3]) : make_float4(e[0], e[1], e[2], 0.0f);
        }
        f.arr[i0 + t] = v;
    }
}

// The device's float4 arrays -> the packed caller layout (requested fields only); all
// fields are staged first, then stored together.
__global__ void __launch_bounds__(PACK_BLOCK) k_pack_state(PackedFields P, int n)
{
    __shared__ __align__(16) float s[MAX_PACKED][PACK_BLOCK * 4];
    const int i0 = blockIdx.x * PACK_BLOCK;
    const int cnt = min(PACK_BLOCK, n - i0);
    const int t = threadIdx.x;
    if (t < cnt)
        for (int k = 0; k < P.count; ++k)
        {
            const PackedField f = P.f[k];
            if (!f.buf)
                continue;
            const float4 v = f.arr[i0 + t];
            float *d = s[k] + f.width * t;
            d[0] = v.x;
            d[1] = v.y;
            d[2] = v.z;
            if (f.width == 4)
                d[3] = v.w;
        }
    __syncthreads();
    for (int k = 0; k < P.count; ++k)
        if (P.f[k].buf)
            packed_store(P.f[k], i0, cnt, s[k]);
}

// Host copies between callers' arrays and the pinned staging. (Splitting them over threads
// was measured slower: starting the threads costs more than the copies.)
struct HostCopy
{
    void *dst;
    const void *src;
    size_t bytes;
};

void copy_host(const std::vector<HostCopy> &copies)
{
    for (const HostCopy &c : copies)
        memcpy(c.dst, c.src, c.bytes);
}

// A caller array in page-locked host memory (cudaHostAlloc, cudaHostRegister, a pinned
// torch tensor) that the device can address: the packing kernels read or write it in place,
// over the bus, with no copy call. Null for any other array.
float *host_mapped(const void *p)
{
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess)
    {
        cudaGetLastError();
        return nullptr;
    }
    return a.type == cudaMemoryTypeHost ? (float *)a.devicePointer : nullptr;
}

bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

// Body state from caller arrays: page-locked arrays are read in place by the unpacking
// kernel; any other array is copied into pinned staging and uploaded first.
int write_state(AvbdContext *ctx, const AvbdBodies *b)
{
    int n = b->count;
    const float *src[5] = {b->position3, b->orientation4, b->velocity3, b->angular3,
                           b->prev_velocity3 ? b->prev_velocity3 : b->velocity3};
    DArr<float4> *dst[5] = {&ctx->pos, &ctx->quat, &ctx->vel, &ctx->angvel, &ctx->prevVel};
    const int width[5] = {3, 4, 3, 3, 3};
    PackedFields P{};
    P.count = 5;
    long long floats = 0;
    float *mapped[5] = {};
    for (int f = 0; f < 5; ++f)
    {
        CHECK(reserve(ctx, *dst[f], std::max(n, 1), false));
        mapped[f] = src[f] && n ? host_mapped(src[f]) : nullptr;
        if (src[f] && !mapped[f])
            floats += (long long)width[f] * n;
    }
    if (!n)
        return AVBD_OK;
    CHECK(stage_reserve(ctx, (size_t)(floats + 3) / 4));
    CHECK(reserve(ctx, ctx->stateStage, (size_t)std::max<long long>(floats, 1), false));
    float *st = (float *)ctx->hStage;
    std::vector<HostCopy> copies;
    long long off = 0;
    for (int f = 0; f < 5; ++f)
    {
        float *buf = nullptr;
        if (mapped[f])
            buf = mapped[f];
        else if (src[f])
        {
            copies.push_back({st + off, src[f], sizeof(float) * width[f] * (size_t)n});
            buf = ctx->stateStage.p + off;
            off += (long long)width[f] * n;
        }
        P.f[f] = PackedField{dst[f]->p, buf, width[f], buf ? (int)aligned16(buf) : 0, f == 1 ? 1.0f : 0.0f};
    }
    if (!copies.empty())
    {
        copy_host(copies);
        for (const HostCopy &c : copies)
            CU(cudaMemcpyAsync(ctx->stateStage.p + ((const float *)c.dst - st), c.dst, c.bytes,
                               cudaMemcpyHostToDevice, ctx->stream));
    }
    CU(cudaEventRecord(ctx->stageDone, ctx->stream));
    k_unpack_state<<<grid_for(n, PACK_BLOCK), PACK_BLOCK, 0, ctx->stream>>>(P, n);
    LAUNCHED();
    return AVBD_OK;
}

template <class T>
int upload(AvbdContext *ctx, DArr<T> &a, const T *src, size_t count)
{
    CHECK(reserve(ctx, a, std::max<size_t>(count, 1), false));
    if (count)
        CU(cudaMemcpyAsync(a.p, src, count * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
    return AVBD_OK;
}

int upload_bodies(AvbdContext *ctx, const AvbdBodies *b, bool props)
{
    int n = b->count;
    CHECK(write_state(ctx, b));
    if (props)
    {
        std::vector<float4> tmp(n);
        for (int i = 0; i < n; ++i)
            tmp[i] = make_float4(b->mass[i], b->moment3[3 * i], b->moment3[3 * i + 1], b->moment3[3 * i + 2]);
        CHECK(upload(ctx, ctx->massMoment, tmp.data(), n));
        for (int i = 0; i < n; ++i)
            tmp[i] = make_float4(b->size3[3 * i], b->size3[3 * i + 1], b->size3[3 * i + 2], b->radius[i]);
        CHECK(upload(ctx, ctx->sizeRad, tmp.data(), n));
        CHECK(upload(ctx, ctx->friction, b->friction, n));
        ctx->hasShapes = ctx->hasSpheres = false;
        if (b->shape)
        {
            for (int i = 0; i < n; ++i)
            {
                int t = b->shape[i];
                if (t < AVBD_SHAPE_BOX || t > AVBD_SHAPE_CYLINDER)
                    return fail(ctx, AVBD_ERR_ARGUMENT, "body %d: unknown shape %d", i, t);
                if (t != AVBD_SHAPE_BOX && (!b->shape_radius || !b->half_length))
                    return fail(ctx, AVBD_ERR_ARGUMENT, "round bodies need shape_radius and half_length");
                ctx->hasShapes |= t != AVBD_SHAPE_BOX;
                ctx->hasSpheres |= t == AVBD_SHAPE_SPHERE;
            }
            if (ctx->hasShapes)
            {
                for (int i = 0; i < n; ++i)
                    tmp[i] = make_float4((float)b->shape[i], b->shape_radius ? b->shape_radius[i] : b->radius[i],
                                         b->half_length ? b->half_length[i] : 0.0f, 0.0f);
                CHECK(upload(ctx, ctx->shape, tmp.data(), n));
            }
        }
        for (DArr<float4> *a : {&ctx->initLin, &ctx->initAng, &ctx->inertLin, &ctx->inertAng, &ctx->dqLin, &ctx->dqAng,
                                &ctx->initAngInv, &ctx->inertAngInv})
        {
            CHECK(reserve(ctx, *a, std::max(n, 1), false));
            CU(cudaMemsetAsync(a->p, 0, sizeof(float4) * std::max(n, 1), ctx->stream));
        }
        CU(cudaStreamSynchronize(ctx->stream));
    }
    return AVBD_OK;
}

// Grid classification per world: bodies above the world's 95th-percentile bounding radius
// are "large" (solver.cpp:297-329). Radii never change, so this is fixed per load. Worlds
// with fewer than two bodies take no part in the broadphase (solver.cpp:292-293).
int classify_bodies(AvbdContext *ctx, const float *radius)
{
    const int W = ctx->W;
    ctx->hBinned.clear();
    ctx->hLarge.clear();
    ctx->hLLItems.clear();
    ctx->hWorldLargeStart.assign(1, 0);
    std::vector<float> binnedR(W, 1e-3f);
    std::vector<int> worldBinned(W, 0);
    std::vector<int> bodyWorld(ctx->n);
    for (int w = 0; w < W; ++w)
    {
        int b0 = ctx->hWorldStart[w], b1 = ctx->hWorldStart[w + 1], nw = b1 - b0;
        for (int b = b0; b < b1; ++b)
            bodyWorld[b] = w;
        if (nw >= 2)
        {
            std::vector<float> r(radius + b0, radius + b1);
            size_t pct = std::min<size_t>((size_t)nw - 1, (size_t)nw * 95 / 100);
            std::nth_element(r.begin(), r.begin() + pct, r.end());
            binnedR[w] = r[pct] > 1e-3f ? r[pct] : 1e-3f;
            int l0 = (int)ctx->hLarge.size();
            for (int b = b0; b < b1; ++b)
            {
                if (radius[b] > binnedR[w])
                    ctx->hLarge.push_back(b);
                else
                {
                    ctx->hBinned.push_back(b);
                    worldBinned[w]++;
                }
            }
            int L = (int)ctx->hLarge.size() - l0;
            int chunks = (L + LL_CHUNK - 1) / LL_CHUNK;
            for (int i = 0; i < L; ++i)
                for (int c = 0; c < chunks; ++c)
                    ctx->hLLItems.push_back(make_int4(l0, L, i, c));
        }
        ctx->hWorldLargeStart.push_back((int)ctx->hLarge.size());
    }
    int nB = (int)ctx->hBinned.size(), nL = (int)ctx->hLarge.size(), nI = (int)ctx->hLLItems.size();
    CHECK(upload(ctx, ctx->bodyWorld, bodyWorld.data(), ctx->n));
    CHECK(upload(ctx, ctx->worldStart, ctx->hWorldStart.data(), (size_t)W + 1));
    CHECK(upload(ctx, ctx->worldLargeStart, ctx->hWorldLargeStart.data(), (size_t)W + 1));
    CHECK(upload(ctx, ctx->worldBinned, worldBinned.data(), W));
    {
        std::vector<int> start(W + 1, 0);
        for (int w = 0; w < W; ++w)
            start[w + 1] = start[w] + worldBinned[w];
        CHECK(upload(ctx, ctx->worldBinnedStart, start.data(), start.size()));
    }
    CHECK(upload(ctx, ctx->binnedRadiusW, binnedR.data(), W));
    CHECK(upload(ctx, ctx->binned, ctx->hBinned.data(), nB));
    CHECK(upload(ctx, ctx->large, ctx->hLarge.data(), nL));
    CHECK(upload(ctx, ctx->llItems, ctx->hLLItems.data(), nI));
    CHECK(reserve(ctx, ctx->llCount, std::max(nI, 1), false));
    CHECK(reserve(ctx, ctx->llOffset, std::max(nI, 1), false));
    CHECK(reserve(ctx, ctx->largeLo, std::max(nL, 1), false));
    CHECK(reserve(ctx, ctx->largeHi, std::max(nL, 1), false));
    CHECK(reserve(ctx, ctx->largeSphere, std::max(nL, 1), false));
    CHECK(reserve(ctx, ctx->largeKeys, (size_t)std::max(nL, 1) * LARGE_MAX_CELLS + 1, false));
    CHECK(reserve(ctx, ctx->largeKeysAlt, (size_t)std::max(nL, 1) * LARGE_MAX_CELLS + 1, false));
    CHECK(reserve(ctx, ctx->bpKeys, std::max(nB, 1), false));
    CHECK(reserve(ctx, ctx->bpKeysAlt, std::max(nB, 1), false));
    CHECK(reserve(ctx, ctx->pairCount, std::max(ctx->n, 1), false));
    CHECK(reserve(ctx, ctx->pairOffset, std::max(ctx->n, 1), false));
    CHECK(reserve(ctx, ctx->bounds, 8 * (size_t)W, false));
    CHECK(reserve(ctx, ctx->grid, W, false));
    CHECK(reserve(ctx, ctx->cappedAny, 1, false));
    auto pow2 = [](size_t x) {
        size_t p = 64;
        while (p < x)
            p <<= 1;
        return p;
    };
    size_t ch = pow2(2 * (size_t)nB), lh = pow2(2 * ((size_t)nL * LARGE_MAX_CELLS + W));
    CHECK(reserve(ctx, ctx->cellHashKeys, ch, false));
    CHECK(reserve(ctx, ctx->cellHashVals, ch, false));
    CHECK(reserve(ctx, ctx->largeHashKeys, lh, false));
    CHECK(reserve(ctx, ctx->largeHashVals, lh, false));
    ctx->cellHashMask = (unsigned)(ch - 1);
    ctx->largeHashMask = (unsigned)(lh - 1);
    if (ctx->hGridCap < (size_t)W)
    {
        if (ctx->hGrid)
            CU(cudaFreeHost(ctx->hGrid));
        CU(cudaMallocHost((void **)&ctx->hGrid, sizeof(GridParams) * W));
        ctx->hGridCap = W;
    }
    return AVBD_OK;
}

} // namespace

extern "C"
{

const char *avbd_backend_name(void) { return "CUDA AVBD (sm_100a)"; }

int avbd_create(AvbdContext **out, int32_t device_ordinal, void *cuda_stream)
{
    if (!out)
        return AVBD_ERR_ARGUMENT;
    *out = nullptr;
    AvbdContext *ctx = new AvbdContext();
    ctx->device = device_ordinal;
    cudaError_t e = cudaSetDevice(device_ordinal);
    if (e != cudaSuccess)
    {
        delete ctx;
        return AVBD_ERR_CUDA;
    }
    if (cuda_stream)
        ctx->stream = (cudaStream_t)cuda_stream;
    else
    {
        if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess)
        {
            delete ctx;
            return AVBD_ERR_CUDA;
        }
        ctx->ownStream = true;
    }
    {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device_ordinal;
        if (cudaMemPoolCreate(&ctx->pool, &props) != cudaSuccess)
        {
            avbd_destroy(ctx);
            return AVBD_ERR_CUDA;
        }
        unsigned long long keep = ~0ull; // keep freed blocks for reuse instead of returning them
        cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    if (cudaMallocHost((void **)&ctx->hCounters, sizeof(StepCounters)) != cudaSuccess ||
        cudaMallocHost((void **)&ctx->hScalars, sizeof(long long) * 16) != cudaSuccess ||
        cudaMallocHost((void **)&ctx->hColourSummary, sizeof(int) * 4) != cudaSuccess ||
        cudaMallocHost((void **)&ctx->hCapped, sizeof(int)) != cudaSuccess ||
        cudaMallocHost((void **)&ctx->hColourStarts, sizeof(int) * 257) != cudaSuccess ||
        cudaMallocHost((void **)&ctx->hIterError, sizeof(int)) != cudaSuccess ||
        cudaMallocHost((void **)&ctx->hState, sizeof(StepState)) != cudaSuccess ||
        cudaMallocHost((void **)&ctx->hStepFlags, sizeof(int)) != cudaSuccess ||
        cudaEventCreate(&ctx->evStart) != cudaSuccess || cudaEventCreate(&ctx->evStop) != cudaSuccess)
    {
        avbd_destroy(ctx);
        return AVBD_ERR_CUDA;
    }
    for (cudaStream_t &sd : ctx->side)
        if (cudaStreamCreateWithFlags(&sd, cudaStreamNonBlocking) != cudaSuccess)
        {
            sd = nullptr;
            avbd_destroy(ctx);
            return AVBD_ERR_CUDA;
        }
    for (cudaEvent_t &e : ctx->sideEv)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
        {
            e = nullptr;
            avbd_destroy(ctx);
            return AVBD_ERR_CUDA;
        }
    memset(ctx->hCounters, 0, sizeof(StepCounters));
    memset(ctx->hState, 0, sizeof(StepState));
    *ctx->hIterError = 0;
    {
        int sms = 0, perSm = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_ordinal);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_colour_all, 256, 0);
        ctx->colourBlocks = std::max(1, sms * std::max(1, perSm));
        // the greedy colouring: co-resident, and at most four blocks per SM (every block
        // reads all blocks' colour counts once; more resident warps mean fewer grid-stride
        // batches per warp, which a chain of neighbours crosses one after another)
        int flowSm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&flowSm, k_colour_greedy, COLOUR_FLOW_BLOCK, 0);
        ctx->colourFlowBlocks = std::max(1, sms * std::min(4, std::max(1, flowSm)));
        // the iteration kernel: one block of ITER_BLOCK threads per SM with its shared batch
        int iterSm = 0;
        size_t smem = sizeof(PrimalShared<ITER_G, ITER_BLOCK>);
        int roundSm = 0, tapeSm = 0;
        if (cudaFuncSetAttribute((const void *)k_iterations<ITER_G, ITER_BLOCK, ITER_SUB, false>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) == cudaSuccess &&
            cudaFuncSetAttribute((const void *)k_iterations<ITER_G, ITER_BLOCK, ITER_SUB, true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) == cudaSuccess &&
            cudaFuncSetAttribute((const void *)k_iterations<ITER_G, ITER_BLOCK, ITER_SUB, false, true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) == cudaSuccess &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&tapeSm, k_iterations<ITER_G, ITER_BLOCK, ITER_SUB, false, true>,
                                                          ITER_BLOCK, smem) == cudaSuccess &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&iterSm, k_iterations<ITER_G, ITER_BLOCK, ITER_SUB, false>,
                                                          ITER_BLOCK, smem) == cudaSuccess &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&roundSm, k_iterations<ITER_G, ITER_BLOCK, ITER_SUB, true>,
                                                          ITER_BLOCK, smem) == cudaSuccess)
            ctx->iterBlocks = sms * std::min({iterSm, roundSm, tapeSm});
        cudaGetLastError(); // an unsupported configuration only leaves the per-colour launches
    }
    if (reserve(ctx, ctx->counters, 1, false) || reserve(ctx, ctx->bounds, 8, false) ||
        reserve(ctx, ctx->grid, 1, false) || reserve(ctx, ctx->stepState, 1, false) ||
        reserve(ctx, ctx->stepFlags, 1, false))
    {
        avbd_destroy(ctx);
        return AVBD_ERR_CUDA;
    }
    ctx->params.dt = 1.0f / 60.0f;
    ctx->params.gravity = -10.0f;
    ctx->params.iterations = 10;
    ctx->params.alpha = 0.99f;
    ctx->params.betaLin = 10000.0f;
    ctx->params.betaAng = 100.0f;
    ctx->params.gamma = 0.999f;
    ctx->params.broadphase = AVBD_BROADPHASE_GRID;
    *out = ctx;
    return AVBD_OK;
}

void avbd_destroy(AvbdContext *ctx)
{
    if (!ctx)
        return;
    cudaSetDevice(ctx->device);
    if (ctx->stream)
        cudaStreamSynchronize(ctx->stream);
    for (cudaStream_t sd : ctx->side)
        if (sd)
            cudaStreamSynchronize(sd);
    adjoint_release(ctx);
    for (DArr<float4> *a : {&ctx->pos, &ctx->quat, &ctx->initLin, &ctx->initAng, &ctx->inertLin, &ctx->inertAng,
                            &ctx->dqLin, &ctx->dqAng, &ctx->initAngInv, &ctx->inertAngInv,
                            &ctx->vel, &ctx->angvel, &ctx->prevVel, &ctx->massMoment, &ctx->sizeRad, &ctx->largeLo,
                            &ctx->largeHi, &ctx->largeSphere, &ctx->spring, &ctx->joint[0], &ctx->joint[1]})
        release(*a);
    release(ctx->friction);
    release(ctx->binned);
    release(ctx->large);
    release(ctx->bounds);
    release(ctx->grid);
    release(ctx->bodyWorld);
    release(ctx->worldStart);
    release(ctx->worldLargeStart);
    release(ctx->worldBinned);
    release(ctx->binnedRadiusW);
    release(ctx->llItems);
    release(ctx->cappedAny);
    release(ctx->cellHashKeys);
    release(ctx->cellHashVals);
    release(ctx->largeHashKeys);
    release(ctx->largeHashVals);
    release(ctx->bpKeys);
    release(ctx->rowCount);
    release(ctx->entryRow);
    release(ctx->rowStart);
    release(ctx->rows);
    release(ctx->sapVals);
    release(ctx->sapValsAlt);
    release(ctx->sapAxis);
    release(ctx->bpKeysAlt);
    release(ctx->pairCount);
    release(ctx->pairRecorded);
    release(ctx->pairOffset);
    release(ctx->llCount);
    release(ctx->llOffset);
    release(ctx->largeKeys);
    release(ctx->largeKeysAlt);
    for (cudaEvent_t e : ctx->evPool)
        cudaEventDestroy(e);
    for (ManBuf &m : ctx->man)
    {
        release(m.ab);
        release(m.seq);
        release(m.n);
        release(m.basis);
        release(m.contact);
    }
    release(ctx->keep);
    release(ctx->keepIdx);
    for (int k = 0; k < 2; ++k)
    {
        release(ctx->jointAB[k]);
        release(ctx->jointSeq[k]);
    }
    release(ctx->shape);
    release(ctx->stateStage);
    release(ctx->snapIds);
    release(ctx->snapIdsAlt);
    release(ctx->snapOrder);
    release(ctx->snapOrderAlt);
    release(ctx->snapRecords);
    release(ctx->editSeq);
    release(ctx->editAB);
    release(ctx->editData);
    release(ctx->editJoint);
    release(ctx->springAB);
    release(ctx->springSeq);
    release(ctx->ignoreAB);
    release(ctx->ignoreSeq);
    release(ctx->adjStart);
    release(ctx->adj);
    release(ctx->incVals);
    release(ctx->incValsAlt);
    release(ctx->incKeys);
    release(ctx->incKeysAlt);
    release(ctx->incKeys32);
    release(ctx->incKeys32Alt);
    release(ctx->colourState);
    release(ctx->colour);
    release(ctx->solveList);
    release(ctx->solveEntry);
    release(ctx->colourStart);
    release(ctx->colourCtl);
    release(ctx->colKeys);
    release(ctx->colKeysAlt);
    release(ctx->cubTemp);
    release(ctx->cubTempSide[0]);
    release(ctx->cubTempSide[1]);
    release(ctx->cubTempSide[2]);
    release(ctx->counters);
    release(ctx->stepState);
    release(ctx->llChunkLo);
    release(ctx->llChunkHi);
    release(ctx->llRecorded);
    release(ctx->pairSetKeys);
    release(ctx->pairLaneCount);
    for (DArr<int> *a : {&ctx->lbvhBodies, &ctx->lbvhBodiesAlt, &ctx->lbvhChild, &ctx->lbvhParent, &ctx->entryOf,
                         &ctx->worldBinnedStart})
        release(*a);
    release(ctx->lbvhCodes);
    release(ctx->lbvhCodesAlt);
    release(ctx->lbvhLo);
    release(ctx->lbvhHi);
    release(ctx->lbvhArrivals);
    release(ctx->colourFlow);
    release(ctx->colourBlockCounts);
    release(ctx->stepFlags);
    if (ctx->hCounters)
        cudaFreeHost(ctx->hCounters);
    if (ctx->hScalars)
        cudaFreeHost(ctx->hScalars);
    if (ctx->hStage)
        cudaFreeHost(ctx->hStage);
    if (ctx->hColourSummary)
        cudaFreeHost(ctx->hColourSummary);
    if (ctx->hGrid)
        cudaFreeHost(ctx->hGrid);
    if (ctx->hCapped)
        cudaFreeHost(ctx->hCapped);
    if (ctx->hColourStarts)
        cudaFreeHost(ctx->hColourStarts);
    if (ctx->hIterError)
        cudaFreeHost(ctx->hIterError);
    if (ctx->hState)
        cudaFreeHost(ctx->hState);
    if (ctx->hStepFlags)
        cudaFreeHost(ctx->hStepFlags);
    release(ctx->iterSync);
    release(ctx->iterDone);
    if (ctx->stageDone)
        cudaEventDestroy(ctx->stageDone);
    if (ctx->evStart)
        cudaEventDestroy(ctx->evStart);
    if (ctx->evStop)
        cudaEventDestroy(ctx->evStop);
    for (cudaEvent_t e : ctx->sideEv)
        if (e)
            cudaEventDestroy(e);
    for (cudaStream_t sd : ctx->side)
        if (sd)
            cudaStreamDestroy(sd);
    if (ctx->pool)
        cudaMemPoolDestroy(ctx->pool);
    if (ctx->ownStream && ctx->stream)
        cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char *avbd_last_error(const AvbdContext *ctx) { return ctx ? ctx->err.c_str() : "no context"; }

void avbd_clear_error(AvbdContext *ctx)
{
    if (ctx)
    {
        ctx->err.clear();
        ctx->errCode = 0;
        ctx->stateDirty = true; // clears the device steps' stop word before the next one
        if (ctx->hIterError)
            *ctx->hIterError = 0; // the failed iteration launch's flag was read already
    }
}

int avbd_set_params(AvbdContext *ctx, const AvbdParams *params)
{
    if (!ctx || !params)
        return fail(ctx, AVBD_ERR_ARGUMENT, "null argument");
    if (!(params->dt > 0.0f) || params->iterations < 0)
        return fail(ctx, AVBD_ERR_ARGUMENT, "invalid dt or iteration count");
    if (params->broadphase != AVBD_BROADPHASE_GRID && params->broadphase != AVBD_BROADPHASE_ALL_PAIRS &&
        params->broadphase != AVBD_BROADPHASE_SAP && params->broadphase != AVBD_BROADPHASE_LBVH)
        return fail(ctx, AVBD_ERR_ARGUMENT, "broadphase mode %d is not available on the GPU", params->broadphase);
    // pending device-resident steps run (or are redone) with the parameters they were issued with
    if (memcmp(&ctx->params, params, sizeof(AvbdParams)) != 0)
        SETTLED();
    ctx->params = *params;
    return AVBD_OK;
}

int avbd_load_world(AvbdContext *ctx, const AvbdBodies *bodies, const AvbdJoints *joints, const AvbdSprings *springs,
                    const AvbdIgnores *ignores, const AvbdManifolds *manifolds, int64_t next_seq)
{
    int32_t ws[2] = {0, bodies ? bodies->count : 0};
    return avbd_load_batch(ctx, 1, ws, bodies, joints, springs, ignores, manifolds, next_seq);
}

// Device layout of one joint: (rA, kLin) (rB, kAng) (C0Lin, fracture) (C0Ang, torqueArm)
// (penaltyLin, broken) (penaltyAng) (lambdaLin) (lambdaAng).
void pack_joint(const AvbdJoints *joints, int j, float4 *d)
{
    const float *s = joints->state28 + 28 * (size_t)j;
    float broken = joints->broken && joints->broken[j] ? 1.0f : 0.0f;
    d[0] = make_float4(s[0], s[1], s[2], s[24]);
    d[1] = make_float4(s[3], s[4], s[5], s[25]);
    d[2] = make_float4(s[6], s[7], s[8], s[26]);
    d[3] = make_float4(s[9], s[10], s[11], s[27]);
    d[4] = make_float4(s[12], s[13], s[14], broken);
    d[5] = make_float4(s[15], s[16], s[17], 0.0f);
    d[6] = make_float4(s[18], s[19], s[20], 0.0f);
    d[7] = make_float4(s[21], s[22], s[23], 0.0f);
}

int avbd_load_batch(AvbdContext *ctx, int32_t num_worlds, const int32_t *world_start, const AvbdBodies *bodies,
                    const AvbdJoints *joints, const AvbdSprings *springs, const AvbdIgnores *ignores,
                    const AvbdManifolds *manifolds, int64_t next_seq)
{
    if (!ctx || !bodies || !world_start)
        return fail(ctx, AVBD_ERR_ARGUMENT, "null argument");
    if (ctx->errCode)
        return AVBD_ERR_LATCHED;
    adjoint_invalidate(ctx);
    ctx->pendingFast = 0; // steps of the old world still in flight no longer matter (stream order)
    int n = bodies->count;
    if (n < 0 || n >= (int)KEY_NO_BODY)
        return fail(ctx, AVBD_ERR_ARGUMENT, "body count %d out of range", n);
    if (num_worlds < 1 || num_worlds >= (1 << 16))
        return fail(ctx, AVBD_ERR_ARGUMENT, "world count %d out of range [1, 65535]", num_worlds);
    if (world_start[0] != 0 || world_start[num_worlds] != n)
        return fail(ctx, AVBD_ERR_ARGUMENT, "world ranges must start at 0 and end at the body count");
    for (int w = 0; w < num_worlds; ++w)
        if (world_start[w + 1] < world_start[w])
            return fail(ctx, AVBD_ERR_ARGUMENT, "world ranges must be non-decreasing");
    if (n > 0 && (!bodies->position3 || !bodies->size3 || !bodies->mass || !bodies->moment3 ||
                  !bodies->friction || !bodies->radius || !bodies->velocity3))
        return fail(ctx, AVBD_ERR_ARGUMENT, "missing body arrays");
    CU(cudaSetDevice(ctx->device));
    ctx->n = n;
    ctx->W = num_worlds;
    ctx->hWorldStart.assign(world_start, world_start + num_worlds + 1);
    std::vector<int> worldOf(n);
    for (int w = 0; w < num_worlds; ++w)
        for (int b = world_start[w]; b < world_start[w + 1]; ++b)
            worldOf[b] = w;
    CHECK(upload_bodies(ctx, bodies, true));
    CHECK(classify_bodies(ctx, bodies->radius));

    auto check_ab = [&](const int32_t *ab, int count, bool allowWorldA) -> bool {
        for (int i = 0; i < count; ++i)
        {
            int a = ab[2 * i], b = ab[2 * i + 1];
            if (b < 0 || b >= n || a >= n || (a < 0 && !(allowWorldA && a == -1)) || a == b)
                return false;
            if (a >= 0 && worldOf[a] != worldOf[b]) // forces never join two worlds
                return false;
        }
        return true;
    };
    auto seqs = [&](const int64_t *s, int count, std::vector<unsigned long long> &out) {
        out.resize(count);
        for (int i = 0; i < count; ++i)
            out[i] = (unsigned long long)s[i];
    };
    // every sequence number lies in [0, next_seq): new forces continue from next_seq and the
    // adjacency keys are sized by it
    auto seqs_below = [&](const int64_t *s, int count) {
        for (int i = 0; i < count; ++i)
            if (s[i] < 0 || s[i] >= next_seq)
                return false;
        return true;
    };
    if (next_seq < 0 || (unsigned long long)next_seq > KEY_SEQ_MASK ||
        (joints && joints->count > 0 && joints->seq && !seqs_below(joints->seq, joints->count)) ||
        (springs && springs->count > 0 && springs->seq && !seqs_below(springs->seq, springs->count)) ||
        (ignores && ignores->count > 0 && ignores->seq && !seqs_below(ignores->seq, ignores->count)) ||
        (manifolds && manifolds->count > 0 && manifolds->seq && !seqs_below(manifolds->seq, manifolds->count)))
        return fail(ctx, AVBD_ERR_ARGUMENT, "sequence numbers must lie in [0, next_seq) with next_seq < 2^40");
    std::vector<unsigned long long> sq;
    // joints
    int J = joints ? joints->count : 0;
    if (J && (!joints->body_ab2 || !joints->seq || !joints->state28 || !check_ab(joints->body_ab2, J, true)))
        return fail(ctx, AVBD_ERR_ARGUMENT, "invalid joint arrays");
    {
        std::vector<float4> d((size_t)8 * J);
        for (int j = 0; j < J; ++j)
            pack_joint(joints, j, &d[8 * (size_t)j]);
        ctx->jcur = 0;
        CHECK(upload(ctx, ctx->joint[0], d.data(), d.size()));
        CHECK(upload(ctx, ctx->jointAB[0], (const int2 *)(J ? joints->body_ab2 : nullptr), J));
        if (J)
            seqs(joints->seq, J, sq);
        CHECK(upload(ctx, ctx->jointSeq[0], sq.data(), J));
        ctx->nJoint = J;
    }
    int S = springs ? springs->count : 0;
    if (S && (!springs->body_ab2 || !springs->seq || !springs->state8 || !check_ab(springs->body_ab2, S, false)))
        return fail(ctx, AVBD_ERR_ARGUMENT, "invalid spring arrays");
    {
        std::vector<float4> d((size_t)2 * S);
        for (int s = 0; s < S; ++s)
        {
            const float *v = springs->state8 + 8 * (size_t)s;
            d[2 * s] = make_float4(v[0], v[1], v[2], v[6]);
            d[2 * s + 1] = make_float4(v[3], v[4], v[5], v[7]);
        }
        CHECK(upload(ctx, ctx->spring, d.data(), d.size()));
        CHECK(upload(ctx, ctx->springAB, (const int2 *)(S ? springs->body_ab2 : nullptr), S));
        if (S)
            seqs(springs->seq, S, sq);
        CHECK(upload(ctx, ctx->springSeq, sq.data(), S));
        ctx->nSpring = S;
    }
    int I = ignores ? ignores->count : 0;
    if (I && (!ignores->body_ab2 || !ignores->seq || !check_ab(ignores->body_ab2, I, false)))
        return fail(ctx, AVBD_ERR_ARGUMENT, "invalid ignore-collision arrays");
    CHECK(upload(ctx, ctx->ignoreAB, (const int2 *)(I ? ignores->body_ab2 : nullptr), I));
    if (I)
        seqs(ignores->seq, I, sq);
    CHECK(upload(ctx, ctx->ignoreSeq, sq.data(), I));
    ctx->nIgnore = I;

    int M = manifolds ? manifolds->count : 0;
    if (M && (!manifolds->body_ab2 || !manifolds->seq || !manifolds->num_contacts ||
              !check_ab(manifolds->body_ab2, M, false)))
        return fail(ctx, AVBD_ERR_ARGUMENT, "invalid manifold arrays");
    ctx->cur = 0;
    CHECK(reserve_manifolds(ctx, ctx->man[0], (size_t)std::max(M, 1), 0));
    if (M)
    {
        std::vector<float4> basis((size_t)3 * M), contact((size_t)32 * M);
        std::vector<int> nc(M);
        for (int m = 0; m < M; ++m)
        {
            nc[m] = std::min(std::max(manifolds->num_contacts[m], 0), 8);
            const float *bs = manifolds->basis9 ? manifolds->basis9 + 9 * (size_t)m : nullptr;
            float fr = manifolds->friction ? manifolds->friction[m] : 0.0f;
            for (int r = 0; r < 3; ++r)
                basis[3 * m + r] = bs ? make_float4(bs[3 * r], bs[3 * r + 1], bs[3 * r + 2], r == 0 ? fr : 0.0f)
                                      : make_float4(0, 0, 0, 0);
            for (int k = 0; k < 8; ++k)
            {
                const float *c = manifolds->contact15x8 ? manifolds->contact15x8 + ((size_t)8 * m + k) * 15 : nullptr;
                float v[15] = {0};
                if (c)
                    memcpy(v, c, sizeof(v));
                unsigned key = manifolds->keys8 ? (unsigned)manifolds->keys8[8 * m + k] & 0x7FFFFFFFu : 0u;
                unsigned stick = manifolds->stick8 && manifolds->stick8[8 * m + k] ? 0x80000000u : 0u;
                float4 *o = &contact[(size_t)32 * m + 4 * k];
                o[0] = make_float4(v[0], v[1], v[2], v[3]);
                o[1] = make_float4(v[4], v[5], v[6], v[7]);
                o[2] = make_float4(v[8], v[9], v[10], v[11]);
                unsigned bits = key | stick;
                float w;
                memcpy(&w, &bits, 4);
                o[3] = make_float4(v[12], v[13], v[14], w);
            }
        }
        CU(cudaMemcpyAsync(ctx->man[0].ab.p, manifolds->body_ab2, sizeof(int2) * M, cudaMemcpyHostToDevice,
                           ctx->stream));
        seqs(manifolds->seq, M, sq);
        CU(cudaMemcpyAsync(ctx->man[0].seq.p, sq.data(), sizeof(unsigned long long) * M, cudaMemcpyHostToDevice,
                           ctx->stream));
        CU(cudaMemcpyAsync(ctx->man[0].n.p, nc.data(), sizeof(int) * M, cudaMemcpyHostToDevice, ctx->stream));
        CU(cudaMemcpyAsync(ctx->man[0].basis.p, basis.data(), sizeof(float4) * 3 * M, cudaMemcpyHostToDevice,
                           ctx->stream));
        CU(cudaMemcpyAsync(ctx->man[0].contact.p, contact.data(), sizeof(float4) * 32 * M, cudaMemcpyHostToDevice,
                           ctx->stream));
        CU(cudaStreamSynchronize(ctx->stream));
    }
    ctx->nMan = M;
    ctx->nextSeq = next_seq;
    {
        // the force lists' sequence numbers: each list ascending and no number in two lists
        // lets the adjacency place incidences by rank (later forces always get larger numbers)
        std::vector<unsigned long long> all;
        bool ascending = true;
        auto take = [&](const int64_t *sq, int count) {
            for (int i = 0; i < count; ++i)
            {
                ascending = ascending && (i == 0 || sq[i] > sq[i - 1]);
                all.push_back((unsigned long long)sq[i]);
            }
        };
        if (J)
            take(joints->seq, J);
        if (S)
            take(springs->seq, S);
        if (I)
            take(ignores->seq, I);
        if (M)
            take(manifolds->seq, M);
        std::sort(all.begin(), all.end());
        ctx->seqRanked = ascending && std::adjacent_find(all.begin(), all.end()) == all.end();
    }
    CHECK(build_adjacency(ctx));
    CU(cudaStreamSynchronize(ctx->stream));
    ctx->nColours = 0;
    ctx->nSolve = 0;
    ctx->loaded = true;
    ctx->stateDirty = true;
    ctx->deviceSteps = ctx->redoneSteps = 0;
    return AVBD_OK;
}

int avbd_write_bodies(AvbdContext *ctx, const AvbdBodies *bodies)
{
    SETTLED();
    if (!ctx || !bodies)
        return fail(ctx, AVBD_ERR_ARGUMENT, "null argument");
    if (!ctx->loaded || bodies->count != ctx->n)
        return fail(ctx, AVBD_ERR_STATE, "body count does not match the loaded world");
    CU(cudaSetDevice(ctx->device));
    adjoint_invalidate(ctx);
    CHECK(upload_bodies(ctx, bodies, false));
    return AVBD_OK;
}

int avbd_step(AvbdContext *ctx, int32_t nsteps)
{
    if (!ctx)
        return AVBD_ERR_ARGUMENT;
    if (ctx->errCode)
        return AVBD_ERR_LATCHED;
    if (!ctx->loaded)
        return fail(ctx, AVBD_ERR_STATE, "no world loaded");
    adjoint_invalidate(ctx);
    CU(cudaSetDevice(ctx->device));
    for (int s = 0; s < nsteps; ++s)
    {
        if (device_step_ok(ctx))
            CHECK(step_device(ctx));
        else
        {
            SETTLED();
            CHECK(step_once(ctx));
            ctx->stateDirty = true;
        }
    }
    // a synchronous step knows its counts: make room for device-resident steps right away
    if (ctx->pendingFast == 0 && device_step_ok(ctx))
        CHECK(device_reserve(ctx));
    return AVBD_OK;
}

int avbd_step_external(AvbdContext *ctx, int32_t num_pairs, const int32_t *pairs_ab2,
                       const AvbdExternalContacts *contacts)
{
    if (!ctx)
        return AVBD_ERR_ARGUMENT;
    if (ctx->errCode)
        return AVBD_ERR_LATCHED;
    if (!ctx->loaded)
        return fail(ctx, AVBD_ERR_STATE, "no world loaded");
    if (num_pairs < 0 || (num_pairs > 0 && !pairs_ab2))
        return fail(ctx, AVBD_ERR_ARGUMENT, "pairs: negative count or null array");
    const int ne = contacts ? contacts->count : 0;
    if (ne < 0 || (ne > 0 && (!contacts->body_ab2 || !contacts->num_contacts || !contacts->basis9 ||
                              !contacts->keys8 || !contacts->contact15x8 || !contacts->stick8)))
        return fail(ctx, AVBD_ERR_ARGUMENT, "external contacts: negative count or null array");
    SETTLED();
    adjoint_invalidate(ctx);
    CU(cudaSetDevice(ctx->device));
    const int n = ctx->n;
    auto world = [&](int b) {
        return (int)(std::upper_bound(ctx->hWorldStart.begin(), ctx->hWorldStart.end(), b) - ctx->hWorldStart.begin());
    };
    auto valid = [&](int a, int b) { return a >= 0 && b >= 0 && a < n && b < n && a != b && world(a) == world(b); };
    // pairs naming a body twice, no body or bodies of two worlds are skipped, as the reference
    // skips invalid ids (solver.cpp:584-593)
    ctx->hExtPairs.clear();
    for (int k = 0; k < num_pairs; ++k)
        if (valid(pairs_ab2[2 * k], pairs_ab2[2 * k + 1]))
            ctx->hExtPairs.push_back(make_int2(pairs_ab2[2 * k], pairs_ab2[2 * k + 1]));
    // contact entries: every valid one replaces the narrowphase of its pair (the last entry
    // for an ordered pair wins); each may also create its pair's manifold (solver.cpp:597-622)
    ctx->hExtEntryPairs.clear();
    std::vector<std::pair<unsigned long long, int>> keyed;
    std::vector<int> num;
    std::vector<float4> basis, rec;
    for (int e = 0; e < ne; ++e)
    {
        int a = contacts->body_ab2[2 * e], b = contacts->body_ab2[2 * e + 1];
        if (!valid(a, b))
            continue;
        const int slot = (int)num.size();
        if (!contacts->creates || contacts->creates[e])
            ctx->hExtEntryPairs.push_back(make_int2(a, b));
        keyed.push_back({((unsigned long long)(unsigned)a << 32) | (unsigned)b, slot});
        int nc = std::min(std::max(contacts->num_contacts[e], 0), 8);
        num.push_back(nc);
        const float *bs = contacts->basis9 + 9 * (size_t)e;
        for (int r = 0; r < 3; ++r)
            basis.push_back(make_float4(bs[3 * r], bs[3 * r + 1], bs[3 * r + 2], 0.0f));
        for (int i = 0; i < 8; ++i)
        {
            const float *c = contacts->contact15x8 + (8 * (size_t)e + i) * 15; // rA rB C0 penalty lambda
            unsigned key = (unsigned)contacts->keys8[8 * (size_t)e + i];
            unsigned stick = contacts->stick8[8 * (size_t)e + i] ? 0x80000000u : 0u;
            rec.push_back(make_float4(c[0], c[1], c[2], c[3]));
            rec.push_back(make_float4(c[4], c[5], c[6], c[7]));
            rec.push_back(make_float4(c[8], c[9], c[10], c[11]));
            unsigned word = (key & 0x7FFFFFFFu) | stick;
            float last;
            memcpy(&last, &word, sizeof(last));
            rec.push_back(make_float4(c[12], c[13], c[14], last));
        }
    }
    // ordered keys, ascending; for a repeated key the later entry is kept
    std::stable_sort(keyed.begin(), keyed.end(),
                     [](const std::pair<unsigned long long, int> &x, const std::pair<unsigned long long, int> &y) {
                         return x.first < y.first;
                     });
    std::vector<unsigned long long> keys;
    std::vector<int> entry;
    for (size_t k = 0; k < keyed.size(); ++k)
    {
        if (k + 1 < keyed.size() && keyed[k + 1].first == keyed[k].first)
            continue;
        keys.push_back(keyed[k].first);
        entry.push_back(keyed[k].second);
    }
    ctx->extKeyCount = (int)keys.size();
    if (ctx->extKeyCount)
    {
        CHECK(upload(ctx, ctx->extKeys, keys.data(), keys.size()));
        CHECK(upload(ctx, ctx->extEntry, entry.data(), entry.size()));
        CHECK(upload(ctx, ctx->extNum, num.data(), num.size()));
        CHECK(upload(ctx, ctx->extBasis, basis.data(), basis.size()));
        CHECK(upload(ctx, ctx->extContact, rec.data(), rec.size()));
    }
    ctx->external = true;
    int rc = step_once(ctx);
    ctx->external = false;
    ctx->extKeyCount = 0;
    ctx->stateDirty = true;
    if (rc == AVBD_OK)
        rc = (cudaStreamSynchronize(ctx->stream) == cudaSuccess) ? AVBD_OK
                                                                  : fail(ctx, AVBD_ERR_CUDA, "external step failed");
    return rc;
}

int avbd_set_step_mode(AvbdContext *ctx, int32_t mode)
{
    if (!ctx || (mode != AVBD_STEP_DEVICE && mode != AVBD_STEP_HOST))
        return fail(ctx, AVBD_ERR_ARGUMENT, "step mode must be AVBD_STEP_DEVICE or AVBD_STEP_HOST");
    SETTLED();
    ctx->stepMode = mode;
    return AVBD_OK;
}

int avbd_set_manifold_headroom(AvbdContext *ctx, int64_t spare)
{
    if (!ctx || spare < 0)
        return fail(ctx, AVBD_ERR_ARGUMENT, "manifold headroom must be zero or positive");
    SETTLED();
    ctx->manifoldSpare = spare;
    return AVBD_OK;
}

int avbd_set_wait_limits(AvbdContext *ctx, uint32_t colouring_polls, uint32_t iteration_polls)
{
    if (!ctx)
        return AVBD_ERR_ARGUMENT;
    SETTLED();
    ctx->waitColour = colouring_polls;
    ctx->waitIteration = iteration_polls;
    return AVBD_OK;
}

int avbd_broadphase_only(AvbdContext *ctx)
{
    SETTLED();
    if (!ctx)
        return AVBD_ERR_ARGUMENT;
    if (ctx->errCode)
        return AVBD_ERR_LATCHED;
    if (!ctx->loaded)
        return fail(ctx, AVBD_ERR_STATE, "no world loaded");
    adjoint_invalidate(ctx);
    CU(cudaSetDevice(ctx->device));
    // Solver::benchmarkBroadphaseOnly (solver.cpp:989-1034): every manifold goes, so only
    // joints, springs and ignore pairs count as constraints for the broadphase
    ctx->nMan = 0;
    CHECK(build_adjacency(ctx));
    CU(cudaMemsetAsync(ctx->counters.p, 0, sizeof(StepCounters), ctx->stream));
    ctx->stats.grid_rescaled = 0;
    {
        PhaseScope ps(ctx, AVBD_PHASE_BROADPHASE);
        CHECK(broadphase(ctx));
    }
    // the new manifolds join their bodies' force lists (no contacts until a step)
    CHECK(build_adjacency(ctx));
    CU(cudaMemcpyAsync(ctx->hCounters, ctx->counters.p, sizeof(StepCounters), cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    ctx->stats.body_count = ctx->n;
    ctx->stats.manifold_count = ctx->nMan;
    ctx->stats.contact_count = 0;
    ctx->stats.pair_checks = (int64_t)ctx->hCounters->pairChecks;
    ctx->stats.sphere_hits = (int64_t)ctx->hCounters->sphereHits;
    ctx->stats.constrained_hits = (int64_t)ctx->hCounters->constrainedHits;
    if (ctx->profiling)
        ctx->stepsProfiled++;
    CHECK(prof_collect(ctx));
    return AVBD_OK;
}

int avbd_synchronize(AvbdContext *ctx)
{
    if (!ctx)
        return AVBD_ERR_ARGUMENT;
    if (ctx->errCode)
        return AVBD_ERR_LATCHED;
    SETTLED();
    CU(cudaStreamSynchronize(ctx->stream));
    if (*ctx->hIterError)
        return fail(ctx, AVBD_ERR_STATE, "iteration kernel wait expired (a grid barrier or a partner body's iteration count)");
    return AVBD_OK;
}

int avbd_read_bodies(AvbdContext *ctx, const AvbdBodyState *out)
{
    if (!ctx || !out)
    {
        SETTLED();
        return fail(ctx, AVBD_ERR_ARGUMENT, "null argument");
    }
    int n = ctx->n;
    DArr<float4> *src[MAX_PACKED] = {&ctx->pos,     &ctx->quat,    &ctx->vel,      &ctx->angvel,  &ctx->prevVel,
                                     &ctx->initLin, &ctx->initAng, &ctx->inertLin, &ctx->inertAng};
    float *dst[MAX_PACKED] = {out->position3,         out->orientation4,         out->velocity3,
                              out->angular3,          out->prev_velocity3,       out->initial_position3,
                              out->initial_orientation4, out->inertial_position3, out->inertial_orientation4};
    const int width[MAX_PACKED] = {3, 4, 3, 3, 3, 3, 4, 3, 4};
    if (!n || std::none_of(dst, dst + MAX_PACKED, [](const float *d) { return d != nullptr; }))
    {
        SETTLED();
        return AVBD_OK;
    }
    // requested fields packed on the device: written in place into page-locked caller arrays,
    // the rest downloaded through the staging buffer (and copied on the host after the wait)
    std::vector<HostCopy> copies;
    auto issue = [&]() -> int {
        PackedFields P{};
        P.count = MAX_PACKED;
        long long floats = 0;
        float *mapped[MAX_PACKED] = {};
        for (int f = 0; f < MAX_PACKED; ++f)
        {
            mapped[f] = dst[f] ? host_mapped(dst[f]) : nullptr;
            if (dst[f] && !mapped[f])
                floats += (long long)width[f] * n;
        }
        CHECK(stage_reserve(ctx, (size_t)(floats + 3) / 4));
        CHECK(reserve(ctx, ctx->stateStage, (size_t)std::max<long long>(floats, 1), false));
        float *st = (float *)ctx->hStage;
        copies.clear();
        long long off = 0;
        for (int f = 0; f < MAX_PACKED; ++f)
        {
            float *buf = nullptr;
            if (mapped[f])
                buf = mapped[f];
            else if (dst[f])
            {
                buf = ctx->stateStage.p + off;
                copies.push_back({dst[f], st + off, sizeof(float) * width[f] * (size_t)n});
                off += (long long)width[f] * n;
            }
            P.f[f] = PackedField{src[f]->p, buf, width[f], buf ? (int)aligned16(buf) : 0, 0.0f};
        }
        k_pack_state<<<grid_for(n, PACK_BLOCK), PACK_BLOCK, 0, ctx->stream>>>(P, n);
        LAUNCHED();
        for (const HostCopy &c : copies)
            CU(cudaMemcpyAsync((void *)c.src, ctx->stateStage.p + ((const float *)c.src - st), c.bytes,
                               cudaMemcpyDeviceToHost, ctx->stream));
        return AVBD_OK;
    };
    // With device steps pending, the packing is queued behind them before the wait for them,
    // so that one wait serves both; if a step stopped on the device and was redone, the
    // fields are packed again after the redo.
    const bool early = ctx->pendingFast > 0 && ctx->errCode == 0;
    if (early)
        CHECK(issue());
    const long long redone = ctx->redoneSteps;
    SETTLED();
    if (!early || ctx->redoneSteps != redone)
        CHECK(issue());
    CU(cudaStreamSynchronize(ctx->stream));
    copy_host(copies);
    return AVBD_OK;
}

int avbd_num_manifolds(AvbdContext *ctx, int32_t *count)
{
    SETTLED();
    if (!ctx || !count)
        return fail(ctx, AVBD_ERR_ARGUMENT, "null argument");
    *count = ctx->nMan;
    return AVBD_OK;
}

int avbd_read_manifolds(AvbdContext *ctx, const AvbdManifoldsOut *out)
{
    SETTLED();
    if (!ctx || !out)
        return fail(ctx, AVBD_ERR_ARGUMENT, "null argument");
    int M = ctx->nMan;
    if (!M)
        return AVBD_OK;
    ManBuf &b = ctx->man[ctx->cur];
    std::vector<int2> ab(M);
    std::vector<unsigned long long> seq(M);
    std::vector<int> nc(M);
    std::vector<float4> basis((size_t)3 * M), contact((size_t)32 * M);
    CU(cudaMemcpyAsync(ab.data(), b.ab.p, sizeof(int2) * M, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaMemcpyAsync(seq.data(), b.seq.p, sizeof(unsigned long long) * M, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaMemcpyAsync(nc.data(), b.n.p, sizeof(int) * M, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaMemcpyAsync(basis.data(), b.basis.p, sizeof(float4) * 3 * M, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaMemcpyAsync(contact.data(), b.contact.p, sizeof(float4) * 32 * M, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    for (int m = 0; m < M; ++m)
    {
        if (out->body_ab2)
        {
            out->body_ab2[2 * m] = ab[m].x;
            out->body_ab2[2 * m + 1] = ab[m].y;
        }
        if (out->seq)
            out->seq[m] = (int64_t)seq[m];
        if (out->num_contacts)
            out->num_contacts[m] = nc[m];
        if (out->basis9)
            for (int r = 0; r < 3; ++r)
            {
                out->basis9[9 * m + 3 * r] = basis[3 * m + r].x;
                out->basis9[9 * m + 3 * r + 1] = basis[3 * m + r].y;
                out->basis9[9 * m + 3 * r + 2] = basis[3 * m + r].z;
            }
        if (out->friction)
            out->friction[m] = basis[3 * m].w;
        for (int k = 0; k < 8; ++k)
        {
            bool live = k < nc[m];
            const float4 *c = &contact[(size_t)32 * m + 4 * k];
            unsigned bits;
            memcpy(&bits, &c[3].w, 4);
            if (out->keys8)
                out->keys8[8 * m + k] = live ? (int)(bits & 0x7FFFFFFFu) : 0;
            if (out->stick8)
                out->stick8[8 * m + k] = live ? (int)(bits >> 31) : 0;
            if (out->contact15x8)
            {
                float *o = out->contact15x8 + ((size_t)8 * m + k) * 15;
                float v[16] = {c[0].x, c[0].y, c[0].z, c[0].w, c[1].x, c[1].y, c[1].z, c[1].w,
                               c[2].x, c[2].y, c[2].z, c[2].w, c[3].x, c[3].y, c[3].z, 0.0f};
                for (int q = 0; q < 15; ++q)
                    o[q] = live ? v[q] : 0.0f;
            }
        }
    }
    return AVBD_OK;
}

int avbd_num_joints(AvbdContext *ctx, int32_t *count)
{
    SETTLED();
    if (!ctx || !count)
        return fail(ctx, AVBD_ERR_ARGUMENT, "null argument");
    *count = ctx->nJoint;
    return AVBD_OK;
}

int avbd_read_joints(AvbdContext *ctx, const AvbdJointsOut *out)
{
    SETTLED();
    if (!ctx || !out)
        return fail(ctx, AVBD_ERR_ARGUMENT, "null argument");
    int J = ctx->nJoint;
    if (!J)
        return AVBD_OK;
    std::vector<int2> ab(J);
    std::vector<unsigned long long> seq(J);
    std::vector<float4> d((size_t)8 * J);
    CU(cudaMemcpyAsync(ab.data(), ctx->jointAB[ctx->jcur].p, sizeof(int2) * J, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaMemcpyAsync(seq.data(), ctx->jointSeq[ctx->jcur].p, sizeof(unsigned long long) * J,
                       cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaMemcpyAsync(d.data(), ctx->joint[ctx->jcur].p, sizeof(float4) * 8 * J, cudaMemcpyDeviceToHost,
                       ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    for (int j = 0; j < J; ++j)
    {
        if (out->body_ab2)
        {
            out->body_ab2[2 * j] = ab[j].x;
            out->body_ab2[2 * j + 1] = ab[j].y;
        }
        if (out->seq)
            out->seq[j] = (int64_t)seq[j];
        if (out->state28)
        {
            float *s = out->state28 + 28 * (size_t)j;
            for (int k = 0; k < 8; ++k)
            {
                s[3 * k] = d[8 * j + k].x;
                s[3 * k + 1] = d[8 * j + k].y;
                s[3 * k + 2] = d[8 * j + k].z;
            }
            s[24] = d[8 * j + 0].w;
            s[25] = d[8 * j + 1].w;
            s[26] = d[8 * j + 2].w;
            s[27] = d[8 * j + 3].w;
        }
        if (out->broken)
            out->broken[j] = d[8 * j + 4].w != 0.0f ? 1 : 0;
    }
    return AVBD_OK;
}

int avbd_next_seq(AvbdContext *ctx, int64_t *next_seq)
{
    SETTLED();
    if (!ctx || !next_seq)
        return fail(ctx, AVBD_ERR_ARGUMENT, "null argument");
    *next_seq = ctx->nextSeq;
    return AVBD_OK;
}

// ---------------------------------------------------------------------------
// Joint edits between steps (SimulationHost's drag: simulation_host.cpp:242-274)
// ---------------------------------------------------------------------------

int edit_begin(AvbdContext *ctx)
{
    if (!ctx)
        return AVBD_ERR_ARGUMENT;
    if (ctx->errCode)
        return AVBD_ERR_LATCHED;
    if (!ctx->loaded)
        return fail(ctx, AVBD_ERR_STATE, "no world loaded");
    CU(cudaSetDevice(ctx->device));
    adjoint_invalidate(ctx);
    return AVBD_OK;
}

int world_of(const AvbdContext *ctx, int body)
{
    const std::vector<int> &ws = ctx->hWorldStart;
    return (int)(std::upper_bound(ws.begin(), ws.end(), body) - ws.begin()) - 1;
}

// Matches `count` sorted sequence numbers (with their bodies, when ab is given) against the
// device joints; keep (optional) receives the survivors of a removal. Returns the matches.
int match_joints(AvbdContext *ctx, const std::vector<unsigned long long> &seq, const std::vector<int2> *ab,
                 bool removal, int &matched)
{
    int E = (int)seq.size(), J = ctx->nJoint;
    CHECK(upload(ctx, ctx->editSeq, seq.data(), (size_t)E));
    if (ab)
        CHECK(upload(ctx, ctx->editAB, ab->data(), (size_t)E));
    CHECK(reserve(ctx, ctx->editJoint, (size_t)E + 1, false));
    int *counter = ctx->editJoint.p + E;
    CU(cudaMemsetAsync(ctx->editJoint.p, 0xFF, sizeof(int) * E, ctx->stream));
    CU(cudaMemsetAsync(counter, 0, sizeof(int), ctx->stream));
    if (removal)
        CHECK(reserve(ctx, ctx->keep, (size_t)std::max(J, 1), false));
    if (J)
    {
        k_joint_match<<<grid_for(J, 128), 128, 0, ctx->stream>>>(
            J, ctx->jointSeq[ctx->jcur].p, ctx->jointAB[ctx->jcur].p, E, ctx->editSeq.p, ab ? ctx->editAB.p : nullptr,
            ctx->editJoint.p, removal ? ctx->keep.p : nullptr, counter);
        LAUNCHED();
    }
    int *h = (int *)(ctx->hScalars + 8);
    CU(cudaMemcpyAsync(h, counter, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    matched = *h;
    return AVBD_OK;
}

int avbd_add_joints(AvbdContext *ctx, const AvbdJoints *joints)
{
    SETTLED();
    CHECK(edit_begin(ctx));
    if (!joints || joints->count < 0)
        return fail(ctx, AVBD_ERR_ARGUMENT, "null or negative joint list");
    int E = joints->count, J = ctx->nJoint, n = ctx->n;
    if (!E)
        return AVBD_OK;
    if (!joints->body_ab2 || !joints->seq || !joints->state28)
        return fail(ctx, AVBD_ERR_ARGUMENT, "missing joint arrays");
    for (int e = 0; e < E; ++e)
    {
        int a = joints->body_ab2[2 * e], b = joints->body_ab2[2 * e + 1];
        if (b < 0 || b >= n || a < -1 || a >= n || a == b || (a >= 0 && world_of(ctx, a) != world_of(ctx, b)))
            return fail(ctx, AVBD_ERR_ARGUMENT, "joint %d: invalid bodies (%d, %d)", e, a, b);
        long long prev = e ? (long long)joints->seq[e - 1] : ctx->nextSeq - 1;
        // a new Joint is the newest force (force.cpp:17-35): sequence numbers keep growing
        if ((long long)joints->seq[e] <= prev || (unsigned long long)joints->seq[e] > KEY_SEQ_MASK)
            return fail(ctx, AVBD_ERR_ARGUMENT, "joint %d: sequence %lld is not above %lld", e,
                        (long long)joints->seq[e], prev);
    }
    std::vector<float4> d((size_t)8 * E);
    std::vector<unsigned long long> sq(E);
    for (int e = 0; e < E; ++e)
    {
        pack_joint(joints, e, &d[8 * (size_t)e]);
        sq[e] = (unsigned long long)joints->seq[e];
    }
    int c = ctx->jcur;
    CHECK(reserve(ctx, ctx->jointAB[c], (size_t)J + E, true, (size_t)J));
    CHECK(reserve(ctx, ctx->jointSeq[c], (size_t)J + E, true, (size_t)J));
    CHECK(reserve(ctx, ctx->joint[c], 8 * ((size_t)J + E), true, 8 * (size_t)J));
    CU(cudaMemcpyAsync(ctx->jointAB[c].p + J, joints->body_ab2, sizeof(int2) * E, cudaMemcpyHostToDevice,
                       ctx->stream));
    CU(cudaMemcpyAsync(ctx->jointSeq[c].p + J, sq.data(), sizeof(unsigned long long) * E, cudaMemcpyHostToDevice,
                       ctx->stream));
    CU(cudaMemcpyAsync(ctx->joint[c].p + 8 * (size_t)J, d.data(), sizeof(float4) * 8 * E, cudaMemcpyHostToDevice,
                       ctx->stream));
    ctx->nJoint = J + E;
    ctx->nextSeq = (long long)sq[E - 1] + 1;
    CHECK(build_adjacency(ctx));
    CU(cudaStreamSynchronize(ctx->stream));
    return AVBD_OK;
}

int avbd_remove_joints(AvbdContext *ctx, int32_t count, const int64_t *seq)
{
    SETTLED();
    CHECK(edit_begin(ctx));
    if (count < 0 || (count && !seq))
        return fail(ctx, AVBD_ERR_ARGUMENT, "null or negative sequence list");
    if (!count)
        return AVBD_OK;
    std::vector<unsigned long long> sq(seq, seq + count);
    std::sort(sq.begin(), sq.end());
    if (std::adjacent_find(sq.begin(), sq.end()) != sq.end())
        return fail(ctx, AVBD_ERR_ARGUMENT, "repeated joint sequence number");
    int J = ctx->nJoint, matched = 0;
    CHECK(match_joints(ctx, sq, nullptr, true, matched));
    if (matched != count)
        return fail(ctx, AVBD_ERR_ARGUMENT, "%d of %d sequence numbers name no joint", count - matched, count);
    int newJ = J - matched, o = ctx->jcur ^ 1; // matched counts the joints cleared from keep
    CHECK(reserve(ctx, ctx->keepIdx, (size_t)std::max(J, 1) * 2, false));
    int *idx = ctx->keepIdx.p, *cnt32 = ctx->keepIdx.p + std::max(J, 1);
    k_u8_to_int<<<grid_for(J, 256), 256, 0, ctx->stream>>>(ctx->keep.p, cnt32, J);
    LAUNCHED();
    CHECK(scan_counts(ctx, cnt32, idx, J, 0));
    CHECK(reserve(ctx, ctx->jointAB[o], (size_t)std::max(newJ, 1), false));
    CHECK(reserve(ctx, ctx->jointSeq[o], (size_t)std::max(newJ, 1), false));
    CHECK(reserve(ctx, ctx->joint[o], 8 * (size_t)std::max(newJ, 1), false));
    k_joint_compact<<<grid_for(J, 128), 128, 0, ctx->stream>>>(
        J, ctx->keep.p, idx, ctx->jointAB[ctx->jcur].p, ctx->jointSeq[ctx->jcur].p, ctx->joint[ctx->jcur].p,
        ctx->jointAB[o].p, ctx->jointSeq[o].p, ctx->joint[o].p);
    LAUNCHED();
    ctx->jcur = o;
    ctx->nJoint = newJ;
    CHECK(build_adjacency(ctx));
    CU(cudaStreamSynchronize(ctx->stream));
    return AVBD_OK;
}

int avbd_write_joints(AvbdContext *ctx, const AvbdJoints *joints)
{
    SETTLED();
    CHECK(edit_begin(ctx));
    if (!joints || joints->count < 0)
        return fail(ctx, AVBD_ERR_ARGUMENT, "null or negative joint list");
    int E = joints->count;
    if (!E)
        return AVBD_OK;
    if (!joints->body_ab2 || !joints->seq || !joints->state28)
        return fail(ctx, AVBD_ERR_ARGUMENT, "missing joint arrays");
    std::vector<int> order(E);
    for (int e = 0; e < E; ++e)
        order[e] = e;
    std::sort(order.begin(), order.end(), [&](int x, int y) { return joints->seq[x] < joints->seq[y]; });
    std::vector<unsigned long long> sq(E);
    std::vector<int2> ab(E);
    std::vector<float4> d((size_t)8 * E);
    for (int i = 0; i < E; ++i)
    {
        int e = order[i];
        sq[i] = (unsigned long long)joints->seq[e];
        ab[i] = make_int2(joints->body_ab2[2 * e], joints->body_ab2[2 * e + 1]);
        pack_joint(joints, e, &d[8 * (size_t)i]);
        if (i && sq[i] == sq[i - 1])
            return fail(ctx, AVBD_ERR_ARGUMENT, "repeated joint sequence number");
    }
    int matched = 0;
    CHECK(match_joints(ctx, sq, &ab, false, matched));
    if (matched != E)
        return fail(ctx, AVBD_ERR_ARGUMENT, "%d of %d joints match no device joint (sequence and bodies)",
                    E - matched, E);
    CHECK(upload(ctx, ctx->editData, d.data(), d.size()));
    k_joint_write<<<grid_for(8 * E, 128), 128, 0, ctx->stream>>>(E, ctx->editJoint.p, ctx->editData.p,
                                                                  ctx->joint[ctx->jcur].p, ctx->nJoint);
    LAUNCHED();
    CU(cudaStreamSynchronize(ctx->stream));
    return AVBD_OK;
}

// ---------------------------------------------------------------------------
// Snapshots for the viewer bridge (viewer_bridge.cpp:748-842)
// ---------------------------------------------------------------------------

constexpr uint32_t SNAPSHOT_MAGIC = 0x53425641u; // "AVBS" read as a little-endian u32
constexpr uint32_t SNAPSHOT_VERSION = 1;
constexpr size_t SNAPSHOT_HEADER = 24, SNAPSHOT_RECORD = 64;

// One 64-byte record per body, four 16-byte stores: id, shape, material
// (materialIdForBody), dynamic, position, rotation (x y z w), full size, shape radius, half
// length (0 for boxes and spheres). Record k is body order[k] with id
// ids[k]; without them, the body of creation rank k (list index n - 1 - k) with id k.
__global__ void k_snapshot_records(DevBodies B, const int *order, const unsigned *ids, int n, uint4 *out)
{
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int k = (int)(t >> 2), part = (int)(t & 3);
    if (k >= n)
        return;
    int b = order ? order[k] : n - 1 - k;
    uint4 w;
    BodyShape sh = body_shape(B, b);
    if (part == 0)
    {
        unsigned id = ids ? ids[k] : (unsigned)k;
        unsigned dyn = B.massMoment[b].x > 0.0f ? 1u : 0u;
        // materialIdForBody (viewer_bridge.cpp:475-493)
        unsigned mat = !dyn                        ? 0u
                       : sh.type == SHAPE_SPHERE   ? 3u
                       : sh.type == SHAPE_CYLINDER ? 4u
                       : sh.type == SHAPE_CAPSULE  ? 5u
                                                   : 1u;
        w = make_uint4(id, (unsigned)sh.type, mat, dyn);
    }
    else if (part == 1)
    {
        float4 p = B.pos[b], q = B.quat[b];
        w = make_uint4(__float_as_uint(p.x), __float_as_uint(p.y), __float_as_uint(p.z), __float_as_uint(q.x));
    }
    else if (part == 2)
    {
        float4 q = B.quat[b], sz = B.sizeRad[b];
        w = make_uint4(__float_as_uint(q.y), __float_as_uint(q.z), __float_as_uint(q.w), __float_as_uint(sz.x));
    }
    else
    {
        float4 sz = B.sizeRad[b];
        float radius = B.shape ? sh.radius : sz.w; // a box's shape radius is its bounding radius
        w = make_uint4(__float_as_uint(sz.y), __float_as_uint(sz.z), __float_as_uint(radius),
                       __float_as_uint(sh.halfLength));
    }
    out[4 * (size_t)k + part] = w;
}

// Records of every body into host memory at `dst`, in ascending id order.
int snapshot_records(AvbdContext *ctx, const int32_t *body_id, unsigned char *dst)
{
    int n = ctx->n;
    if (n == 0)
        return AVBD_OK;
    const int *order = nullptr;
    const unsigned *ids = nullptr;
    if (body_id)
    {
        for (int i = 0; i < n; ++i)
            if (body_id[i] < 0)
                return fail(ctx, AVBD_ERR_ARGUMENT, "body %d: negative snapshot id", i);
        std::vector<int> idx(n);
        for (int i = 0; i < n; ++i)
            idx[i] = i;
        CHECK(upload(ctx, ctx->snapIds, (const unsigned *)body_id, n));
        CHECK(upload(ctx, ctx->snapOrder, idx.data(), n));
        CHECK(reserve(ctx, ctx->snapIdsAlt, n, false));
        CHECK(reserve(ctx, ctx->snapOrderAlt, n, false));
        cub::DoubleBuffer<unsigned> dk(ctx->snapIds.p, ctx->snapIdsAlt.p);
        cub::DoubleBuffer<int> dv(ctx->snapOrder.p, ctx->snapOrderAlt.p);
        size_t bytes = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, bytes, dk, dv, n, 0, 32, ctx->stream);
        CHECK(ensure_temp(ctx, bytes));
        CU(cub::DeviceRadixSort::SortPairs(ctx->cubTemp.p, bytes, dk, dv, n, 0, 32, ctx->stream));
        ids = dk.Current();
        order = dv.Current();
    }
    CHECK(reserve(ctx, ctx->snapRecords, 4 * (size_t)n, false));
    k_snapshot_records<<<grid_for(4ll * n, 256), 256, 0, ctx->stream>>>(dev_bodies(ctx), order, ids, n,
                                                                          ctx->snapRecords.p);
    LAUNCHED();
    CU(cudaMemcpyAsync(dst, ctx->snapRecords.p, SNAPSHOT_RECORD * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return AVBD_OK;
}

int avbd_snapshot_binary(AvbdContext *ctx, uint64_t frame, const char *scene_name, const int32_t *body_id,
                         uint8_t *out, int64_t capacity, int64_t *size)
{
    SETTLED();
    if (!ctx || !size)
        return fail(ctx, AVBD_ERR_ARGUMENT, "null argument");
    if (!ctx->loaded)
        return fail(ctx, AVBD_ERR_STATE, "no world loaded");
    CU(cudaSetDevice(ctx->device));
    size_t sceneBytes = scene_name ? strlen(scene_name) : 0;
    size_t total = SNAPSHOT_HEADER + sceneBytes + SNAPSHOT_RECORD * (size_t)ctx->n;
    *size = (int64_t)total;
    if (!out)
        return AVBD_OK;
    if (capacity < (int64_t)total)
        return fail(ctx, AVBD_ERR_CAPACITY, "snapshot needs %zu bytes, buffer holds %lld", total, (long long)capacity);
    uint32_t head[2] = {SNAPSHOT_MAGIC, SNAPSHOT_VERSION}, counts[2] = {(uint32_t)sceneBytes, (uint32_t)ctx->n};
    memcpy(out, head, 8);
    memcpy(out + 8, &frame, 8);
    memcpy(out + 16, counts, 8);
    if (sceneBytes)
        memcpy(out + SNAPSHOT_HEADER, scene_name, sceneBytes);
    return snapshot_records(ctx, body_id, out + SNAPSHOT_HEADER + sceneBytes);
}

// makeSnapshotJson's text (viewer_bridge.cpp:748-777, jsonEscape :495-530) from the same
// records, with the same stream settings (fixed, 5 decimals).
int avbd_snapshot_json(AvbdContext *ctx, uint64_t frame, const char *scene_name, const int32_t *body_id, char *out,
                       int64_t capacity, int64_t *size)
{
    SETTLED();
    if (!ctx || !size)
        return fail(ctx, AVBD_ERR_ARGUMENT, "null argument");
    if (!ctx->loaded)
        return fail(ctx, AVBD_ERR_STATE, "no world loaded");
    CU(cudaSetDevice(ctx->device));
    int n = ctx->n;
    std::vector<unsigned char> rec(SNAPSHOT_RECORD * (size_t)n);
    CHECK(snapshot_records(ctx, body_id, rec.data()));
    std::string scene;
    for (const char *c = scene_name ? scene_name : ""; *c; ++c)
    {
        if (*c == '"' || *c == '\\')
        {
            scene.push_back('\\');
            scene.push_back(*c);
        }
        else if (*c == '\n')
            scene += "\\n";
        else if (*c == '\r')
            scene += "\\r";
        else if (*c == '\t')
            scene += "\\t";
        else if ((unsigned char)*c < 0x20)
        {
            char escaped[7];
            snprintf(escaped, sizeof(escaped), "\\u%04x", (unsigned char)*c);
            scene += escaped;
        }
        else
            scene.push_back(*c);
    }
    std::ostringstream os;
    os << std::fixed << std::setprecision(5);
    os << "{\"type\":\"snapshot\",\"version\":1,\"frame\":" << frame << ",\"scene\":\"" << scene
       << "\",\"bodies\":[";
    for (int k = 0; k < n; ++k)
    {
        const unsigned char *r = rec.data() + SNAPSHOT_RECORD * (size_t)k;
        uint32_t w[4];
        float f[12];
        memcpy(w, r, 16);
        memcpy(f, r + 16, 48);
        if (k)
            os << ",";
        static const char *names[4] = {"box", "sphere", "capsule", "cylinder"}; // shapeName (:458-473)
        os << "{\"id\":" << w[0] << ",\"shape\":\"" << names[w[1] & 3] << "\"" << ",\"position\":[" << f[0] << "," << f[1] << ","
           << f[2] << "]" << ",\"rotation\":[" << f[3] << "," << f[4] << "," << f[5] << "," << f[6] << "]"
           << ",\"size\":[" << f[7] << "," << f[8] << "," << f[9] << "]" << ",\"radius\":" << f[10]
           << ",\"halfLength\":" << f[11] << ",\"dynamic\":" << (w[3] ? "true" : "false")
           << ",\"material\":" << w[2] << "}";
    }
    os << "]}";
    std::string text = os.str();
    *size = (int64_t)text.size() + 1;
    if (!out)
        return AVBD_OK;
    if (capacity < *size)
        return fail(ctx, AVBD_ERR_CAPACITY, "snapshot text needs %lld bytes, buffer holds %lld", (long long)*size,
                    (long long)capacity);
    memcpy(out, text.c_str(), text.size() + 1);
    return AVBD_OK;
}

int avbd_read_colours(AvbdContext *ctx, int32_t *colour, int32_t *num_colours)
{
    SETTLED();
    if (!ctx)
        return AVBD_ERR_ARGUMENT;
    if (num_colours)
        *num_colours = ctx->nColours;
    if (colour && ctx->n)
    {
        if (!ctx->colour.p)
        {
            for (int i = 0; i < ctx->n; ++i)
                colour[i] = -1;
            return AVBD_OK;
        }
        CU(cudaMemcpyAsync(colour, ctx->colour.p, sizeof(int) * ctx->n, cudaMemcpyDeviceToHost, ctx->stream));
        CU(cudaStreamSynchronize(ctx->stream));
    }
    return AVBD_OK;
}

int avbd_read_solve_order(AvbdContext *ctx, int32_t *order, int32_t *count)
{
    SETTLED();
    if (!ctx)
        return AVBD_ERR_ARGUMENT;
    if (count)
        *count = ctx->nSolve;
    if (order && ctx->nSolve)
    {
        CU(cudaMemcpyAsync(order, ctx->solveList.p, sizeof(int) * ctx->nSolve, cudaMemcpyDeviceToHost, ctx->stream));
        CU(cudaStreamSynchronize(ctx->stream));
    }
    return AVBD_OK;
}

int avbd_get_stats(AvbdContext *ctx, AvbdStats *stats)
{
    SETTLED();
    if (ctx)
    {
        ctx->stats.device_steps = ctx->deviceSteps;
        ctx->stats.redone_steps = ctx->redoneSteps;
    }
    if (!ctx || !stats)
        return AVBD_ERR_ARGUMENT;
    *stats = ctx->stats;
    return AVBD_OK;
}

int avbd_device_pose(AvbdContext *ctx, void **position4, void **orientation4)
{
    SETTLED();
    if (!ctx)
        return AVBD_ERR_ARGUMENT;
    if (position4)
        *position4 = ctx->pos.p;
    if (orientation4)
        *orientation4 = ctx->quat.p;
    return AVBD_OK;
}

int avbd_num_primal_variants(int32_t *count, int32_t *group4, int32_t *min_blocks4)
{
    if (count)
        *count = kNumPrimalVariants;
    for (int v = 0; v < kNumPrimalVariants; ++v)
    {
        if (group4)
            group4[v] = kPrimalVariants[v].group;
        if (min_blocks4)
            min_blocks4[v] = kPrimalVariants[v].minBlocks;
    }
    return AVBD_OK;
}

int avbd_set_primal_variant(AvbdContext *ctx, int32_t variant)
{
    SETTLED();
    if (!ctx)
        return AVBD_ERR_ARGUMENT;
    if (variant < 0 || variant >= kNumPrimalVariants)
        return fail(ctx, AVBD_ERR_ARGUMENT, "primal variant %d out of range [0, %d)", variant, kNumPrimalVariants);
    ctx->primalVariant = variant;
    return AVBD_OK;
}

int avbd_autotune(AvbdContext *ctx, int32_t repeats, int32_t *best_variant, float *variant_us)
{
    SETTLED();
    if (!ctx)
        return AVBD_ERR_ARGUMENT;
    if (ctx->errCode)
        return AVBD_ERR_LATCHED;
    if (!ctx->loaded || ctx->nSolve == 0 || (int)ctx->hColourStart.size() < ctx->nColours + 1)
        return fail(ctx, AVBD_ERR_STATE, "autotune needs a stepped world (run avbd_step first)");
    CU(cudaSetDevice(ctx->device));
    int n = ctx->n;
    DArr<float4> savePos, saveQuat, saveDqLin, saveDqAng;
    CHECK(reserve(ctx, savePos, n, false));
    CHECK(reserve(ctx, saveQuat, n, false));
    CHECK(reserve(ctx, saveDqLin, n, false));
    CHECK(reserve(ctx, saveDqAng, n, false));
    CU(cudaMemcpyAsync(savePos.p, ctx->pos.p, sizeof(float4) * n, cudaMemcpyDeviceToDevice, ctx->stream));
    CU(cudaMemcpyAsync(saveQuat.p, ctx->quat.p, sizeof(float4) * n, cudaMemcpyDeviceToDevice, ctx->stream));
    CU(cudaMemcpyAsync(saveDqLin.p, ctx->dqLin.p, sizeof(float4) * n, cudaMemcpyDeviceToDevice, ctx->stream));
    CU(cudaMemcpyAsync(saveDqAng.p, ctx->dqAng.p, sizeof(float4) * n, cudaMemcpyDeviceToDevice, ctx->stream));
    DevBodies B = dev_bodies(ctx);
    DevForces F = dev_forces(ctx);
    Params P = dev_params(ctx->params);
    repeats = std::max(1, repeats);
    int best = ctx->primalVariant;
    float bestUs = 1e30f;
    for (int v = 0; v < kNumPrimalVariants; ++v)
    {
        const PrimalVariant &pv = kPrimalVariants[v];
        int GPB = PRIMAL_BLOCK / pv.group;
        float total = 0.0f;
        for (int r = 0; r <= repeats; ++r)
        {
            CU(cudaEventRecord(ctx->evStart, ctx->stream));
            for (int c = 0; c < ctx->nColours; ++c)
            {
                int first = ctx->hColourStart[c], count = ctx->hColourStart[c + 1] - first;
                if (count > 0)
                    pv.kernel<<<grid_for(count, GPB), PRIMAL_BLOCK, 0, ctx->stream>>>(B, F, P, ctx->solveEntry.p,
                                                                                       first, count);
            }
            CU(cudaGetLastError());
            CU(cudaEventRecord(ctx->evStop, ctx->stream));
            CU(cudaMemcpyAsync(ctx->pos.p, savePos.p, sizeof(float4) * n, cudaMemcpyDeviceToDevice, ctx->stream));
            CU(cudaMemcpyAsync(ctx->quat.p, saveQuat.p, sizeof(float4) * n, cudaMemcpyDeviceToDevice, ctx->stream));
            CU(cudaMemcpyAsync(ctx->dqLin.p, saveDqLin.p, sizeof(float4) * n, cudaMemcpyDeviceToDevice, ctx->stream));
            CU(cudaMemcpyAsync(ctx->dqAng.p, saveDqAng.p, sizeof(float4) * n, cudaMemcpyDeviceToDevice, ctx->stream));
            CU(cudaEventSynchronize(ctx->evStop));
            float ms = 0.0f;
            CU(cudaEventElapsedTime(&ms, ctx->evStart, ctx->evStop));
            if (r > 0) // first run warms caches and instruction memory
                total += ms;
        }
        float us = total * 1e3f / repeats;
        if (variant_us)
            variant_us[v] = us;
        if (us < bestUs)
        {
            bestUs = us;
            best = v;
        }
    }
    CU(cudaStreamSynchronize(ctx->stream));
    release(savePos);
    release(saveQuat);
    release(saveDqLin);
    release(saveDqAng);
    ctx->primalVariant = best;
    if (best_variant)
        *best_variant = best;
    return AVBD_OK;
}

int avbd_set_iteration_mode(AvbdContext *ctx, int32_t mode)
{
    SETTLED();
    if (!ctx)
        return AVBD_ERR_ARGUMENT;
    if (mode != AVBD_ITERATIONS_PER_COLOUR && mode != AVBD_ITERATIONS_PERSISTENT)
        return fail(ctx, AVBD_ERR_ARGUMENT, "unknown iteration mode %d", mode);
    ctx->iterationMode = mode;
    return AVBD_OK;
}

int avbd_iteration_mode(AvbdContext *ctx, int32_t *mode)
{
    if (!ctx || !mode)
        return AVBD_ERR_ARGUMENT;
    // the mode the next step runs in (per-colour launches where the device cannot hold the
    // persistent kernel's blocks)
    *mode = ctx->iterationMode == AVBD_ITERATIONS_PERSISTENT && ctx->iterBlocks > 0 ? AVBD_ITERATIONS_PERSISTENT
                                                                                    : AVBD_ITERATIONS_PER_COLOUR;
    return AVBD_OK;
}

int avbd_set_colouring(AvbdContext *ctx, int32_t mode)
{
    SETTLED();
    if (!ctx)
        return AVBD_ERR_ARGUMENT;
    if (mode != AVBD_COLOUR_GREEDY && mode != AVBD_COLOUR_HASHED)
        return fail(ctx, AVBD_ERR_ARGUMENT, "unknown colouring mode %d", mode);
    ctx->colourMode = mode;
    return AVBD_OK;
}

int avbd_set_profiling(AvbdContext *ctx, int32_t enable)
{
    SETTLED();
    if (!ctx)
        return AVBD_ERR_ARGUMENT;
    ctx->profiling = enable != 0;
    return AVBD_OK;
}

int avbd_read_profile(AvbdContext *ctx, AvbdProfile *out)
{
    SETTLED();
    if (!ctx || !out)
        return AVBD_ERR_ARGUMENT;
    CHECK(prof_collect(ctx));
    out->steps = ctx->stepsProfiled;
    for (int k = 0; k < AVBD_PHASE_COUNT; ++k)
    {
        out->phase_ms[k] = ctx->phaseMs[k];
        out->phase_spans[k] = ctx->phaseLaunches[k];
    }
    out->launches = ctx->launches;
    return AVBD_OK;
}

int avbd_reset_profile(AvbdContext *ctx)
{
    SETTLED();
    if (!ctx)
        return AVBD_ERR_ARGUMENT;
    CHECK(prof_collect(ctx));
    for (int k = 0; k < AVBD_PHASE_COUNT; ++k)
    {
        ctx->phaseMs[k] = 0.0;
        ctx->phaseLaunches[k] = 0;
    }
    ctx->launches = 0;
    ctx->stepsProfiled = 0;
    return AVBD_OK;
}

} // extern "C"

#include "avbd_adjoint.cuh"
