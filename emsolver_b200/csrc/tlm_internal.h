// tlm_internal.h -- internals shared by the translation units of the library
// (the solver handle, its helpers); not part of the C ABI.
#pragma once

#include "tlm_b200.h"
#include "tlm_device.cuh"

#include <atomic>
#include <type_traits>
#include <string>
#include <vector>

namespace tlmi {
struct PortInfo
{
    std::vector<uint64_t> cells;  // kept (air) cells, caller order
    int pol = 2;
    float amp = 1.0f;
    long long nb[4] = { -1, -1, -1, -1 };  // reference linear indices of the current loop
};
struct SourceInfo
{
    uint64_t cell;
    int pol;
    float amp;
};

// Scoped device selection that restores the caller's current device.
struct DeviceGuard
{
    int prev = -1;
    explicit DeviceGuard(int dev)
    {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard()
    {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

inline size_t storageBytes(int storage)
{
    switch (storage)
    {
    case TLM_STORE_F64: return 8;
    case TLM_STORE_BF16:
    case TLM_STORE_F16:
    case TLM_STORE_BFP16: return 2;
    default: return 4;
    }
}
inline size_t realBytes(int storage) { return storage == TLM_STORE_F64 ? 8 : 4; }

// Step-kernel tile shapes per storage mode: {nodes per thread V, min blocks
// per SM, scatter style}. Entry 0 is the default (tlmk::Traits<S>, the
// fastest shape measured on B200 for the 192^3 heterogeneous grid); the
// autotuner and tlm_config.kernel_variant pick among the others.
struct Shape
{
    int V, minb;
    int select;  // 1: warp-uniform select between air and stub scatter; 0: per-node branch
};
constexpr Shape kShapesF32[] = { { 2, 4, 1 }, { 4, 3, 1 }, { 4, 3, 0 }, { 4, 2, 0 } };
constexpr Shape kShapesF64[] = { { 1, 4, 1 }, { 1, 4, 0 }, { 2, 3, 0 } };
constexpr Shape kShapesHalf[] = { { 4, 3, 1 }, { 4, 3, 0 }, { 2, 4, 1 }, { 8, 2, 0 }, { 4, 2, 1 } };
// block floating point: a thread owns whole 4-node groups
constexpr Shape kShapesBfp[] = { { 4, 3, 1 }, { 4, 3, 0 }, { 4, 2, 0 } };

template <class S> struct ShapeTable;
template <> struct ShapeTable<float>
{
    static constexpr const Shape *v = kShapesF32;
    static constexpr int n = sizeof(kShapesF32) / sizeof(Shape);
};
template <> struct ShapeTable<double>
{
    static constexpr const Shape *v = kShapesF64;
    static constexpr int n = sizeof(kShapesF64) / sizeof(Shape);
};
template <> struct ShapeTable<__half>
{
    static constexpr const Shape *v = kShapesHalf;
    static constexpr int n = sizeof(kShapesHalf) / sizeof(Shape);
};
template <> struct ShapeTable<__nv_bfloat16>
{
    static constexpr const Shape *v = kShapesHalf;
    static constexpr int n = sizeof(kShapesHalf) / sizeof(Shape);
};
template <> struct ShapeTable<tlmk::Bfp4>
{
    static constexpr const Shape *v = kShapesBfp;
    static constexpr int n = sizeof(kShapesBfp) / sizeof(Shape);
};

// Entry 0 of every table is the storage type's default kernel shape.
template <class S> constexpr bool defaultShapeMatches()
{
    return ShapeTable<S>::v[0].V == tlmk::Traits<S>::V && ShapeTable<S>::v[0].minb == tlmk::Traits<S>::kMinBlocks &&
           (ShapeTable<S>::v[0].select != 0) == tlmk::Traits<S>::kSelect;
}
static_assert(defaultShapeMatches<float>() && defaultShapeMatches<double>() && defaultShapeMatches<__half>() &&
                  defaultShapeMatches<__nv_bfloat16>() && defaultShapeMatches<tlmk::Bfp4>(),
              "entry 0 of a shape table must be the Traits default");

// Calls f(V, MINB, SEL) (std::integral_constant arguments) for shape
// `variant` of storage type S; the one place where table entries become
// kernel template arguments.
template <class S, int I = 0, class F> void withShape(int variant, F &&f)
{
    if constexpr (I < ShapeTable<S>::n)
    {
        if (variant == I)
        {
            constexpr Shape sh = ShapeTable<S>::v[I];
            f(std::integral_constant<int, sh.V>{}, std::integral_constant<int, sh.minb>{},
              std::integral_constant<bool, sh.select != 0>{});
        }
        else
            withShape<S, I + 1>(variant, f);
    }
}

inline int shapeCount(int storage)
{
    switch (storage)
    {
    case TLM_STORE_F64: return ShapeTable<double>::n;
    case TLM_STORE_BF16:
    case TLM_STORE_F16: return ShapeTable<__half>::n;
    case TLM_STORE_BFP16: return ShapeTable<tlmk::Bfp4>::n;
    case TLM_STORE_F32: return ShapeTable<float>::n;
    default: return 0;
    }
}
inline Shape shapeOf(int storage, int variant)
{
    switch (storage)
    {
    case TLM_STORE_F64: return kShapesF64[variant];
    case TLM_STORE_BF16:
    case TLM_STORE_F16: return kShapesHalf[variant];
    case TLM_STORE_BFP16: return kShapesBfp[variant];
    default: return kShapesF32[variant];
    }
}

} // namespace tlmi

namespace tlmi {
// Surface monitors of one handle (TlmSolver.cpp:303-348, 616-675, 715-763):
// PEC-face surface currents, Huygens-box phasors, |E| cut plane, frames.
struct SurfaceState
{
    // face lists in the reference's order (reference linear cell indices)
    std::vector<uint64_t> jsCell;
    std::vector<int> jsAxis, jsSign;
    std::vector<float> jsCenter;  // 3 per face
    std::vector<uint64_t> huyCell;
    std::vector<int> huyAxis, huySign;
    std::vector<float> huyPos;  // 3 per face, relative to the domain centre
    // device copies and accumulators (element type: the storage's real type)
    long long *dJsNode = nullptr, *dHuyNode = nullptr;  // node * 8 + axis * 2 + (sign < 0)
    void *dJsInst = nullptr, *dJsAcc = nullptr, *dHuyAcc = nullptr;
    // cut plane (set by tlm_set_field_plane)
    int planeAxis = -1, planeIndex = 0;
    int planeN1 = 0, planeN2 = 0, planeAxisDone = -1, planeIndexDone = 0;
    bool planeValid = false;
    void *dPlane = nullptr;
    size_t planeCap = 0;  // elements
    // playback frames
    struct Frame
    {
        int step, hasPlane, axis, index, n1, n2;
        size_t off;  // element offset in dFrames
    };
    std::vector<Frame> frames;
    void *dFrames = nullptr;
    size_t framesCap = 0, framesUsed = 0;  // elements
};
} // namespace tlmi

struct tlm_solver
{
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaMemPool_t pool = nullptr;
    std::string err;

    std::atomic<bool> running{ false };
    std::atomic<bool> finished{ false };
    std::atomic<bool> stopFlag{ false };
    std::atomic<int> doneStep{ 0 };
    std::atomic<float> energy{ 0.0f };

    // configuration
    bool configured = false;
    tlm_grid g{};
    tlm_config cfg{};
    int storage = TLM_STORE_F32;
    std::vector<uint8_t> mat;
    std::vector<float> epsr, sigma;
    std::vector<float> yhat32, ghat32;
    std::vector<double> yhat64, ghat64;
    int nx = 0, ny = 0, nz = 0, px = 0, V = 4, nq = 0;
    long long P = 0, ncell = 0, nquads = 0;
    int nblocks = 0;
    bool anyDiel = false;
    float dt32 = 0.0f;
    double dt64 = 0.0;
    float scale = 1.0f;
    int window = 64;
    int variant = 0;

    // sources and monitors
    std::vector<tlmi::SourceInfo> sources;
    std::vector<tlmi::PortInfo> ports;
    std::vector<uint64_t> probeCells;
    std::vector<float> svTable;
    std::vector<double> dftFreqs;
    bool prepared = false;
    int nsamp = 0;
    int specCount = 0;     // entries of dSpec

    // time-loop state
    int curStep = 0;       // steps enqueued
    // host copies of the probe and port records, read back once after steps
    // and served to every getter until more steps are enqueued or the state
    // is rewound (recVersion moves then)
    unsigned long long recVersion = 1, recHostVersion = 0;
    int recHostSteps = 0;
    std::vector<double> precHost, vrecHost, irecHost;
    int curBuf = 0;        // pulse buffer holding the current state
    bool stateIncident = false;

    // z-slab of a grid split over several solvers (tlm_set_slab): the first
    // and/or last plane is a ghost copy of the neighbouring slab's plane
    int ghostLo = 0, ghostHi = 0;

    // device memory
    void *dPulses[2] = { nullptr, nullptr };
    // near-field box of 16-bit storage (tlm_config.near_field): its extent
    // (nearBox.bP == 0: none) and the residual planes beside each pulse buffer
    tlmk::NearBox nearBox{};
    float *dLo[2] = { nullptr, nullptr };
    void *dStub = nullptr;
    uint8_t *dMat = nullptr;
    void *dYhat = nullptr, *dGhat = nullptr;
    tlmk::SpecEntry *dSpec = nullptr;
    int *dTile = nullptr;
    uint8_t *dTileFlags = nullptr;  // per step-kernel tile: tlmk::kTileGeneral / kTileDiel / kTileEdge
    int *dStaged = nullptr, *dListed = nullptr;  // tiles of the staged kernel / of the list kernel
    int nStaged = 0, nListed = 0, stagedGrid = 0;
    bool sparseStaged = false;  // a staged tile is a sparse-stub tile (FP32)
    // host copies (a batch builds its tile tables from them); staged and edge
    // tiles as packed entries (tlmk::packStagedEntry: tile | flags << 24)
    std::vector<int> stagedTiles, listedTiles;
    std::vector<int> edgeTiles;                 // interior tiles on an outer face (listed alone, staged in a batch)
    cudaStream_t side = nullptr;      // the list kernel's stream (forked from and joined to `stream`)
    cudaEvent_t evFork = nullptr, evJoin = nullptr;
    // z-slab steps in two phases (tlm_slab_step_begin / _end): tile lists of
    // the own planes next to a ghost plane (boundary), of the other own
    // planes (interior: listed, and staged as packed entries), the stream
    // the halo messages travel on, and the open launch window
    bool slabLists = false;
    int *dSlabB = nullptr, *dSlabI = nullptr, *dSlabS = nullptr;
    int nSlabB = 0, nSlabI = 0, nSlabS = 0, slabStagedGrid = 0;
    cudaStream_t halo = nullptr;
    cudaEvent_t evBoundary = nullptr, evHalo = nullptr;
    bool slabBegun = false, slabOpen = false;
    int slabPos = 0;
    long long slabBase = 0, slabEFirst = 0;
    std::vector<uint8_t> tileFlagsHost;
    void *dSamples = nullptr;
    double *dEpart = nullptr;
    int *dPortOff = nullptr, *dPortSlots = nullptr, *dPortPol = nullptr, *dPortNb = nullptr;
    int *dProbeSlot = nullptr;
    double *dVrec = nullptr, *dIrec = nullptr, *dPrec = nullptr;
    long long recCap = 0;
    double *dEhist = nullptr;
    double *dElatest = nullptr;
    double *dWdt = nullptr, *dDft = nullptr;
    unsigned *dFault = nullptr;
    size_t devBytes = 0;

    // batched execution (tlm_batch_*): the batch that drives this handle, and
    // the per-step source values the batched kernel reads from device memory
    struct tlm_batch_s *batch = nullptr;
    void *dSv = nullptr;
    long long svCount = 0;

    // surface monitors
    tlmi::SurfaceState surf;

    // kernel timing
    bool timing = false;
    std::vector<cudaEvent_t> evs;
    size_t evUsed = 0;

    tlm_status fail(tlm_status s, const std::string &m)
    {
        err = m;
        return s;
    }
    tlm_status cuda(cudaError_t e, const char *what)
    {
        if (e == cudaSuccess) return TLM_OK;
        err = std::string(what) + ": " + cudaGetErrorString(e);
        return e == cudaErrorMemoryAllocation ? TLM_ENOMEM : TLM_ECUDA;
    }
};

#define TLM_TRY(expr)                                  \
    do                                                 \
    {                                                  \
        tlm_status _s = (expr);                        \
        if (_s != TLM_OK) return _s;                   \
    } while (0)
#define TLM_CU(h, call) TLM_TRY((h)->cuda((call), #call))

namespace tlmi {

// Device memory of a handle comes from a per-device stream-ordered pool that
// keeps freed blocks for reuse (no device-wide synchronisation and no
// driver round trip per allocation), ordered on the handle's stream.
template <class T> tlm_status devAlloc(tlm_solver *h, T **p, size_t bytes)
{
    *p = nullptr;
    if (bytes == 0) return TLM_OK;
    void *q = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&q, bytes, h->pool, h->stream);
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        return h->fail(TLM_ENOMEM, "device allocation of " + std::to_string(bytes) +
                                       " bytes failed: " + cudaGetErrorString(e));
    }
    h->devBytes += bytes;
    *p = static_cast<T *>(q);
    return TLM_OK;
}
// Short-lived buffers of one API call (not counted in the handle's bytes).
template <class T> tlm_status tmpAlloc(tlm_solver *h, T **p, size_t bytes)
{
    void *q = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&q, bytes > 0 ? bytes : 1, h->pool, h->stream);
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        *p = nullptr;
        return h->fail(TLM_ENOMEM, std::string("temporary device allocation failed: ") +
                                       cudaGetErrorString(e));
    }
    *p = static_cast<T *>(q);
    return TLM_OK;
}
template <class T> void devFree(tlm_solver *h, T *&p)
{
    if (p) cudaFreeAsync((void *)p, h->stream);
    p = nullptr;
}

// Defined in tlm_solver.cu.
void setThreadError(const std::string &m);
void freeMonitors(tlm_solver *h);
void freeAll(tlm_solver *h);
bool busy(tlm_solver *h);
double sourceValue(const tlm_solver *h, int n);
long long paddedNode(const tlm_solver *h, uint64_t cell);
tlm_status prepare(tlm_solver *h);
tlm_status ensureRecords(tlm_solver *h, long long need);
tlm_status syncState(tlm_solver *h);
tlm_status checkHandle(tlm_solver *h);
tlm_status checkReady(tlm_solver *h);
tlm_status chooseScale(tlm_solver *h);
int gridBlocksFor(long long n);
// Batched execution support (defined in tlm_solver.cu).
tlm_status uploadSourceTable(tlm_solver *h, long long steps);
tlm_status setWindow(tlm_solver *h, int window);
tlm_status rewind(tlm_solver *h);
tlm_status reshape(tlm_solver *h, int variant);
// Surface monitors (defined in tlm_surface.cu).
void buildFaceLists(int nx, int ny, int nz, const float origin[3], float dl, const uint8_t *mat, bool surfaceOn,
                    int huyOffset, SurfaceState &s);
struct FarField
{
    float uMax = 0, directivity = 0, peakTheta = 0, peakPhi = 0;
};
tlm_status farFieldTransform(cudaStream_t stream, cudaMemPool_t pool, bool f64, const void *dAcc,
                             const long long *dCode, const float *hostPos, int nh, float f0, int n_theta,
                             int n_phi, float *U, FarField &out, std::string &err);
void buildSurfaceLists(tlm_solver *h);
tlm_status prepareSurface(tlm_solver *h);
void freeSurface(tlm_solver *h);
tlm_status rewindSurface(tlm_solver *h);
bool surfaceActive(const tlm_solver *h);
tlm_status launchSurface(tlm_solver *h, int n);
// The library's memory pool on a device (created on first use), the bytes it
// could hand out (free device memory plus blocks it keeps for reuse), and
// whether the blocks it keeps alone hold `bytes`.
cudaMemPool_t devicePool(int device);
size_t poolAvailable(int device);
bool poolCovers(int device, size_t bytes);

} // namespace tlmi
