// tlm_noalloc.cu -- one TLM step over caller-owned device memory that
// performs no device allocation of its own.
//
// Who needs it: callers that may not call cudaMalloc/cudaFree. Typical cases
// are a host application that reserves the GPU's memory in its own pool at
// start-up and hands plug-ins only buffers it owns, and a time-critical loop
// that must not pay the implicit device-wide synchronisation that
// cudaMalloc/cudaFree can cause. Such a caller keeps the pulse planes itself
// and asks this entry point to advance them one step.
//
// The scratch the step needs is one FP64 energy partial per thread block and
// a copy of the caller's dielectric tables padded to every possible material
// id (ids past the caller's table read NaN there instead of reading past the
// caller's buffer). They live in the file-scope arrays below, a fixed
// 514 KiB of device memory that every GPU which loads this library holds
// until the process exits. Host code must not pass an array's name to a
// kernel (on the host that name is a stand-in, not a device address); the
// device addresses are looked up once per device with cudaGetSymbolAddress.
#include "tlm_b200.h"

#include "tlm_step_kernel.cuh"

#include <mutex>
#include <string>

// Defined in tlm_solver.cu: the calling thread's message, read back by
// tlm_last_error(NULL).
void tlmSetThreadError(const std::string &m);

// Scratch: one energy partial per step-kernel block. 65,536 blocks of 256
// threads x 4 nodes bound the grid at 67,108,864 padded nodes.
constexpr int kNoAllocMaxBlocks = 65536;
constexpr int kNoAllocV = 4;  // nodes per thread: 65536 blocks x 256 x 4 = 67,108,864 nodes
static __device__ __align__(256) double g_noallocPartials[kNoAllocMaxBlocks];
// Dielectric tables (yhat, ghat) for every material id 2..255: the caller's
// n_diel entries, then NaN.
constexpr int kNoAllocTable = 256 - tlmk::kDiel0;
static __device__ __align__(256) float g_noallocTables[2 * kNoAllocTable];
// Bounds-check record of the checked library build (cleared before every
// step, read back after it there); the regular build never writes it.
static __device__ __align__(256) unsigned g_noallocFault;

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_noallocMutex;

struct NoAllocScratch
{
    double *partials = nullptr;
    float *tables = nullptr;
    unsigned *fault = nullptr;
};
NoAllocScratch g_noallocAddr[kMaxDevices];

tlm_status noallocFail(tlm_status s, const std::string &m)
{
    tlmSetThreadError(m);
    return s;
}

// Fixed-order sum of the block partials into the caller's output.
__global__ void __launch_bounds__(256) noallocEnergyReduce(const double *partials, int n, double *out)
{
    __shared__ double red[tlmk::kBlock / 32];
    double s = 0.0;
    for (int b = threadIdx.x; b < n; b += blockDim.x) s += partials[b];
    const double tot = tlmk::blockSumDouble(s, red);
    if (threadIdx.x == 0) *out = tot;
}

// The caller's yhat/ghat (n entries each) into the padded static tables;
// the entries of ids past the caller's table are NaN, so a node with such an
// id steps to NaN pulses instead of reading past the caller's buffers.
__global__ void __launch_bounds__(kNoAllocTable) noallocTables(const float *yhat, const float *ghat, int n,
                                                               float *tables)
{
    const int t = threadIdx.x;
    if (t >= kNoAllocTable) return;
    tables[t] = t < n ? yhat[t] : __int_as_float(0x7fc00000);
    tables[kNoAllocTable + t] = t < n ? ghat[t] : __int_as_float(0x7fc00000);
}

// Device addresses of the scratch arrays for the current device, looked up
// on the first call on that device (with that device current).
tlm_status scratchForCurrentDevice(NoAllocScratch *out)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    {
        cudaGetLastError();
        return noallocFail(TLM_ENODEV, std::string("no current CUDA device: ") +
                                           (e != cudaSuccess ? cudaGetErrorString(e) : "bad index"));
    }
    std::lock_guard<std::mutex> lk(g_noallocMutex);
    NoAllocScratch &sc = g_noallocAddr[dev];
    if (!sc.partials)
    {
        void *p = nullptr, *t = nullptr, *f = nullptr;
        e = cudaGetSymbolAddress(&p, g_noallocPartials);
        if (e == cudaSuccess) e = cudaGetSymbolAddress(&t, g_noallocTables);
        if (e == cudaSuccess) e = cudaGetSymbolAddress(&f, g_noallocFault);
        if (e != cudaSuccess || !p || !t || !f)
        {
            cudaGetLastError();
            return noallocFail(TLM_ECUDA, std::string("cudaGetSymbolAddress of the scratch arrays: ") +
                                              cudaGetErrorString(e));
        }
        sc.tables = static_cast<float *>(t);
        sc.fault = static_cast<unsigned *>(f);
        sc.partials = static_cast<double *>(p);
    }
    *out = sc;
    return TLM_OK;
}

bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

} // namespace

extern "C" {

tlm_status tlm_step_planes_noalloc(const float *in_planes, float *out_planes, float *stubs,
                                   const uint8_t *mat, const float *yhat, const float *ghat, int n_diel,
                                   int nx, int ny, int nz, float rho, int input_is_incident,
                                   double *energy_out, void *stream)
{
    if (!in_planes || !out_planes || !mat)
        return noallocFail(TLM_EINVAL, "null pulse planes or material map");
    if (in_planes == out_planes)
        return noallocFail(TLM_EINVAL, "input and output planes must be different buffers");
    if (nx <= 0 || ny <= 0 || nz <= 0)
        return noallocFail(TLM_EINVAL, "grid dimensions must be positive");
    if (n_diel < 0 || n_diel > kNoAllocTable)
        return noallocFail(TLM_EINVAL, "n_diel must be in 0.." + std::to_string(kNoAllocTable));
    if (n_diel > 0 && (!stubs || !yhat || !ghat))
        return noallocFail(TLM_EINVAL, "a dielectric table (n_diel > 0) needs stubs, yhat and ghat");
    if (!aligned16(in_planes) || !aligned16(out_planes) || (stubs && !aligned16(stubs)) ||
        ((uintptr_t)mat & 3u))
        return noallocFail(TLM_EINVAL, "planes must be 16-byte aligned, the material map 4-byte aligned");
    constexpr int V = kNoAllocV;
    constexpr long long kMaxNodes = (long long)kNoAllocMaxBlocks * tlmk::kBlock * V;
    // the plane size grows one factor at a time, each partial product
    // checked against the limit, so nothing overflows
    const long long px = ((long long)nx + tlmk::kPadX - 1) / tlmk::kPadX * tlmk::kPadX;
    const long long row = px <= kMaxNodes ? px * ny : kMaxNodes + 1;
    const long long P = row <= kMaxNodes ? row * nz : kMaxNodes + 1;
    if (P <= 0 || P > kMaxNodes)
        return noallocFail(TLM_EINVAL,
                           "grid has more than " + std::to_string(kMaxNodes) + " padded nodes; the no-allocation "
                           "step handles at most " + std::to_string(kMaxNodes));
    const long long nq = px / V;
    const long long nquads = nq * ny * nz;
    const long long nblocks = (nquads + tlmk::kBlock - 1) / tlmk::kBlock;
    if (nblocks <= 0 || nblocks > kNoAllocMaxBlocks)
        return noallocFail(TLM_EINVAL, "grid block count out of range");
    NoAllocScratch sc;
    tlm_status st = scratchForCurrentDevice(&sc);
    if (st != TLM_OK) return st;

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    noallocTables<<<1, kNoAllocTable, 0, s>>>(yhat, ghat, n_diel, sc.tables);
    cudaError_t e = cudaGetLastError();
#ifdef TLM_CHECKED
    if (e == cudaSuccess) e = cudaMemsetAsync(sc.fault, 0, sizeof(unsigned), s);
#endif
    if (e != cudaSuccess)
        return noallocFail(TLM_ECUDA, std::string("no-allocation step set-up: ") + cudaGetErrorString(e));

    tlmk::StepArgs<float> a;
    a.in = in_planes;
    a.out = out_planes;
    a.stub = stubs;
    a.mat = mat;
    a.yhat = sc.tables;
    a.ghat = sc.tables + kNoAllocTable;
    a.P = P;
    a.nquads = nquads;
    a.nx = nx;
    a.ny = ny;
    a.nz = nz;
    a.px = (int)px;
    a.nq = (int)nq;
    a.div_nq = tlmk::makeFastDiv((unsigned)nq);
    a.div_ny = tlmk::makeFastDiv((unsigned)ny);
    a.rho = rho;
    a.scale = 1.0f;
    a.inv_scale = 1.0f;
    a.tile_begin = nullptr;
    a.spec = nullptr;
    a.tile_flags = nullptr;  // every tile takes the general body
    a.neg_zero = -0.0f;
    a.sv = 0.0f;
    a.samples = nullptr;
    a.epart = energy_out ? sc.partials : nullptr;
    a.e_lo = 0;
    a.e_hi = LLONG_MAX;
    a.fault = sc.fault;
    a.stage_wait_ns = tlmk::kStageWaitNs;
    if (input_is_incident)
        tlmk::stepKernelShaped<float, kNoAllocV, 3, true, false><<<(unsigned)nblocks, tlmk::kBlock, 0, s>>>(a);
    else
        tlmk::stepKernelShaped<float, kNoAllocV, 3, false, false><<<(unsigned)nblocks, tlmk::kBlock, 0, s>>>(a);
    e = cudaGetLastError();
    if (e == cudaSuccess && energy_out)
    {
        noallocEnergyReduce<<<1, 256, 0, s>>>(sc.partials, (int)nblocks, energy_out);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess)
        return noallocFail(TLM_ECUDA, std::string("no-allocation step launch: ") + cudaGetErrorString(e));
#ifdef TLM_CHECKED
    // the checked build reports an index outside a buffer (and skips that
    // access): wait for the step and read the record back
    unsigned f = 0;
    e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = cudaMemcpy(&f, sc.fault, sizeof(unsigned), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return noallocFail(TLM_ECUDA, std::string("no-allocation step: ") + cudaGetErrorString(e));
    if (f) return noallocFail(TLM_ECUDA, "bounds check tripped in the no-allocation step, code mask " + std::to_string(f));
#endif
    return TLM_OK;
}

} // extern "C"
