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
// The only scratch the step needs is one FP64 energy partial per thread
// block. It lives in the file-scope array below, a fixed 512 KiB of device
// memory that every GPU which loads this library holds until the process
// exits. Host code must not pass the array's name to a kernel (on the host
// that name is a stand-in, not a device address); the device address is
// looked up once per device with cudaGetSymbolAddress.
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
// Sink for the bounds-check record of the checked library build (unused by
// the regular build), so that no kernel is ever handed a null fault word.
static __device__ __align__(256) unsigned g_noallocFault;

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_noallocMutex;
double *g_noallocAddr[kMaxDevices] = {};
unsigned *g_noallocFaultAddr[kMaxDevices] = {};

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

// Device addresses of the scratch array and the fault sink for the current
// device, looked up on the first call on that device (with that device
// current).
tlm_status scratchForCurrentDevice(double **out, unsigned **fault)
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
    if (!g_noallocAddr[dev])
    {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noallocPartials);
        if (e != cudaSuccess || p == nullptr)
        {
            cudaGetLastError();
            return noallocFail(TLM_ECUDA, std::string("cudaGetSymbolAddress of the scratch array: ") +
                                              cudaGetErrorString(e));
        }
        void *f = nullptr;
        e = cudaGetSymbolAddress(&f, g_noallocFault);
        if (e != cudaSuccess || f == nullptr)
        {
            cudaGetLastError();
            return noallocFail(TLM_ECUDA, std::string("cudaGetSymbolAddress of the fault word: ") +
                                              cudaGetErrorString(e));
        }
        g_noallocAddr[dev] = static_cast<double *>(p);
        g_noallocFaultAddr[dev] = static_cast<unsigned *>(f);
    }
    *out = g_noallocAddr[dev];
    *fault = g_noallocFaultAddr[dev];
    return TLM_OK;
}

bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

} // namespace

extern "C" {

tlm_status tlm_step_planes_noalloc(const float *in_planes, float *out_planes, float *stubs,
                                   const uint8_t *mat, const float *yhat, const float *ghat,
                                   int nx, int ny, int nz, float rho, int input_is_incident,
                                   double *energy_out, void *stream)
{
    if (!in_planes || !out_planes || !mat)
        return noallocFail(TLM_EINVAL, "null pulse planes or material map");
    if (in_planes == out_planes)
        return noallocFail(TLM_EINVAL, "input and output planes must be different buffers");
    if (nx <= 0 || ny <= 0 || nz <= 0)
        return noallocFail(TLM_EINVAL, "grid dimensions must be positive");
    if (!aligned16(in_planes) || !aligned16(out_planes) || (stubs && !aligned16(stubs)) ||
        ((uintptr_t)mat & 3u))
        return noallocFail(TLM_EINVAL, "planes must be 16-byte aligned, the material map 4-byte aligned");
    constexpr int V = kNoAllocV;
    const long long px = (long long)(nx + tlmk::kPadX - 1) / tlmk::kPadX * tlmk::kPadX;
    const long long P = px * ny * nz;
    const long long nq = px / V;
    const long long nquads = nq * ny * nz;
    const long long nblocks = (nquads + tlmk::kBlock - 1) / tlmk::kBlock;
    if (nblocks > kNoAllocMaxBlocks)
        return noallocFail(TLM_EINVAL,
                           "grid has " + std::to_string(P) + " padded nodes; the no-allocation step "
                           "handles at most " +
                               std::to_string((long long)kNoAllocMaxBlocks * tlmk::kBlock * V));
    double *scratch = nullptr;
    unsigned *fault = nullptr;
    tlm_status st = scratchForCurrentDevice(&scratch, &fault);
    if (st != TLM_OK) return st;

    tlmk::StepArgs<float> a;
    a.in = in_planes;
    a.out = out_planes;
    a.stub = stubs;
    a.mat = mat;
    a.yhat = yhat;
    a.ghat = ghat;
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
    a.epart = energy_out ? scratch : nullptr;
    a.e_lo = 0;
    a.e_hi = LLONG_MAX;
    a.fault = fault;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (input_is_incident)
        tlmk::stepKernelShaped<float, kNoAllocV, 3, true, false><<<(unsigned)nblocks, tlmk::kBlock, 0, s>>>(a);
    else
        tlmk::stepKernelShaped<float, kNoAllocV, 3, false, false><<<(unsigned)nblocks, tlmk::kBlock, 0, s>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && energy_out)
    {
        noallocEnergyReduce<<<1, 256, 0, s>>>(scratch, (int)nblocks, energy_out);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess)
        return noallocFail(TLM_ECUDA, std::string("no-allocation step launch: ") + cudaGetErrorString(e));
    return TLM_OK;
}

} // extern "C"
