// sc_noalloc.cu -- the open-boundary Poisson solve for callers that cannot
// allocate device memory.
//
// Some callers cannot call cudaMalloc: host frameworks that own every byte
// of device memory through their own pool allocator (a plugin may only use
// the buffers it is handed), and latency-critical loops where the implicit
// device-wide synchronisation of cudaMalloc/cudaFree is not acceptable.  For
// them, scgpu_compute_potential_noalloc solves on caller-provided device
// buffers and keeps its scratch (the half spectrum, the Green's function and
// its transform, twiddles and the solver scalars) in one file-scope device
// array of fixed size.  That array is part of the library image: every GPU
// that loads the library holds it until the process exits.
#include <mutex>

#include "scgpu.h"
#include "sc_internal.h"

namespace sc {
namespace {

constexpr size_t kScratchBytes = 4u << 20;  // 4 MiB
constexpr int kMaxCellsPerAxis = 32;        // 64-point doubled axes
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Host code must not use g_scratch as an address: on the host the name only
// stands in for the symbol.  Its device address is looked up once per device.
std::mutex g_mutex;
void* g_scratch_dev[kMaxDevices] = {};

int scratch_address(int device, void** out) {
    if (device < 0 || device >= kMaxDevices) return SCGPU_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_dev[device]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess || !p) {
            cudaGetLastError();
            return SCGPU_ERR_CUDA;
        }
        g_scratch_dev[device] = p;
    }
    *out = g_scratch_dev[device];
    return SCGPU_OK;
}

__global__ void k_noalloc_twiddles(double2* tw, int L) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < L; e += gridDim.x * blockDim.x) {
        double s, c;
        sincospi(-2.0 * (double)e / (double)L, &s, &c);
        tw[e] = make_double2(c, s);
    }
}

__global__ void k_noalloc_hr(StepState* st, double h0, double h1, double h2) {
    st->hr_scaled[0] = h0;
    st->hr_scaled[1] = h1;
    st->hr_scaled[2] = h2;
}

inline size_t up256(size_t v) { return (v + 255) & ~size_t(255); }

}  // namespace
}  // namespace sc

using namespace sc;

extern "C" int scgpu_compute_potential_noalloc(const double* rho_dev, double* phi_dev, int nx, int ny, int nz,
                                               const double hr[3], void* cuda_stream) {
    if (!rho_dev || !phi_dev || !hr) return SCGPU_ERR_ARG;
    for (int d = 0; d < 3; ++d)
        if (!(hr[d] > 0.0) || !(hr[d] < 1e300)) return SCGPU_ERR_ARG;
    const int n[3] = {nx, ny, nz};
    for (int d = 0; d < 3; ++d)
        if (n[d] < 3 || n[d] > kMaxCellsPerAxis || make_plan(2 * n[d]).nst <= 0) return SCGPU_ERR_UNSUPPORTED;
    // carve the scratch: spectrum, G antiderivative, G, its transform, twiddles, scalars
    const size_t S = (size_t)(nz + 1) * (2 * ny) * (2 * nx);
    const size_t T3 = (size_t)(nx + 2) * (ny + 2) * (nz + 2);
    const size_t G3 = (size_t)(nx + 1) * (ny + 1) * (nz + 1);
    size_t off[8], o = 0;
    off[0] = o; o = up256(o + S * sizeof(double2));
    off[1] = o; o = up256(o + T3 * sizeof(double));
    off[2] = o; o = up256(o + G3 * sizeof(double));
    off[3] = o; o = up256(o + G3 * sizeof(double));
    for (int d = 0; d < 3; ++d) {
        off[4 + d] = o;
        o = up256(o + (size_t)(2 * n[d]) * (sizeof(double2) + sizeof(float2)));
    }
    off[7] = o; o = up256(o + sizeof(StepState));
    if (o > kScratchBytes) return SCGPU_ERR_UNSUPPORTED;

    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return SCGPU_ERR_CUDA;
    void* base = nullptr;
    int rc = scratch_address(device, &base);
    if (rc) return rc;
    unsigned char* p = static_cast<unsigned char*>(base);
    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);

    DevBunch b{};
    b.precision = SCGPU_PLAIN_FP64;
    b.bc.n[0] = nx;
    b.bc.n[1] = ny;
    b.bc.n[2] = nz;
    b.rho = const_cast<double*>(rho_dev);
    b.phi = phi_dev;
    b.spec = p + off[0];
    b.gtmp = reinterpret_cast<double*>(p + off[1]);
    b.gline = reinterpret_cast<double*>(p + off[2]);
    b.ghat = p + off[3];
    for (int d = 0; d < 3; ++d) b.tw[d] = p + off[4 + d];
    b.st = reinterpret_cast<StepState*>(p + off[7]);

    // Nothing in the scratch has to start at zero: every element a stage
    // reads was written earlier in the same call (the pruned passes never
    // read the spectrum outside the part the previous pass wrote).
    for (int d = 0; d < 3; ++d) k_noalloc_twiddles<<<1, 256, 0, s>>>(reinterpret_cast<double2*>(b.tw[d]), 2 * n[d]);
    k_noalloc_hr<<<1, 1, 0, s>>>(b.st, hr[0], hr[1], hr[2]);
    launch_igf(b, nullptr, s);
    launch_green_transform(b, s);
    launch_convolution(b, kConvPotential, s);
    if (cudaGetLastError() != cudaSuccess) return SCGPU_ERR_CUDA;
    return SCGPU_OK;
}
