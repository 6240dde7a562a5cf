// sc_noalloc.cu -- the open-boundary Poisson solve for callers that cannot
// allocate device memory.
//
// Some callers cannot call cudaMalloc: host frameworks that own every byte
// of device memory through their own pool allocator (a plugin may only use
// the buffers it is handed), and latency-critical loops where the implicit
// device-wide synchronisation of cudaMalloc/cudaFree is not acceptable.  For
// them, scgpu_compute_potential_noalloc solves on caller-provided device
// buffers and keeps its scratch (the half spectrum, the Green's function and
// its transform, and the solver scalars) in one file-scope device array of
// fixed size, beside a file-scope table of twiddle factors.  Both are part
// of the library image: every GPU that loads the library holds them until
// the process exits.
#include <cmath>
#include <mutex>
#include <string>
#include <vector>

#include "scgpu.h"
#include "sc_internal.h"

namespace sc {
namespace {

constexpr size_t kScratchBytes = 4u << 20;  // 4 MiB
constexpr int kMaxCellsPerAxis = 32;        // 64-point doubled axes
constexpr int kMinCellsPerAxis = 3;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Twiddle factors of every doubled-axis length 2n, n in [3, 32], one table
// after the other: the values the allocating path uploads per context, so
// both entry points compute the same bits.  Written once per device.
constexpr int tw_offset(int L) {  // entries before length L (L even, >= 6)
    return (L / 2 - kMinCellsPerAxis) * (L / 2 + kMinCellsPerAxis - 1);
}
constexpr int kTwEntries = tw_offset(2 * kMaxCellsPerAxis + 2);
static __device__ __align__(256) double2 g_twiddles[kTwEntries];

// Host code must not use g_scratch or g_twiddles as addresses: on the host
// the names only stand in for the symbols.  Their device addresses are
// looked up once per device, with that device current.
std::mutex g_mutex;
struct DeviceSetup {
    void* scratch = nullptr;
    double2* twiddles = nullptr;
};
DeviceSetup g_setup[kMaxDevices];

int device_setup(int device, DeviceSetup* out) {
    if (device < 0 || device >= kMaxDevices) return SCGPU_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_mutex);
    DeviceSetup& d = g_setup[device];
    if (!d.scratch) {
        void* p = nullptr;
        void* t = nullptr;
        if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess || !p ||
            cudaGetSymbolAddress(&t, g_twiddles) != cudaSuccess || !t) {
            cudaGetLastError();
            return SCGPU_ERR_CUDA;
        }
        std::vector<double2> tw(kTwEntries);
        for (int n = kMinCellsPerAxis; n <= kMaxCellsPerAxis; ++n)
            twiddle_values(2 * n, tw.data() + tw_offset(2 * n), nullptr);
        // synchronous, from pageable memory: nothing is allocated
        if (cudaMemcpyToSymbol(g_twiddles, tw.data(), kTwEntries * sizeof(double2)) != cudaSuccess) {
            cudaGetLastError();
            return SCGPU_ERR_CUDA;
        }
        d.twiddles = static_cast<double2*>(t);
        d.scratch = p;
    }
    *out = d;
    return SCGPU_OK;
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
        if (!(hr[d] > 0.0) || !std::isfinite(hr[d])) return SCGPU_ERR_ARG;
    const int n[3] = {nx, ny, nz};
    for (int d = 0; d < 3; ++d)
        if (n[d] < kMinCellsPerAxis || n[d] > kMaxCellsPerAxis || make_plan(2 * n[d]).nst <= 0)
            return SCGPU_ERR_UNSUPPORTED;
    // carve the scratch: spectrum, G antiderivative, G, its transform, scalars
    const size_t S = (size_t)(nz + 1) * (2 * ny) * (2 * nx);
    const size_t T3 = (size_t)(nx + 2) * (ny + 2) * (nz + 2);
    const size_t G3 = (size_t)(nx + 1) * (ny + 1) * (nz + 1);
    size_t off[5], o = 0;
    off[0] = o; o = up256(o + S * sizeof(double2));
    off[1] = o; o = up256(o + T3 * sizeof(double));
    off[2] = o; o = up256(o + G3 * sizeof(double));
    off[3] = o; o = up256(o + G3 * sizeof(double));
    off[4] = o; o = up256(o + sizeof(StepState));
    if (o > kScratchBytes) return SCGPU_ERR_UNSUPPORTED;

    // An error left pending by the caller's own earlier CUDA work is not
    // taken for this call's, nor cleared: nothing is enqueued.
    if (cudaPeekAtLastError() != cudaSuccess) return SCGPU_ERR_CUDA;
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return SCGPU_ERR_CUDA;
    const size_t M = (size_t)nx * ny * nz;
    std::string why;
    if (!device_buffer_ok(rho_dev, M * sizeof(double), device, &why) ||
        !device_buffer_ok(phi_dev, M * sizeof(double), device, &why))
        return SCGPU_ERR_ARG;
    DeviceSetup ds;
    int rc = device_setup(device, &ds);
    if (rc) return rc;
    unsigned char* p = static_cast<unsigned char*>(ds.scratch);
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
    for (int d = 0; d < 3; ++d) b.tw[d] = ds.twiddles + tw_offset(2 * n[d]);
    b.st = reinterpret_cast<StepState*>(p + off[4]);

    // Nothing in the scratch has to start at zero: every element a stage
    // reads was written earlier in the same call (the pruned passes never
    // read the spectrum outside the part the previous pass wrote).
    k_noalloc_hr<<<1, 1, 0, s>>>(b.st, hr[0], hr[1], hr[2]);
    launch_igf(b, nullptr, s);
    launch_green_transform(b, s);
    launch_convolution(b, kConvPotential, s);
    // no error was pending at entry, so one now is this call's (work may be
    // partly enqueued)
    if (cudaGetLastError() != cudaSuccess) return SCGPU_ERR_CUDA;
    return SCGPU_OK;
}
