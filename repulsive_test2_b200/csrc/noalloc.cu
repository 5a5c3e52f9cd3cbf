// tpe_energy_noalloc: calculateEnergy for callers that must not allocate.
//
// Some callers cannot call cudaMalloc: an embedding application whose device
// memory is all handed out by its own allocator or pool (a second allocator
// would fragment or overcommit its budget), or a real-time loop that must
// never enter the driver's allocator (cudaMalloc and cudaFree can synchronise
// the whole device and take an unbounded time). This entry point takes device
// pointers for its input and output, creates no context and allocates
// nothing: its scratch (edge records, partial sums and one flag) lives in the
// file-scope device array below, which every GPU that loads the library holds
// until the process exits.
#include <mutex>

#include "tpe_internal.h"

namespace {

// Maximum number of edges the static scratch serves.
constexpr int32_t kMaxEdges = 16384;
// Partial sums: ceil(E/128) edge blocks x at most 16 J chunks.
constexpr int32_t kMaxParts = ((kMaxEdges + 127) / 128) * 16;
constexpr size_t kScratchBytes = 2 * sizeof(double4) * (size_t)kMaxEdges +
                                 sizeof(double) * (size_t)kMaxParts + 256;

// The scratch (1 MiB of edge records, 16 KiB of partials, the bad-index flag).
// In host code this name is only a host-side stand-in: its device address
// comes from cudaGetSymbolAddress, taken once per device below.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_addr[kMaxDevices] = {};

}  // namespace

extern "C" int32_t tpe_energy_noalloc(const double* d_xyz, const int32_t* d_edges, int32_t V,
                                      int32_t E, const tpe_params* p, double* d_energy,
                                      void* stream) {
    return tpe::guarded(nullptr, [&]() -> int32_t {
        if (!d_xyz || !d_edges || !p || !d_energy || V <= 0 || E <= 0) return TPE_ERR_BAD_ARG;
        if (E > kMaxEdges) return TPE_ERR_TOO_LARGE;
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return TPE_ERR_CUDA;
        void* base = nullptr;
        {
            std::lock_guard<std::mutex> lock(g_mu);
            if (!g_addr[dev]) {
                // First call on this device: resolve the device address of the
                // scratch with this device current. The address is kept for the
                // life of the process (cudaDeviceReset is not supported here).
                void* a = nullptr;
                if (cudaGetSymbolAddress(&a, g_scratch) != cudaSuccess || !a) {
                    cudaGetLastError();
                    return TPE_ERR_CUDA;
                }
                g_addr[dev] = a;
            }
            base = g_addr[dev];
        }
        double4* ea = static_cast<double4*>(base);
        double4* eb = ea + kMaxEdges;
        double* partial = reinterpret_cast<double*>(eb + kMaxEdges);
        int32_t* bad = reinterpret_cast<int32_t*>(partial + kMaxParts);
        // Every scratch element read below is written earlier in the same call:
        // the flag is cleared first, the edge records by the prep kernel, one
        // partial per block by the energy kernel.
        return tpe::energy_fp64_scratch(static_cast<cudaStream_t>(stream), d_xyz,
                                        reinterpret_cast<const int2*>(d_edges), V, E, p->alpha,
                                        p->beta, p->epsilon, ea, eb, partial, kMaxParts, bad,
                                        d_energy);
    });
}
