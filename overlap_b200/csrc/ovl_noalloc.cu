// ovl_ncsdot_noalloc: the Chern-Simons rate NCsDot of device-resident fields,
// for callers that must not allocate device memory.
//
// Who needs it: code that runs where an allocation is not allowed or not
// wanted -- a time-step loop that must never block on cudaMalloc (which can
// synchronise the device), a caller whose device memory is owned by another
// allocator that has already reserved it, or a caller between the set-up and
// the replay of captured work.  Such a caller owns its inputs and its output
// and only needs the reduction.
//
// Scratch: the partial sums live in the file-scope device array below, one
// double per block of 256 sites, at most kNoAllocPartials of them, so the
// entry point accepts lattices of up to kNoAllocPartials * 256 = 262144 sites
// (64^3) and rejects larger ones with OVL_E_ARG.  The array is 8 KiB of device
// memory that every GPU loading this library holds until the process exits.
// Every call overwrites exactly the partial sums it then reads, so nothing has
// to start at zero; all calls share the one array, so calls whose work
// overlaps on the GPU (different streams, or different host threads on the
// same device) race and must be serialised by the caller.
//
// Set-up: the first call on each device, with that device current, looks up
// the array's device address (cudaGetSymbolAddress) and caches it.  Make that
// first call before any stream capture begins.  Devices with an ordinal of 64
// or more are not served (OVL_E_UNSUPPORTED).
//
// Errors: an error already pending in the runtime from other work is left in
// place and not reported as this call's; a launch of this call that fails is
// reported as OVL_E_CUDA and its error cleared.

#include <mutex>

#include "ovl.h"
#include "ovl_device.cuh"
#include "ovl_internal.h"

namespace {

constexpr int kNoAllocPartials = 1024;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_ncsdot_partials[kNoAllocPartials];

std::mutex g_setup_mutex;
double *g_partials_addr[kMaxDevices] = {};

}  // namespace

extern "C" int ovl_ncsdot_noalloc(const double *links, const double *efield, int N0, int N1, int N2, double *out,
                                  uint64_t stream) {
    if (!links || !efield || !out) return OVL_E_ARG;
    if (N0 < 3 || N1 < 3 || N2 < 3) return OVL_E_ARG;
    const long long V = (long long)N0 * N1 * N2;
    if (V > (long long)kNoAllocPartials * 256) return OVL_E_ARG;  // beyond the scratch array
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return OVL_E_CUDA;
    if (dev < 0 || dev >= kMaxDevices) return OVL_E_UNSUPPORTED;
    double *partials = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_partials_addr[dev]) {
            void *addr = nullptr;
            if (cudaGetSymbolAddress(&addr, g_ncsdot_partials) != cudaSuccess) return OVL_E_CUDA;
            g_partials_addr[dev] = static_cast<double *>(addr);
        }
        partials = g_partials_addr[dev];
    }
    const ovl::Lattice L{N0, N1, N2, (int)V};
    const int blocks = ovl::ncsdot_blocks_exact(L);
    // the runtime's last error before and after the launches: a change is this
    // call's failure; an error that was already there belongs to earlier work
    const cudaError_t before = cudaPeekAtLastError();
    ovl::launch_ncsdot_into(links, efield, L, blocks, partials, out, reinterpret_cast<cudaStream_t>(stream));
    const cudaError_t after = cudaPeekAtLastError();
    if (after != before) {
        cudaGetLastError();
        return OVL_E_CUDA;
    }
    return OVL_OK;
}
