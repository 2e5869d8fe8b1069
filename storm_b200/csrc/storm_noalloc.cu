// Emission photon allocation that allocates no device memory.
//
// Who needs it: callers that cannot call cudaMalloc while they run -- a host
// framework whose caching allocator owns the device memory, or a real-time
// loop with a no-allocation rule -- but that still want the per-cell photon counts of an emission step computed on the
// GPU from energies already in device memory.  The regular path
// (storm_cuda_phase_emit) keeps its scratch in buffers its handle allocates;
// this variant keeps it in one fixed array in the library image instead.
//
// Scratch: g_allocScratch, a file-scope __device__ array.  Every GPU that loads
// this library holds it (about 128 KiB) until the process exits.  In host code
// the symbol is only a host-side stand-in, so its device address is looked up
// with cudaGetSymbolAddress once per device, with that device current, and the
// address is what the kernels receive.  That set-up happens once, on the first
// call for a device.  Every call
// shares the array: two calls whose work overlaps on the GPU race on it.  Each
// call clears the one word that must start at zero (the ambiguity flag) and
// overwrites the rest of the scratch it reads (the energy total and every tile
// sum) before reading it.  The cached address belongs to the device's context
// as it was at the first call: do not use this entry point across a
// cudaDeviceReset of that device.
//
// The counts floor each cell's share against the reference's left-to-right
// total of the energies.  As in the regular path, a deterministic blocked total
// with a rigorous error interval settles almost every call; where a floor is
// ambiguous the kernels flag it, and two further kernels (which return at once
// when the flag is clear) recompute the exact left-to-right total and the
// counts, all on the device with no host readback.
//
// Errors: the call reports launch errors of its own kernels as STORM_ERR_CUDA.
// If an earlier CUDA error is already pending on the calling thread, it
// launches nothing, leaves that error pending for its owner and returns
// STORM_ERR_CUDA.
#include <cuda_runtime.h>

#include <mutex>

#include "storm_cuda.h"
#include "storm_internal.h"

using namespace storm;

namespace {

constexpr uint32_t kTiles = (STORM_NOALLOC_MAX_CELLS + 1023u) / 1024u;
// layout in 8-byte words: [0] energy total, [1] photon total, [2] ambiguity flag
// (an int32 in the word's first half), [3, 3 + kTiles) tile sums
constexpr size_t kScratchWords = 3 + kTiles;

static __device__ __align__(256) unsigned long long g_allocScratch[kScratchWords];

constexpr int kMaxDevices = 64;
std::mutex g_setupMutex;
void *g_scratchAddr[kMaxDevices] = {};

// Device address of g_allocScratch on `device` (current).  Looked up once per device.
int scratch_address(int device, void **out) {
    std::lock_guard<std::mutex> lock(g_setupMutex);
    if (g_scratchAddr[device] == nullptr) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_allocScratch);
        if (e != cudaSuccess || p == nullptr) return STORM_ERR_CUDA;
        g_scratchAddr[device] = p;
    }
    *out = g_scratchAddr[device];
    return STORM_OK;
}

}  // namespace

extern "C" int storm_cuda_emission_allocation_noalloc(int device, const double *d_energy, uint32_t ncells,
                                                      uint64_t new_photons_per_cell, uint64_t *d_photons,
                                                      uint64_t *d_offsets, void *stream) {
    if (!d_energy || !d_photons || !d_offsets || new_photons_per_cell == 0) return STORM_ERR_INVALID_ARG;
    if (ncells == 0 || ncells > STORM_NOALLOC_MAX_CELLS) return STORM_ERR_INVALID_ARG;
    if (device < 0 || device >= kMaxDevices) return STORM_ERR_INVALID_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return STORM_ERR_NO_DEVICE;
    if (device >= ndev) return STORM_ERR_INVALID_ARG;
    if (cudaPeekAtLastError() != cudaSuccess) return STORM_ERR_CUDA;   // someone else's, left pending
    int previous = 0;
    if (cudaGetDevice(&previous) != cudaSuccess) return STORM_ERR_CUDA;
    if (cudaSetDevice(device) != cudaSuccess) return STORM_ERR_CUDA;
    void *scratch = nullptr;
    int rc = scratch_address(device, &scratch);
    if (rc == STORM_OK) {
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        double *energyTotal = static_cast<double *>(scratch);
        uint64_t *photonTotal = static_cast<uint64_t *>(scratch) + 1;
        int32_t *ambiguous = reinterpret_cast<int32_t *>(static_cast<uint64_t *>(scratch) + 2);
        uint64_t *tileSums = static_cast<uint64_t *>(scratch) + 3;
        Ctx C{};
        C.ncells = ncells;
        CellArrays A{};
        A.emitE = const_cast<double *>(d_energy);
        A.photons = d_photons;
        const double rel = 4.0 * (static_cast<double>(ncells) + 1100.0) * 0x1p-53;   // both orders' rounding
        if (cudaMemsetAsync(ambiguous, 0, sizeof(int32_t), s) != cudaSuccess) rc = STORM_ERR_CUDA;
        if (rc == STORM_OK) {
            launch_blocked_sum(s, d_energy, ncells, energyTotal);
            launch_allocate_checked(s, C, A, energyTotal, new_photons_per_cell, rel, ambiguous);
            launch_sequential_sum_if(s, d_energy, ncells, energyTotal, ambiguous);
            launch_allocate_if(s, C, A, energyTotal, new_photons_per_cell, ambiguous);
            launch_scan_u64(s, d_photons, ncells, d_offsets, tileSums, photonTotal);
            if (cudaGetLastError() != cudaSuccess) rc = STORM_ERR_CUDA;
        }
    }
    cudaSetDevice(previous);
    return rc;
}
