// Morton ordering that allocates nothing: ob_morton_order_noalloc.
//
// Some callers cannot allocate device memory at the moment they need an
// ordering: callers that hand out device memory only from their own fixed pool
// and forbid other allocations, and long-running services that must not
// fragment or grow the device heap once they are up (a cudaMalloc can also
// synchronise the device, which such a service's other streams would feel).
// This entry point serves them: the caller
// passes device memory for the inputs and the outputs, and every intermediate
// buffer the ordering needs -- the second key/index buffer of the radix sort,
// the digit histograms, the onesweep look-back words and tile tickets, the
// bounding-cube partials -- lives in one file-scope __device__ array of fixed
// size, allocated by the CUDA runtime when the library is loaded on a device
// and held by every device that loads it until the process exits.
//
// The kernels are the ones the tree solver uses (sort.cu); only where their
// scratch comes from differs.
#include <cstdint>
#include <mutex>

#include <cuda_runtime.h>

#include "common.cuh"
#include "orrery_b200.h"
#include "runtime.hpp"
#include "tree_kernels.hpp"

namespace ob {
namespace {

static_assert(OB_DEVICE_STATUS_TIMEOUT == kStatusTimeout, "the header names the timeout bit");

// Largest particle count the fixed scratch holds.
constexpr uint32_t kNoAllocMaxParticles = 1u << 20;
constexpr uint32_t kNoAllocMaxTiles = (kNoAllocMaxParticles + kSortTile - 1) / kSortTile;

// Layout of the scratch array, in bytes from its start (every piece 256-byte
// aligned so the 16-byte bulk and vector accesses of the kernels stay legal).
constexpr size_t align256(size_t v) { return (v + 255) & ~size_t{255}; }
constexpr size_t kKeysOffset = 0;
constexpr size_t kKeysBytes = align256(sizeof(unsigned long long) * kNoAllocMaxParticles);
constexpr size_t kValsOffset = kKeysOffset + kKeysBytes;
constexpr size_t kValsBytes = align256(sizeof(uint32_t) * kNoAllocMaxParticles);
constexpr size_t kHistOffset = kValsOffset + kValsBytes;
constexpr size_t kHistBytes = align256(sizeof(uint32_t) * kRadixPasses * kRadix);
constexpr size_t kLookbackOffset = kHistOffset + kHistBytes;
constexpr size_t kLookbackBytes =
    align256(sizeof(uint32_t) * kRadixPasses * static_cast<size_t>(kNoAllocMaxTiles) * kRadix);
constexpr size_t kTicketOffset = kLookbackOffset + kLookbackBytes;
constexpr size_t kTicketBytes = align256(sizeof(uint32_t) * kRadixPasses);
constexpr size_t kStatusOffset = kTicketOffset + kTicketBytes;
constexpr size_t kStatusBytes = align256(sizeof(unsigned));
constexpr size_t kMetaOffset = kStatusOffset + kStatusBytes;
constexpr size_t kMetaBytes = align256(sizeof(TreeMeta));
constexpr size_t kCubeOffset = kMetaOffset + kMetaBytes;
constexpr size_t kCubeBytes = align256(sizeof(double) * 6 * kCubeBlocks);
constexpr size_t kScratchBytes = kCubeOffset + kCubeBytes;

// The fixed scratch (about 17 MB). Host code must not use this name as a
// device address: its host-side value is a stand-in, and the device address
// comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_order_scratch[kScratchBytes];

// Device address of g_order_scratch per device, looked up on the first call
// made with that device current.
constexpr int kMaxDevices = 64;
unsigned char *g_scratch_address[kMaxDevices] = {};
std::mutex g_scratch_mutex;

unsigned char *scratch_for_current_device() {
    int device = 0;
    check(cudaGetDevice(&device), "cudaGetDevice");
    if (device < 0 || device >= kMaxDevices) {
        throw Error(OB_ERROR_UNSUPPORTED, "device index beyond the scratch table");
    }
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (g_scratch_address[device] == nullptr) {
        void *address = nullptr;
        check(cudaGetSymbolAddress(&address, g_order_scratch),
              "looking up the fixed ordering scratch");
        g_scratch_address[device] = static_cast<unsigned char *>(address);
    }
    return g_scratch_address[device];
}

} // namespace
} // namespace ob

extern "C" int ob_morton_order_noalloc(uint64_t n, const double *x, const double *y,
                                       const double *z, uint64_t *codes, uint32_t *indices,
                                       uint32_t *status_out, void *stream) {
    using namespace ob;
    try {
        if (n > kNoAllocMaxParticles) {
            return set_error(OB_ERROR_CAPACITY,
                             "ob_morton_order_noalloc orders at most 1048576 particles (its "
                             "fixed scratch holds no more)");
        }
        if (n > 0 && (x == nullptr || y == nullptr || z == nullptr || codes == nullptr ||
                      indices == nullptr)) {
            return set_error(OB_ERROR_INVALID_ARGUMENT, "NULL array");
        }
        const auto count = static_cast<uint32_t>(n);
        const auto s = static_cast<cudaStream_t>(stream);
        unsigned char *base = scratch_for_current_device();
        if (count == 0) {
            if (status_out != nullptr) {
                check(cudaMemsetAsync(status_out, 0, sizeof(uint32_t), s), "clearing status");
            }
            return OB_OK;
        }
        auto *alt_keys = reinterpret_cast<unsigned long long *>(base + kKeysOffset);
        auto *alt_vals = reinterpret_cast<uint32_t *>(base + kValsOffset);
        auto *hist = reinterpret_cast<uint32_t *>(base + kHistOffset);
        auto *lookback = reinterpret_cast<uint32_t *>(base + kLookbackOffset);
        auto *tickets = reinterpret_cast<uint32_t *>(base + kTicketOffset);
        auto *status = reinterpret_cast<unsigned *>(base + kStatusOffset);
        auto *meta = reinterpret_cast<TreeMeta *>(base + kMetaOffset);
        auto *cube = reinterpret_cast<double *>(base + kCubeOffset);
        auto *keys = reinterpret_cast<unsigned long long *>(codes);
        const uint32_t tiles = sort_tiles(count);
        // The array keeps the previous call's contents: clear everything the
        // kernels expect to start at zero.
        check(cudaMemsetAsync(hist, 0, sizeof(uint32_t) * kRadixPasses * kRadix, s), "clearing");
        check(cudaMemsetAsync(lookback, 0,
                              sizeof(uint32_t) * kRadixPasses * static_cast<size_t>(tiles) *
                                  kRadix,
                              s),
              "clearing");
        check(cudaMemsetAsync(tickets, 0, sizeof(uint32_t) * kRadixPasses, s), "clearing");
        check(cudaMemsetAsync(status, 0, sizeof(unsigned), s), "clearing");
        check(cudaMemsetAsync(meta, 0, sizeof(TreeMeta), s), "clearing");
        check(launch_bounding_cube(x, y, z, count, cube, meta, s), "cube");
        check(launch_encode(x, y, z, count, meta, keys, indices, hist, s), "Morton codes");
        check(launch_scan_histograms(hist, s), "digit offsets");
        // Eight passes alternate caller buffer -> scratch -> caller, ending in
        // the caller's arrays.
        for (int pass = 0; pass < kRadixPasses; ++pass) {
            const bool from_caller = (pass & 1) == 0;
            check(launch_onesweep(from_caller ? keys : alt_keys, from_caller ? indices : alt_vals,
                                  from_caller ? alt_keys : keys, from_caller ? alt_vals : indices,
                                  count, pass, hist,
                                  lookback + static_cast<size_t>(pass) * tiles * kRadix,
                                  tickets + pass, status, s),
                  "radix sort pass");
        }
        // A pass whose bounded look-back wait ran out set a bit in the status
        // word and left its tile unscattered; hand the word to the caller, on
        // the stream, so the failure is visible without a host wait here.
        if (status_out != nullptr) {
            check(cudaMemcpyAsync(status_out, status, sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                                  s),
                  "reporting the status word");
        }
        return OB_OK;
    } catch (const Error &e) {
        return set_error(e.code(), e.what());
    }
}
