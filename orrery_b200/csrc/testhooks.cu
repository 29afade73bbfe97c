// Test-only entry points that drive the library's failure paths on the device
// without faulting it: a bounded wait made to run out. They allocate their
// own buffers and never touch a solver's or a system's state.
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "common.cuh"
#include "orrery_b200.h"
#include "runtime.hpp"
#include "tree_kernels.hpp"

extern "C" int ob_test_lookback_timeout(uint64_t n, uint32_t poll_limit, int skip_first_tile) {
    using namespace ob;
    try {
        if (n == 0 || n > (1u << 24)) {
            return set_error(OB_ERROR_INVALID_ARGUMENT, "n must be in [1, 2^24]");
        }
        const auto count = static_cast<uint32_t>(n);
        const uint32_t tiles = sort_tiles(count);
        // Keys descending with their index: one digit pass reorders them.
        std::vector<unsigned long long> keys(count);
        std::vector<uint32_t> vals(count);
        for (uint32_t i = 0; i < count; ++i) {
            keys[i] = static_cast<unsigned long long>(count - 1u - i) & 0xffu;
            vals[i] = i;
        }
        std::vector<uint32_t> offsets(kRadixPasses * kRadix, 0u);
        {
            std::vector<uint32_t> hist(kRadix, 0u);
            for (uint32_t i = 0; i < count; ++i) {
                ++hist[keys[i] & 0xffu];
            }
            uint32_t run = 0;
            for (int d = 0; d < kRadix; ++d) {
                offsets[d] = run;
                run += hist[d];
            }
        }
        DeviceArray<unsigned long long> k_in, k_out;
        DeviceArray<uint32_t> v_in, v_out, off, lookback, ticket;
        DeviceArray<unsigned> status;
        k_in.reserve(count);
        k_out.reserve(count);
        v_in.reserve(count);
        v_out.reserve(count);
        off.reserve(offsets.size());
        // One tile more than the input holds: with the first ticket skipped,
        // the last CTA takes ticket `tiles` (no items; it still publishes).
        lookback.reserve(static_cast<size_t>(tiles + 1) * kRadix);
        ticket.reserve(1);
        status.reserve(1);
        check(cudaMemcpy(k_in.data(), keys.data(), k_in.bytes(), cudaMemcpyHostToDevice), "keys");
        check(cudaMemcpy(v_in.data(), vals.data(), v_in.bytes(), cudaMemcpyHostToDevice), "vals");
        check(cudaMemcpy(off.data(), offsets.data(), off.bytes(), cudaMemcpyHostToDevice),
              "offsets");
        check(cudaMemset(k_out.data(), 0, k_out.bytes()), "clearing");
        check(cudaMemset(v_out.data(), 0, v_out.bytes()), "clearing");
        check(cudaMemset(lookback.data(), 0, lookback.bytes()), "clearing");
        check(cudaMemset(status.data(), 0, sizeof(unsigned)), "clearing");
        // With the ticket starting at 1 no CTA takes tile 0, so its look-back
        // words are never published: every tile that reaches them polls until
        // the limit and gives up. Every tile still publishes its own prefix
        // before it returns, so no wait depends on one that never ends.
        const uint32_t first = skip_first_tile != 0 ? 1u : 0u;
        check(cudaMemcpy(ticket.data(), &first, sizeof(first), cudaMemcpyHostToDevice), "ticket");
        check(launch_onesweep(k_in.data(), v_in.data(), k_out.data(), v_out.data(), count, 0,
                              off.data(), lookback.data(), ticket.data(), status.data(), nullptr,
                              poll_limit),
              "look-back pass");
        check(cudaDeviceSynchronize(), "look-back pass");
        unsigned word = 0;
        check(cudaMemcpy(&word, status.data(), sizeof(word), cudaMemcpyDeviceToHost), "status");
        if ((word & kStatusTimeout) != 0u) {
            return set_error(OB_ERROR_TIMEOUT,
                             "a onesweep tile's look-back wait ran out of polls (its "
                             "predecessor never published)");
        }
        // A completed pass must have sorted the digit stably.
        std::vector<unsigned long long> got(count);
        std::vector<uint32_t> got_vals(count);
        check(cudaMemcpy(got.data(), k_out.data(), k_out.bytes(), cudaMemcpyDeviceToHost), "keys");
        check(cudaMemcpy(got_vals.data(), v_out.data(), v_out.bytes(), cudaMemcpyDeviceToHost),
              "vals");
        for (uint32_t i = 1; i < count; ++i) {
            const bool ordered = got[i - 1] < got[i] ||
                                 (got[i - 1] == got[i] && got_vals[i - 1] < got_vals[i]);
            if (!ordered) {
                return set_error(OB_ERROR_CUDA, "the look-back pass did not sort its input");
            }
        }
        return OB_OK;
    } catch (const Error &e) {
        return set_error(e.code(), e.what());
    }
}

