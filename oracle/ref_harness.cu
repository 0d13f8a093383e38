// TEST INFRASTRUCTURE ONLY.  A C driver around the reference's own CUDA search and
// permutation filter, compiled together with the reference sources (oracle/Makefile, target
// `ref`) into oracle/_ref/libtdp_ref.so.  It replaces the reference's JNI layer
// (src/native/jni/jni_sorter.cu:25-150) with plain C entry points so that tests and the
// fixture generators can run the reference kernel on the same inputs as this project's
// kernels.  The product library never links or loads it.
//
// What it calls, unchanged:
//   initGpuSortSlots / destroyGpuSortSlots / cancelGpuSort (slot_manager.cu:22-125),
//   getGpuSortSlotDevice / getGpuSortSlotStream (slot_manager.cu:154-175),
//   performGpuSortingSearch (sorting_search.cu:701-856),
//   performGpuPiFilter (pi_filter.cu:157-260).
//
// A watchdog thread calls the reference's own cancelGpuSort when a search runs longer than
// the caller's limit; the search then ends through the reference's cancel path and is
// reported as timed out (the reference's warps poll the cancel flag at every pop and every
// 32 children, sorting_search.cu:221-226, 466, 531).
#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <exception>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "backtracking/pi_filter.cuh"
#include "backtracking/slot_manager.cuh"
#include "backtracking/sorting_search.cuh"
#include "core/cuda_error.cuh"

namespace {

thread_local std::string gError;

enum RefStatus : int {
    kRefNotFound = 0,
    kRefFound = 1,
    kRefTimedOut = 2,
    kRefOverflow = 3,
    kRefError = -1,
};

// One watchdog per search call: it fires cancelGpuSort(slot) once the deadline passes unless
// the call disarms it first.  Disarming and firing share one mutex, so a disarmed watchdog
// never cancels a later search on the same slot.
struct Watchdog {
    std::mutex mu;
    std::condition_variable cv;
    bool armed = true;
    bool fired = false;
    std::thread th;

    Watchdog(int slot, double seconds) {
        th = std::thread([this, slot, seconds] {
            std::unique_lock<std::mutex> lock(mu);
            const auto until = std::chrono::steady_clock::now() +
                               std::chrono::microseconds(static_cast<long long>(seconds * 1e6));
            while (armed) {
                if (cv.wait_until(lock, until) == std::cv_status::timeout) {
                    if (armed) {
                        cancelGpuSort(slot);
                        fired = true;
                    }
                    break;
                }
            }
        });
    }
    bool disarm() {
        {
            std::lock_guard<std::mutex> lock(mu);
            armed = false;
        }
        cv.notify_all();
        th.join();
        return fired;
    }
};

bool is_permutation(const uint8_t *v, int n) {
    uint64_t seen = 0;
    for (int i = 0; i < n; ++i) {
        if (v[i] >= n || ((seen >> v[i]) & 1ull)) return false;
        seen |= 1ull << v[i];
    }
    return true;
}

}  // namespace

extern "C" {

const char *ref_last_error(void) { return gError.c_str(); }

// initGpuSortSlots (slot_manager.cu:62-98): queue budget in bytes, dedup table in entries.
int ref_init(int total_slots, int devices_count, long long queue_bytes_budget, int dedup_table_size) {
    try {
        initGpuSortSlots(total_slots, devices_count, static_cast<size_t>(queue_bytes_budget), dedup_table_size);
        return 0;
    } catch (const std::exception &e) {
        gError = e.what();
        return kRefError;
    }
}

int ref_destroy(void) {
    try {
        destroyGpuSortSlots();
        return 0;
    } catch (const std::exception &e) {
        gError = e.what();
        return kRefError;
    }
}

// The reference's searchForSortingSeq path (jni_sorter.cu:45-104) without the JVM: bytes are
// widened to short, the slot's device and stream are selected, and performGpuSortingSearch
// runs.  Returns RefStatus; on kRefFound out_positions gets 3*depth ints (i,j,k per move) and
// out_depth the depth.  out_ms receives the call's wall time.  Inputs must be permutations
// of 0..n-1 (the reference's cycle walk does not terminate otherwise).
int ref_search(int slot, const uint8_t *pi, const uint8_t *spi, int n, int initial_even_cycles, float min_rate,
               int max_moves, int full_sorting, double timeout_s, int32_t *out_positions, int32_t *out_depth,
               double *out_ms) {
    *out_depth = 0;
    if (n < 1 || n > 63 || !is_permutation(pi, n) || !is_permutation(spi, n)) {
        gError = "ref_search: spi/pi must be permutations of 0..n-1 with 1 <= n <= 63";
        return kRefError;
    }
    std::vector<short> vpi(n), vspi(n);
    for (int i = 0; i < n; ++i) {
        vpi[i] = static_cast<short>(pi[i]);
        vspi[i] = static_cast<short>(spi[i]);
    }
    const auto t0 = std::chrono::steady_clock::now();
    Watchdog *dog = nullptr;
    int rc = kRefError;
    try {
        const int device = getGpuSortSlotDevice(slot);
        if (device < 0) throw std::invalid_argument("invalid slot");
        CHECK_CUDA(cudaSetDevice(device));
        cudaStream_t stream = getGpuSortSlotStream(slot);
        dog = new Watchdog(slot, timeout_s);
        const auto moves = performGpuSortingSearch(std::move(vpi), std::move(vspi), initial_even_cycles,
                                                   static_cast<double>(min_rate), max_moves, full_sorting != 0,
                                                   stream, slot);
        const bool fired = dog->disarm();
        delete dog;
        dog = nullptr;
        if (!moves.empty()) {
            for (size_t d = 0; d < moves.size(); ++d) {
                out_positions[3 * d] = moves[d].firstIndex;
                out_positions[3 * d + 1] = moves[d].secondIndex;
                out_positions[3 * d + 2] = moves[d].thirdIndex;
            }
            *out_depth = static_cast<int32_t>(moves.size());
            rc = kRefFound;
        } else {
            // a not-found answer that raced with the watchdog is still a complete search
            (void)fired;
            rc = kRefNotFound;
        }
    } catch (const GpuSortCancelledException &e) {
        gError = e.what();
        rc = kRefTimedOut;
    } catch (const GpuMemoryExhaustedException &e) {
        gError = e.what();
        rc = kRefOverflow;
    } catch (const std::exception &e) {
        gError = e.what();
        rc = kRefError;
    }
    if (dog) {
        dog->disarm();
        delete dog;
    }
    *out_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return rc;
}

// performGpuPiFilter (pi_filter.cu:157-260) on the current device.  Copies up to max_rows
// rows of n bytes (in the reference's arbitrary order) and returns the number of rows the
// reference returned (it keeps at most 1,048,576), or -1.  Symbols of cycle and
// oriented_triple must be < n (the reference indexes per-symbol arrays with them).
long long ref_pi_filter(const uint8_t *cycle, int cycle_len, const uint8_t *oriented_triple, int triple_len, int n,
                        int skip_2move_check, uint8_t *out, long long max_rows) {
    if (n < 1 || n > 63 || cycle_len < 1 || triple_len < 1) {
        gError = "ref_pi_filter: bad sizes";
        return -1;
    }
    for (int i = 0; i < cycle_len; ++i)
        if (cycle[i] >= n) {
            gError = "ref_pi_filter: cycle symbol >= n";
            return -1;
        }
    for (int i = 0; i < triple_len; ++i)
        if (oriented_triple[i] >= n) {
            gError = "ref_pi_filter: triple symbol >= n";
            return -1;
        }
    try {
        const PiFilterResult r =
            performGpuPiFilter(cycle, cycle_len, oriented_triple, triple_len, n, skip_2move_check != 0);
        const long long rows = static_cast<long long>(r.permutations.size());
        for (long long i = 0; i < rows && i < max_rows; ++i) std::memcpy(out + i * n, r.permutations[i].data(), n);
        return rows;
    } catch (const std::exception &e) {
        gError = e.what();
        return -1;
    }
}

}  // extern "C"
