// fhtgs_sort_instances_noalloc: the renderer's stable instance sort for callers that must not
// allocate device memory.
//
// Who needs it: code that runs where a device allocation is not acceptable — a VR compositor
// or display thread with a hard per-frame deadline (cudaMalloc/cudaFree can synchronise the
// device and stall for milliseconds), or a plugin inside a host application that owns the whole
// device-memory budget and does not let plugins allocate.  Such callers pass their own input
// and output buffers; the sort's working memory (one ping-pong buffer, the per-tile digit
// histograms and the pair count) lives in a fixed, file-scope device array that every GPU which
// loads libfhtgs.so holds until the process exits.
//
// Limits and rules:
//   * at most kNoAllocMaxPairs (1,048,576) pairs per call; larger requests are rejected;
//   * the order is decided by the key bits below end_bit alone, as cub::DeviceRadixSort's
//     end_bit: the last 8-bit pass masks the higher bits out of its digit, and the keys come
//     out with all their bits;
//   * the output buffers may be the input buffers themselves (an in-place sort); any other
//     overlap between the four buffers is rejected;
//   * the scratch array is shared by every call on a device and keeps the last call's
//     contents.  Nothing in it has to start at zero: each call writes the pair count and every
//     histogram entry it reads.  Calls that overlap on the GPU (two streams, or two host threads)
//     race on it: serialise them;
//   * the first call on each device looks up the array's device address (cudaGetSymbolAddress
//     with that device current) and keeps it for the life of the process; make that first call
//     before any stream capture.  A cudaDeviceReset unloads the library's device code, and the
//     array may come back at another address, so do not reset a device while this library is in
//     use on it;
//   * a CUDA error left pending by an earlier call of the caller is not consumed: the sort then
//     refuses to run and reports that error, so it is never blamed on the sort.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

#include "../../include/fhtgs.h"
#include "fhtgs_types.cuh"

namespace fhtgs {
void set_last_error(const std::string& msg);  // fhtgs_host.cu
}

namespace {

constexpr int64_t kNoAllocMaxPairs = int64_t(1) << 20;
constexpr int kMaxSortTiles = static_cast<int>((kNoAllocMaxPairs + fhtgs::kSortTile - 1) / fhtgs::kSortTile);
constexpr size_t align256(size_t x) { return (x + 255) / 256 * 256; }
// Layout of the scratch array: status | digit totals | histograms | keys | values.
constexpr size_t kOffStatus = 0;
constexpr size_t kOffDigitTot = align256(kOffStatus + sizeof(fhtgs::FrameStatus));
constexpr size_t kOffHist = align256(kOffDigitTot + 4 * fhtgs::kSortBins);
constexpr size_t kOffKeys = align256(kOffHist + 4ull * fhtgs::kSortBins * kMaxSortTiles);
constexpr size_t kOffVals = align256(kOffKeys + 4ull * kNoAllocMaxPairs);
constexpr size_t kScratchBytes = align256(kOffVals + 4ull * kNoAllocMaxPairs);  // about 8.3 MB

static __device__ __align__(256) unsigned char g_sort_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void* g_scratch_ptr[kMaxDevices] = {};

// The pair count the sort kernels read from the frame status.
__global__ void set_pair_count(fhtgs::FrameStatus* status, unsigned long long n) {
    status->n_instances = n;
    status->overflow = 0;
}

fhtgs_status noalloc_fail(fhtgs_status s, const std::string& msg) {
    fhtgs::set_last_error(msg);  // reported by fhtgs_last_error()
    return s;
}

// Byte ranges [a, a + na) and [b, b + nb) share at least one byte.
bool overlaps(const void* a, size_t na, const void* b, size_t nb) {
    const uintptr_t x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
    return x < y + nb && y < x + na;
}

// Error of the launch just made (launch errors are not sticky; cudaGetLastError clears them).
fhtgs_status launch_check(const char* what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return noalloc_fail(FHTGS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return FHTGS_OK;
}

// Device address of g_sort_scratch on the current device; looked up once per device.
fhtgs_status scratch_for_current_device(char** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return noalloc_fail(FHTGS_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(FHTGS_ERR_INVALID_ARGUMENT, "device index out of range");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_sort_scratch);
        if (e != cudaSuccess || !p)
            return noalloc_fail(FHTGS_ERR_CUDA, std::string("cudaGetSymbolAddress(g_sort_scratch): ") + cudaGetErrorString(e));
        g_scratch_ptr[dev] = p;
    }
    *out = static_cast<char*>(g_scratch_ptr[dev]);
    return FHTGS_OK;
}

}  // namespace

extern "C" fhtgs_status fhtgs_sort_instances_noalloc(const void* keys_in, const uint32_t* values_in, void* keys_out,
                                                     uint32_t* values_out, int64_t n, int32_t key_bytes,
                                                     int32_t end_bit, void* stream) {
    if (n < 0) return noalloc_fail(FHTGS_ERR_INVALID_ARGUMENT, "n must be >= 0");
    if (n > kNoAllocMaxPairs)
        return noalloc_fail(FHTGS_ERR_INVALID_ARGUMENT,
                            "n = " + std::to_string(n) + " exceeds the no-allocation sort's maximum of " +
                                std::to_string(kNoAllocMaxPairs) + " pairs");
    if (key_bytes != 2 && key_bytes != 4) return noalloc_fail(FHTGS_ERR_INVALID_ARGUMENT, "key_bytes must be 2 or 4");
    if (end_bit < 1 || end_bit > 8 * key_bytes)
        return noalloc_fail(FHTGS_ERR_INVALID_ARGUMENT, "end_bit must be in [1, 8 * key_bytes]");
    if (n == 0) return FHTGS_OK;
    if (!keys_in || !values_in || !keys_out || !values_out)
        return noalloc_fail(FHTGS_ERR_INVALID_ARGUMENT, "null buffer");
    const size_t kb = static_cast<size_t>(n) * key_bytes, vb = static_cast<size_t>(n) * 4;
    const bool keys_in_place = keys_out == keys_in, values_in_place = values_out == values_in;
    if ((!keys_in_place && overlaps(keys_out, kb, keys_in, kb)) || overlaps(keys_out, kb, values_in, vb) ||
        (!values_in_place && overlaps(values_out, vb, values_in, vb)) || overlaps(values_out, vb, keys_in, kb) ||
        overlaps(keys_out, kb, values_out, vb))
        return noalloc_fail(FHTGS_ERR_INVALID_ARGUMENT,
                            "output buffers overlap the inputs or each other (only keys_out == keys_in and "
                            "values_out == values_in, an in-place sort, are allowed)");
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess)
        return noalloc_fail(FHTGS_ERR_CUDA, std::string("an earlier CUDA call left an error pending (not cleared): ") +
                                                cudaGetErrorString(e));
    char* scratch = nullptr;
    fhtgs_status st = scratch_for_current_device(&scratch);
    if (st != FHTGS_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    fhtgs::FrameParams fp{};
    fp.n_views = 1;
    fp.key_u32 = key_bytes == 4 ? 1 : 0;
    fp.end_bit = end_bit;
    fp.sort_key_bits = end_bit;
    fp.cap = n;
    fhtgs::FrameBuffers fb{};
    fb.status = reinterpret_cast<fhtgs::FrameStatus*>(scratch + kOffStatus);
    fb.sort_digit_tot = reinterpret_cast<uint32_t*>(scratch + kOffDigitTot);
    fb.sort_hist = reinterpret_cast<uint32_t*>(scratch + kOffHist);
    fb.sort_tiles = static_cast<int>((n + fhtgs::kSortTile - 1) / fhtgs::kSortTile);
    fb.sort_items = fhtgs::kSortItems;
    // Ping-pong between the caller's output and the scratch buffer; the input stays untouched.
    fb.keys[0] = keys_out;
    fb.vals[0] = values_out;
    fb.keys[1] = scratch + kOffKeys;
    fb.vals[1] = reinterpret_cast<uint32_t*>(scratch + kOffVals);

    if (!keys_in_place) e = cudaMemcpyAsync(keys_out, keys_in, kb, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess && !values_in_place) e = cudaMemcpyAsync(values_out, values_in, vb, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return noalloc_fail(FHTGS_ERR_CUDA, std::string("cudaMemcpyAsync: ") + cudaGetErrorString(e));
    set_pair_count<<<1, 1, 0, s>>>(fb.status, static_cast<unsigned long long>(n));
    if ((st = launch_check("pair count launch")) != FHTGS_OK) return st;
    fhtgs::kernels_fast().sort(fp, fb, s);
    if ((st = launch_check("sort launch")) != FHTGS_OK) return st;
    if (fb.final_buf == 1) {
        e = cudaMemcpyAsync(keys_out, fb.keys[1], kb, cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(values_out, fb.vals[1], vb, cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return noalloc_fail(FHTGS_ERR_CUDA, std::string("cudaMemcpyAsync: ") + cudaGetErrorString(e));
    }
    return FHTGS_OK;
}
