// abf_collect_ids_noalloc: bitmap -> ascending ids without any allocation.
//
// Some callers cannot allocate device memory at the point where they need
// ids: an engine that owns every byte of device memory and forbids plugins
// to allocate, a serving thread for which cudaMalloc's possible device-wide
// synchronisation would stall the other streams, or code that must not run
// into out-of-memory in the middle of a request. This entry point uses no
// cudaMalloc/cudaFree (and no allocating library call): the compaction's
// scratch -- one look-back status word per 1024-word chunk, the item ticket
// and an error word -- lives in one file-scope device array, sized for
// bitmaps of at most ABF_NOALLOC_MAX_BITS bits (about 256 KB, held on every
// device that loads the library until the process exits).
//
// Host code may not pass the array's name to a kernel (on the host it is
// only a stand-in symbol): the first call on each device looks up its device
// address with cudaGetSymbolAddress while that device is current and keeps
// it. That first call should come before any stream capture. All calls on a
// device share the array and it keeps the last call's contents; the parts
// that must start at zero (status words, ticket, error word) are cleared on
// the stream by every call, and calls whose work overlaps on the GPU (other
// streams, no ordering) race on it. abf_collect_ids_noalloc_check reads the
// error word that the last call on the device left (a look-back wait that
// gave up).
#include "abf_kernels.cuh"

#include <mutex>
#include <vector>

namespace {

constexpr uint64_t kMaxBits = ABF_NOALLOC_MAX_BITS;
constexpr uint64_t kMaxChunks = (kMaxBits / 32 + abf::kCompactChunkWords - 1) / abf::kCompactChunkWords;
// layout in 8-byte words: status[kMaxChunks] (one look-back word per chunk),
// the item ticket, the error word (low 4 bytes)
constexpr uint64_t kStatusAt = 0;
constexpr uint64_t kTicketAt = kStatusAt + kMaxChunks;
constexpr uint64_t kErrAt = kTicketAt + 1;
constexpr uint64_t kScratchWords = kErrAt + 1;

static __device__ __align__(256) unsigned long long g_noalloc_scratch[kScratchWords];

struct DeviceSlot {
    unsigned long long* base = nullptr;  // device address of g_noalloc_scratch
    int sm_count = 0;
};
std::mutex g_mu;
std::vector<DeviceSlot> g_slots;

abf_status slot_for(int dev, DeviceSlot* out) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_slots.empty()) {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) return abf::fail(ABF_ERR_CUDA, "no CUDA device");
        g_slots.resize(size_t(n));
    }
    if (dev < 0 || size_t(dev) >= g_slots.size()) return abf::fail(ABF_ERR_CUDA, "bad current device");
    DeviceSlot& s = g_slots[size_t(dev)];
    if (!s.base) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            return abf::fail(ABF_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        int sms = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return abf::fail(ABF_ERR_CUDA, std::string("cudaDeviceGetAttribute: ") + cudaGetErrorString(e));
        s.base = static_cast<unsigned long long*>(p);
        s.sm_count = sms > 0 ? sms : 148;
    }
    *out = s;
    return ABF_OK;
}

}  // namespace

extern "C" abf_status abf_collect_ids_noalloc(const uint32_t* d_bitmap, uint64_t n_bits, uint32_t* d_ids,
                                              uint64_t ids_capacity, uint64_t* d_count, void* stream) {
    try {
        if (!d_bitmap || !d_count || (ids_capacity && !d_ids))
            return abf::fail(ABF_ERR_INVALID, "abf_collect_ids_noalloc: null pointer");
        if (n_bits == 0) return abf::fail(ABF_ERR_INVALID, "abf_collect_ids_noalloc: n_bits is 0");
        if (n_bits > kMaxBits)
            return abf::fail(ABF_ERR_CAPACITY, "abf_collect_ids_noalloc: n_bits above ABF_NOALLOC_MAX_BITS (" +
                                                   std::to_string(kMaxBits) + "); use abf_collect_ids");
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return abf::fail(ABF_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
        DeviceSlot slot;
        abf_status st = slot_for(dev, &slot);
        if (st != ABF_OK) return st;
        unsigned long long* b = slot.base;
        abf::CompactArgs ca{};
        ca.bm = d_bitmap;
        ca.stride = (n_bits + 31) / 32;
        ca.n_q = 1;
        ca.n_bits = n_bits;
        ca.n_chunks = abf::compact_chunks(n_bits);
        ca.status = reinterpret_cast<uint64_t*>(b + kStatusAt);
        ca.ticket = b + kTicketAt;
        ca.err = reinterpret_cast<uint32_t*>(b + kErrAt);
        ca.ids = d_ids;
        ca.capacity = ids_capacity;
        ca.id_offsets = nullptr;
        ca.id_counts = d_count;
        ca.spin_limit = abf::kDefaultSpinLimit;
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        // the error word starts clear for every call; launch_compact clears
        // the status words, the ticket and *d_count on the stream
        if ((e = cudaMemsetAsync(ca.err, 0, sizeof(uint32_t), s)) != cudaSuccess ||
            (e = abf::launch_compact(ca, slot.sm_count, 6u, s)) != cudaSuccess)
            return abf::fail(ABF_ERR_CUDA, std::string("abf_collect_ids_noalloc launch: ") + cudaGetErrorString(e));
        return ABF_OK;
    } catch (...) {
        return abf::fail(ABF_ERR_INTERNAL, "abf_collect_ids_noalloc: unexpected exception");
    }
}

extern "C" abf_status abf_collect_ids_noalloc_check(void* stream) {
    try {
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return abf::fail(ABF_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
        DeviceSlot slot;
        abf_status st = slot_for(dev, &slot);
        if (st != ABF_OK) return st;
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        uint32_t err = 0;
        if ((e = cudaMemcpyAsync(&err, slot.base + kErrAt, sizeof(err), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (e = cudaStreamSynchronize(s)) != cudaSuccess)
            return abf::fail(ABF_ERR_CUDA, std::string("abf_collect_ids_noalloc_check: ") + cudaGetErrorString(e));
        if (err) return abf::fail(ABF_ERR_TIMEOUT, "abf_collect_ids_noalloc: a look-back wait gave up (code " +
                                                       std::to_string(err) + "); its ids are not valid");
        return ABF_OK;
    } catch (...) {
        return abf::fail(ABF_ERR_INTERNAL, "abf_collect_ids_noalloc_check: unexpected exception");
    }
}
