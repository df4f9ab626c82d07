// tdg_group_run_static: the group-by for callers that cannot allocate.
//
// Some callers of this library cannot call cudaMalloc: a host engine living
// inside another runtime whose caching allocator has already reserved the
// device's memory (a cudaMalloc there fails or fragments that pool), or a
// latency-critical query path that cannot afford cudaMalloc's implicit
// device-wide synchronization.  They still own their input and output
// buffers, but they cannot provide the group-by's scratch workspace.  This
// entry point takes its scratch from a fixed array compiled into the library
// instead, so the call allocates nothing.
//
// Limits and sharing, stated once here and in include/tdg.h:
//   - the array holds TDG_STATIC_SCRATCH_BYTES (16 MiB); every GPU that loads
//     the library keeps it for the life of the process;
//   - a group-by whose plan needs more scratch is refused with TD_ERR_RANGE;
//   - all calls share the one array and it keeps the last call's contents;
//     each call re-initializes every part it reads before reading it
//     (accumulator records, hash-table states, error word, sampling tables),
//     but calls that overlap on the GPU -- on two streams or from two host
//     threads -- race on it and must be serialized by the caller;
//   - the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (a host-side symbol is not a device address);
//   - each call waits for its stream before it returns (the group count and
//     the error word are read back), so no call may be made while its stream
//     is being captured into a CUDA graph.
#include "tdg_hash.cuh"
#include <mutex>

namespace tdg {
tdg_status group_run_joined(const tdg_group_desc* d, const tdg_group_plan* p, void* ws,
                            const tdg_expr* pred, const uint64_t* sel, const JoinK* J, int64_t n_left,
                            int64_t n_right, const tdg_group_out* out, cudaStream_t s);
}

using namespace tdg;

static __device__ __align__(256) unsigned char g_static_scratch[TDG_STATIC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
static void* g_scratch_addr[kMaxDevices];
static std::mutex g_scratch_mu;

// Device address of the scratch array on the current device (looked up once
// per device, with that device current).
static tdg_status static_scratch(void** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return E_IO;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return E_IO;
        }
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return E_OK;
}

extern "C" tdg_status tdg_group_run_static(const tdg_group_desc* d, const tdg_expr* pred, const uint64_t* sel_in,
                                           const tdg_group_out* out, void* stream) {
    if (!d || !out) return E_TYPE;
    tdg_group_plan plan;
    tdg_status st = tdg_group_plan_make(d, 0, &plan);
    if (st) return st;
    if (plan.ws_bytes > (size_t)TDG_STATIC_SCRATCH_BYTES) return E_RANGE;
    void* ws = nullptr;
    st = static_scratch(&ws);
    if (st) return st;
    ThreadTimingOff no_events;          // no CUDA events either
    ThreadNoAlloc no_host_buffers;      // nor page-locked status buffers
    return group_run_joined(d, &plan, ws, pred, sel_in, nullptr, 0, 0, out, (cudaStream_t)stream);
}
