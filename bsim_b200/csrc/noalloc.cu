// bsim_run_noalloc: the simulation step for callers that cannot allocate device
// memory themselves or let a library do it.
//
// Who needs it: a host application that owns the GPU's memory through its own
// pool and hands plug-ins ready-made buffers (a cudaMalloc there would bypass
// its accounting, and cudaMalloc/cudaFree can synchronise the whole device and
// stall the host's other streams); a closed-loop, real-time driver that steps a
// network every few milliseconds and cannot afford an allocation's latency or
// implicit synchronisation inside its loop; and a process that has already
// reserved all remaining device memory. They pass every input and output; the
// working memory the step needs (input accumulators, fire ring, fired bitmaps,
// counters) comes from one fixed-size array in this file.
//
// The array is a file-scope __device__ variable, so every GPU that loads this
// library holds it (about 3.4 MB) until the process exits. All calls on a device
// share it: each call clears what must start at zero and then overwrites the
// rest, so calls whose work overlaps on the GPU (different streams, or threads
// without ordering) race on it and must not be issued that way.
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <mutex>
#include <string>

#include "engine.h"

namespace bsim {
cudaError_t step_occupancy(int block, int accumulate, int *blocks_per_sm);
cudaError_t launch_step_exact(const StepArgs &a, int grid, int block, cudaStream_t stream);
int record_error(int code, const std::string &msg);
}  // namespace bsim

using namespace bsim;

namespace {

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

constexpr int64_t kMaxN = BSIM_NOALLOC_MAX_NEURONS;
constexpr int32_t kMaxD = BSIM_NOALLOC_MAX_DELAY;
constexpr int64_t kSlots = kMaxD + 2;
constexpr int64_t kWords = (kMaxN + 31) / 32;
// layout of the scratch array
constexpr size_t kAccOff = 0;                                                     // longlong2 [2][kMaxN]
constexpr size_t kRingOff = kAccOff + align256(2 * kMaxN * sizeof(longlong2));     // int32 [kSlots][kMaxN]
constexpr size_t kBitmapOff = kRingOff + align256(kSlots * kMaxN * sizeof(int32_t));  // uint32 [kSlots][kWords]
constexpr size_t kCntOff = kBitmapOff + align256(kSlots * kWords * sizeof(uint32_t));  // int32 [kSlots]
constexpr size_t kCtrOff = kCntOff + align256(kSlots * sizeof(int32_t));            // cycle, events, ticket, error
constexpr size_t kScratchBytes = kCtrOff + 256;

static_assert(sizeof(bsim_class_params) == sizeof(ClassParams), "class table layout");
static_assert(offsetof(bsim_class_params, refrac_time) == offsetof(ClassParams, refrac_time), "class table layout");
static_assert(offsetof(bsim_class_params, scale_up) == offsetof(ClassParams, scale_up), "class table layout");
static_assert(offsetof(bsim_class_params, inst) == offsetof(ClassParams, inst), "class table layout");

}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
int g_grid[kMaxDevices];  // launch shape per device (0: not sized yet)

// Errors are reported through bsim_last_error(), like every other entry point.
int noalloc_fail(int code, const char *msg, cudaError_t st = cudaSuccess)
{
    std::string m = msg;
    if (st != cudaSuccess) {
        m += ": ";
        m += cudaGetErrorString(st);
    }
    return record_error(code, m);
}

// The array's device address, looked up on every call with the caller's device
// current (the lookup allocates nothing and stays right across a device reset),
// and the launch shape, sized once per device.
int setup_device(int dev, unsigned char **scratch, int *grid)
{
    void *p = nullptr;
    cudaError_t st = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (st != cudaSuccess) return noalloc_fail(BSIM_ERR_CUDA, "cudaGetSymbolAddress(g_noalloc_scratch)", st);
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_grid[dev]) {
        int sms = 0, bps = 0;
        st = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (st != cudaSuccess) return noalloc_fail(BSIM_ERR_CUDA, "cudaDeviceGetAttribute", st);
        st = step_occupancy(512, BSIM_ACC_EXACT, &bps);
        if (st != cudaSuccess) return noalloc_fail(BSIM_ERR_CUDA, "cudaOccupancyMaxActiveBlocksPerMultiprocessor", st);
        g_grid[dev] = sms * (bps > 0 ? bps : 1);
    }
    *scratch = static_cast<unsigned char *>(p);
    *grid = g_grid[dev];
    return BSIM_OK;
}

__device__ __forceinline__ void check_fail(int32_t *err, int code) { atomicCAS(err, 0, code); }

// The check pass over the caller's arrays (within the sizes the caller gives):
// row offsets from 0 to n_syn and ascending, targets inside the network, class
// indices inside the table, every class of the LIF kind. Any failure raises the
// error flag, after which the step launches return at once.
__global__ void noalloc_check_kernel(StepArgs a, int32_t n_classes, int64_t n_syn)
{
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t rows = a.N * a.D;
    if (tid == 0 && (a.row_off[0] != 0 || a.row_off[rows] != n_syn)) check_fail(a.err, BSIM_DEVERR_ROWS_END);
    for (int64_t i = tid; i < rows; i += stride)
        if (a.row_off[i + 1] < a.row_off[i]) check_fail(a.err, BSIM_DEVERR_ROW);
    for (int64_t k = tid; k < n_syn; k += stride)
        if ((int64_t)a.syn[k].x >= a.N) check_fail(a.err, BSIM_DEVERR_TARGET);
    for (int64_t j = tid; j < a.N; j += stride)
        if ((int32_t)a.cls[j] >= n_classes) check_fail(a.err, BSIM_DEVERR_CLASS);
    for (int64_t c = tid; c < n_classes; c += stride)
        if (a.ctab[c].kind != BSIM_NEURON_LIF) check_fail(a.err, BSIM_DEVERR_CLASS);
}

}  // namespace

extern "C" int bsim_run_noalloc(int64_t n, int32_t max_delay, void *state_dev, const float *vtmp_dev,
                                const uint16_t *cls_dev, const bsim_class_params *ctab_dev, int32_t n_classes,
                                const int64_t *row_off_dev, const uint32_t *syn_dev, int64_t n_synapses,
                                int32_t *fire_count_dev, int64_t steps, void *stream)
{
    if (n < 1 || n > kMaxN)
        return noalloc_fail(BSIM_ERR_LIMIT, "bsim_run_noalloc: n_neurons must be 1..BSIM_NOALLOC_MAX_NEURONS (32768)");
    if (max_delay < 1 || max_delay > kMaxD)
        return noalloc_fail(BSIM_ERR_LIMIT, "bsim_run_noalloc: max_delay must be 1..BSIM_NOALLOC_MAX_DELAY (16)");
    if (!state_dev || !vtmp_dev || !cls_dev || !ctab_dev || !row_off_dev || !syn_dev || !fire_count_dev || steps < 0)
        return noalloc_fail(BSIM_ERR_ARG, "bsim_run_noalloc: null pointer or negative step count");
    if (n_classes < 1 || n_classes > BSIM_MAX_CLASSES || n_synapses < 0)
        return noalloc_fail(BSIM_ERR_ARG, "bsim_run_noalloc: n_classes must be 1..65535, n_synapses >= 0");
    if ((reinterpret_cast<uintptr_t>(state_dev) & 15) || (reinterpret_cast<uintptr_t>(syn_dev) & 15))
        return noalloc_fail(BSIM_ERR_ARG, "bsim_run_noalloc: state and synapse arrays must be 16-byte aligned");
    int dev = 0;
    cudaError_t st = cudaGetDevice(&dev);
    if (st != cudaSuccess) return noalloc_fail(BSIM_ERR_CUDA, "cudaGetDevice", st);
    if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(BSIM_ERR_LIMIT, "bsim_run_noalloc: device ordinal >= 64");
    unsigned char *scratch = nullptr;
    int grid = 0;
    int rc = setup_device(dev, &scratch, &grid);
    if (rc != BSIM_OK) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    StepArgs a{};
    a.N = n;
    a.D = max_delay;
    a.R = max_delay + 2;
    a.cap = n;
    a.W = (n + 31) / 32;
    a.state = static_cast<float4 *>(state_dev);
    a.vtmp = vtmp_dev;
    a.cls = cls_dev;
    a.ctab = reinterpret_cast<const ClassParams *>(ctab_dev);
    a.acc = scratch + kAccOff;
    a.ring = reinterpret_cast<int32_t *>(scratch + kRingOff);
    a.bitmap = reinterpret_cast<uint32_t *>(scratch + kBitmapOff);
    a.ring_cnt = reinterpret_cast<int32_t *>(scratch + kCntOff);
    unsigned long long *ctr = reinterpret_cast<unsigned long long *>(scratch + kCtrOff);
    a.step_ctr = ctr;
    a.events = ctr + 1;
    a.ticket = reinterpret_cast<unsigned int *>(ctr + 2);
    a.err = reinterpret_cast<int32_t *>(ctr + 3);
    a.row_off = row_off_dev;
    a.syn = reinterpret_cast<const uint2 *>(syn_dev);
    a.fire_count = fire_count_dev;
    a.delivery = BSIM_DELIVERY_PUSH;
    a.n_pops = 1;
    a.n_planes = 1;
    a.acc_clear = 1;

    // The previous call's contents are still in the array: clear what must
    // start at zero (input accumulators of both parities, ring counts, bitmaps,
    // cycle/event/ticket/error words). The ring's ids are always written
    // before they are read.
    if ((st = cudaMemsetAsync(a.acc, 0, 2 * (size_t)n * sizeof(longlong2), s)) != cudaSuccess ||
        (st = cudaMemsetAsync(a.ring_cnt, 0, (size_t)a.R * sizeof(int32_t), s)) != cudaSuccess ||
        (st = cudaMemsetAsync(a.bitmap, 0, (size_t)a.R * a.W * sizeof(uint32_t), s)) != cudaSuccess ||
        (st = cudaMemsetAsync(ctr, 0, 4 * sizeof(unsigned long long), s)) != cudaSuccess)
        return noalloc_fail(BSIM_ERR_CUDA, "bsim_run_noalloc: clearing the scratch array", st);
    noalloc_check_kernel<<<grid, 512, 0, s>>>(a, n_classes, n_synapses);
    if ((st = cudaGetLastError()) != cudaSuccess) return noalloc_fail(BSIM_ERR_CUDA, "bsim_run_noalloc: check", st);
    for (int64_t k = 0; k < steps; k++) {
        st = launch_step_exact(a, grid, 512, s);
        if (st != cudaSuccess) return noalloc_fail(BSIM_ERR_CUDA, "bsim_run_noalloc: launch", st);
    }
    return BSIM_OK;
}

extern "C" int bsim_noalloc_status(void *stream, int32_t *device_error)
{
    if (!device_error) return noalloc_fail(BSIM_ERR_ARG, "bsim_noalloc_status: null output");
    void *p = nullptr;
    cudaError_t st = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (st != cudaSuccess) return noalloc_fail(BSIM_ERR_CUDA, "cudaGetSymbolAddress(g_noalloc_scratch)", st);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int32_t err = 0;
    if ((st = cudaMemcpyAsync(&err, static_cast<unsigned char *>(p) + kCtrOff + 3 * sizeof(unsigned long long),
                              sizeof(int32_t), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (st = cudaStreamSynchronize(s)) != cudaSuccess)
        return noalloc_fail(BSIM_ERR_CUDA, "bsim_noalloc_status", st);
    *device_error = err;
    if (err) {
        static const char *names[] = {"", "row offsets not ascending", "synapse target outside the network",
                                      "class index or kind out of range", "row offsets do not span 0..n_synapses",
                                      "a bounded wait inside the step ran out"};
        std::string m = "bsim_run_noalloc: device error flag " + std::to_string(err);
        if (err > 0 && err <= 5) m += std::string(" (") + names[err] + ")";
        return record_error(BSIM_ERR_DEVICE, m);
    }
    return BSIM_OK;
}
