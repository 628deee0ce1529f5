// Simulated-annealing run of one problem with no device allocation.
//
// Some callers cannot call cudaMalloc: hosts that hand the GPU to a framework
// with its own fixed memory pool and forbid other allocators, and
// latency-critical services that must not risk a blocking or failing
// allocation mid-request. ie_sa_run_static serves them: the caller
// provides the problem and the output buffers in device memory it already
// owns, and every byte of scratch the run needs (the site-record stream, the
// instance descriptor, the master-stream key and position, the work-queue
// counter, the lane-major spin words and the temperature schedule) lives in
// one file-scope device array, g_static_scratch, of fixed size. The array
// exists on every GPU that loads this library, for as long as the process
// runs.
//
// The run is the f64 mode of the batched kernel (one instance, four threads
// per generator lane); for integral input it gives the same spins and
// energies as the integer mode, bit for bit.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>

#include "../../include/ising_b200.h"
#include "ie_device.cuh"
#include "ie_kernels.cuh"
#include "ie_launch.h"

namespace ie {

// Limits of the static path.
constexpr uint32_t kStaticMaxSites = 16384;
constexpr uint32_t kStaticMaxCouplings = 262144;  // both triangles
constexpr uint64_t kStaticMaxSteps = 65536;
constexpr size_t kStaticScratchBytes = 12u << 20;

// Scratch layout (byte offsets, each 256-aligned).
constexpr size_t kOffDesc = 0;                                    // InstDesc
constexpr size_t kOffKey = 256;                                   // 8 x u32
constexpr size_t kOffMisc = 512;                                  // pos u64, deo i32, queue u32, err i32, quad 4 x u32, quad_h i32
constexpr size_t kOffEi = 1024;                                   // 64 x i32 (unused by the f64 mode)
constexpr size_t kOffTemps = 2048;                                // kStaticMaxSteps x f64
constexpr size_t kOffSpins = kOffTemps + kStaticMaxSteps * 8;     // kStaticMaxSites x u64 (lane-major)
constexpr size_t kOffRecs = kOffSpins + (size_t)kStaticMaxSites * 8;
constexpr size_t kStaticRecWords = (kStaticScratchBytes - kOffRecs) / 4;
static_assert(kOffRecs + (size_t)64 * 1024 * 4 < kStaticScratchBytes, "record area too small");

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

// Checks the caller's CSR on many threads before anything reads it through
// the row offsets: rows[0] == 0, rows[n] <= nnz, monotone row offsets, and
// every stored column below n. A violation sets *err = 4. Every index used
// here is below n + 1 (rows) or nnz (cols), the sizes the caller declared.
__global__ void static_check_kernel(const uint32_t* rows, const uint32_t* cols, uint32_t n, uint32_t nnz,
                                    int32_t* err) {
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 0 && (rows[0] != 0 || rows[n] > nnz)) atomicExch(err, 4);
    for (uint32_t v = t; v < n; v += stride)
        if (rows[v + 1] < rows[v]) atomicExch(err, 4);
    for (uint32_t e = t; e < nnz; e += stride)
        if (cols[e] >= n) atomicExch(err, 4);
}

// Packs the f64 site-record stream (layout in ie_kernels.cuh) of the problem
// into the scratch record area. One thread: chunk packing is sequential (about
// 1M words at the coupling limit). It runs only on a CSR that
// static_check_kernel passed; every write is bounds-checked. On a bad CSR
// (*err = 4) or too little room (*err = 3) the descriptor gets n = 0, so the
// later kernels of the call touch nothing.
__global__ void static_records_kernel(const uint32_t* rows, const uint32_t* cols, const double* vals,
                                      const double* lin, uint32_t n, uint32_t nnz, uint32_t* recs, uint64_t cap,
                                      InstDesc* desc, int32_t* err) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    InstDesc bad{};
    bad.mode = kModeF64;
    bad.nt = 1;
    bad.rec_len = 0;
    if (*err != 0) {
        *desc = bad;
        return;
    }
    uint64_t w = 0;   // words written
    uint32_t c = 0;   // position in the current chunk
    bool ok = true;
    auto put = [&](uint32_t x) {
        if (w >= cap) {
            ok = false;
            return;
        }
        recs[w++] = x;
    };
    for (uint32_t v = 0; v < n && ok; v++) {
        uint32_t e0 = rows[v];
        const uint32_t end = rows[v + 1];
        do {
            const uint32_t deg = min(end - e0, kRecMaxDeg);
            const uint32_t deg4 = (deg + 3u) & ~3u;
            const uint32_t len = 4 + 3 * deg4;
            const uint32_t cont = (e0 + deg < end) ? kRecCont : 0u;
            if (c + len > kChunk) {
                put(kRecPad);
                while ((w % kChunk) != 0 && ok) put(0);
                c = 0;
            }
            const uint64_t lb = __double_as_longlong(lin[v]);
            put(deg | cont);
            put(0);
            put((uint32_t)lb);
            put((uint32_t)(lb >> 32));
            for (uint32_t e = 0; e < deg4; e++) put(e < deg ? cols[e0 + e] : 0u);
            for (uint32_t e = 0; e < deg4; e++) {
                const uint64_t vb = e < deg ? (uint64_t)__double_as_longlong(vals[e0 + e]) : 0ULL;
                put((uint32_t)vb);
                put((uint32_t)(vb >> 32));
            }
            c = (c + len) % kChunk;
            e0 += deg;
        } while (e0 < end && ok);
    }
    if (ok && (c != 0 || w == 0)) {
        if (c != 0) put(kRecPad);
        while (ok && ((w % kChunk) != 0 || w == 0)) put(0);
    }
    if (!ok) {
        *err = 3;
        *desc = bad;
        return;
    }
    InstDesc d{};
    d.n = n;
    d.H = 0;
    d.mode = kModeF64;
    d.nt = 1;
    d.rec = 0;
    d.rec_len = w;
    *desc = d;
}

// Random init (ultimate.rs:248-280 with no clamps): word v is draw v of the
// master stream, stored lane-major.
__global__ void static_init_kernel(const uint32_t* key, uint32_t n, uint64_t* spins, uint64_t* pos) {
    uint32_t k[8];
#pragma unroll
    for (int i = 0; i < 8; i++) k[i] = key[i];
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        spins[v] = transpose8x8(chacha8_draw(k, v));
    if (blockIdx.x == 0 && threadIdx.x == 0) *pos = n;
}

// Final spins in the reference word layout (bit r = replica r).
__global__ void static_export_kernel(const uint64_t* spins, uint32_t n, uint64_t* out) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        out[v] = transpose8x8(spins[v]);
}

}  // namespace ie

namespace {

std::mutex g_static_mu;
// Device address of the scratch array per device ordinal, looked up on the
// first call on that device and valid for the life of its CUDA context.
void* g_static_ptr[64] = {nullptr};

// Restores the caller's current device on every return path.
struct DeviceGuard {
    int prev = -1;
    DeviceGuard() {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

ie_status static_fail(ie_status s, const char* msg) {
    ie::set_last_error(msg);
    return s;
}

// rand_core 0.6.4 seed_from_u64 (PCG32 outputs as the ChaCha8 key words).
void static_key(uint64_t state, uint32_t key[8]) {
    for (int i = 0; i < 8; i++) {
        state = state * 6364136223846793005ULL + 11634580027462260723ULL;
        const uint32_t xs = (uint32_t)(((state >> 18) ^ state) >> 27);
        const uint32_t rot = (uint32_t)(state >> 59);
        key[i] = (xs >> rot) | (xs << ((32 - rot) & 31));
    }
}

}  // namespace

extern "C" ie_status ie_sa_run_static(const ie_problem_device* problem, uint64_t seed, const double* temps,
                                      uint64_t n_steps, uint64_t* words, double* energies, int32_t device,
                                      void* stream) {
    using namespace ie;
    if (!problem || !temps || !words || !energies) return static_fail(IE_ERR_INVALID, "NULL argument");
    if (problem->num_vars == 0 || problem->num_vars > kStaticMaxSites)
        return static_fail(IE_ERR_INVALID, "ie_sa_run_static: num_vars must be in [1, 16384]");
    if (problem->nnz > kStaticMaxCouplings)
        return static_fail(IE_ERR_INVALID, "ie_sa_run_static: at most 262144 stored couplings");
    if (n_steps == 0 || n_steps > kStaticMaxSteps)
        return static_fail(IE_ERR_INVALID, "ie_sa_run_static: n_steps must be in [1, 65536]");
    if (!problem->row_offsets || !problem->linear || (problem->nnz && (!problem->col_indices || !problem->values)))
        return static_fail(IE_ERR_INVALID, "ie_sa_run_static: problem arrays must be device pointers");
    if (device < 0 || device >= 64) return static_fail(IE_ERR_INVALID, "ie_sa_run_static: bad device ordinal");
    for (uint64_t i = 0; i < n_steps; i++)
        if (!(temps[i] > 0.0)) return static_fail(IE_ERR_INVALID, "ie_sa_run_static: temperatures must be positive");
    DeviceGuard guard;
    if (cudaSetDevice(device) != cudaSuccess) return static_fail(IE_ERR_CUDA, "cudaSetDevice failed");
    unsigned char* base = nullptr;
    {
        // Once per device, with that device current: the device address of the
        // scratch array (its host-side name is only a stand-in).
        std::lock_guard<std::mutex> lock(g_static_mu);
        if (!g_static_ptr[device]) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_static_scratch) != cudaSuccess || !p)
                return static_fail(IE_ERR_CUDA, "cudaGetSymbolAddress(g_static_scratch) failed");
            g_static_ptr[device] = p;
        }
        base = static_cast<unsigned char*>(g_static_ptr[device]);
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    InstDesc* d_desc = reinterpret_cast<InstDesc*>(base + kOffDesc);
    uint32_t* d_key = reinterpret_cast<uint32_t*>(base + kOffKey);
    uint64_t* d_pos = reinterpret_cast<uint64_t*>(base + kOffMisc);
    int32_t* d_deo = reinterpret_cast<int32_t*>(base + kOffMisc + 8);
    uint32_t* d_queue = reinterpret_cast<uint32_t*>(base + kOffMisc + 12);
    int32_t* d_err = reinterpret_cast<int32_t*>(base + kOffMisc + 16);
    uint32_t* d_quad = reinterpret_cast<uint32_t*>(base + kOffMisc + 32);
    int32_t* d_quadh = reinterpret_cast<int32_t*>(base + kOffMisc + 48);
    int32_t* d_ei = reinterpret_cast<int32_t*>(base + kOffEi);
    double* d_temps = reinterpret_cast<double*>(base + kOffTemps);
    uint64_t* d_spins = reinterpret_cast<uint64_t*>(base + kOffSpins);
    uint32_t* d_recs = reinterpret_cast<uint32_t*>(base + kOffRecs);

    // The array keeps the previous call's contents: reset what must start at
    // zero (position, phase, queue counter, error word) and the work item.
    uint32_t key[8];
    static_key(seed, key);
    unsigned char misc[64];
    std::memset(misc, 0, sizeof(misc));
    const uint32_t quad[4] = {0u, 0xffffffffu, 0xffffffffu, 0xffffffffu};
    std::memcpy(misc + 32, quad, sizeof(quad));
    if (cudaMemcpyAsync(d_key, key, sizeof(key), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(base + kOffMisc, misc, sizeof(misc), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(d_temps, temps, n_steps * sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess)
        return static_fail(IE_ERR_CUDA, "copy into the static scratch failed");

    const uint32_t n = problem->num_vars;
    static_check_kernel<<<64, 256, 0, st>>>(problem->row_offsets, problem->col_indices, n, problem->nnz, d_err);
    static_records_kernel<<<1, 1, 0, st>>>(problem->row_offsets, problem->col_indices, problem->values,
                                           problem->linear, n, problem->nnz, d_recs, kStaticRecWords, d_desc,
                                           d_err);
    static_init_kernel<<<(n + 255) / 256, 256, 0, st>>>(d_key, n, d_spins, d_pos);
    DevArrays A{};
    A.desc = d_desc;
    A.rows = problem->row_offsets;
    A.cols = problem->col_indices;
    A.vals = problem->values;
    A.lin = problem->linear;
    A.recs = d_recs;
    A.keys = d_key;
    A.spins = d_spins;
    A.Ei = d_ei;
    A.Ef = energies;
    A.pos = d_pos;
    A.deo = d_deo;
    A.err = d_err;
    if (launch_energy(A, 0, 1, st) != cudaSuccess) return static_fail(IE_ERR_CUDA, "energy launch failed");
    RunArgs R{};
    R.temps = d_temps;
    R.temps_per_step = 1;
    R.steps = (uint32_t)n_steps;
    R.step_base = 0;
    R.exchange_interval = 1;
    R.quads = d_quad;
    R.quad_h = d_quadh;
    R.nquads = 1;
    R.queue = d_queue;
    const uint32_t cap = (n + 63u) & ~63u;
    if (batch_occupancy(kModeF64, 4, cap, false) <= 0) return static_fail(IE_ERR_UNSUPPORTED, "kernel does not fit");
    if (launch_batch(A, R, kModeF64, 4, cap, 1, st) != cudaSuccess)
        return static_fail(IE_ERR_CUDA, "sweep launch failed");
    static_export_kernel<<<(n + 255) / 256, 256, 0, st>>>(d_spins, n, words);
    if (cudaGetLastError() != cudaSuccess) return static_fail(IE_ERR_CUDA, "launch failed");
    if (cudaStreamSynchronize(st) != cudaSuccess) return static_fail(IE_ERR_CUDA, "run failed on the device");
    int32_t err = 0;
    if (cudaMemcpy(&err, d_err, sizeof(err), cudaMemcpyDeviceToHost) != cudaSuccess)
        return static_fail(IE_ERR_CUDA, "reading the error word failed");
    if (err == 3) return static_fail(IE_ERR_INVALID, "ie_sa_run_static: site records exceed the static scratch");
    if (err == 4) return static_fail(IE_ERR_INVALID, "ie_sa_run_static: invalid CSR (row offsets or column index)");
    if (err) return static_fail(IE_ERR_DEVICE, "device-side check failed");
    return IE_OK;
}
