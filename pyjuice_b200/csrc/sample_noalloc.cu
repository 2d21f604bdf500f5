// Whole-circuit ancestral sampling in one kernel, with no device allocation by anyone.
//
// For callers that may not allocate device memory when they sample: a server that works
// from a fixed, pre-reserved memory pool, a plugin running inside another framework's
// allocator, or a loop that must not call cudaMalloc (which can synchronise the device).
// The per-layer sampling entry points (sample_kernels.cu) need caller-provided working
// lists; this variant keeps those lists in a fixed file-scope device array instead, so
// the caller passes only inputs (the circuit's tables and parameters) and outputs (the
// samples and an error word).
//
// One thread walks the whole circuit for one sample, with the same draw rules and the
// same uniforms (SplitMix64 of (seed, node id, sample)) as the per-layer entry points, so
// the samples are identical bit for bit. Two calls that overlap in time on one device
// share the array and overwrite each other's lists.
#include <atomic>

#include "common.cuh"

namespace {

// Working lists of all samples of one call: per sample cap_n node slots, then cap_e
// element slots. 2^21 int32 = 8 MiB per device. Each sample's lists are initialised by
// the kernel itself (root node, empty element list), so nothing has to be cleared
// between calls.
constexpr int64_t kScratchInts = PCB_SAMPLE_NOALLOC_MAX_INTS;
static __device__ __align__(256) int32_t g_sample_scratch[kScratchInts];

__device__ __forceinline__ float uniform(uint64_t seed, uint32_t node, uint32_t sample) {
    uint64_t z = seed + (((uint64_t)node << 32) | (uint64_t)sample) * 0x9E3779B97F4A7C15ull + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z = z ^ (z >> 31);
    return (float)(z >> 40) * (1.0f / 16777216.0f);
}

__global__ void sample_circuit_kernel(int32_t* __restrict__ scratch, const PcbSampleStep* __restrict__ steps,
                                      int num_steps, int root_id, int S, int cap_n, int cap_e,
                                      int64_t* __restrict__ samples, int64_t sld, uint64_t seed,
                                      int32_t* __restrict__ err) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    int32_t* nl = scratch + (int64_t)s * (cap_n + cap_e);
    int32_t* el = nl + cap_n;
    int n = 1, ne = 0;
    nl[0] = root_id;
    for (int si = 0; si < num_steps; ++si) {
        const PcbSampleStep st = steps[si];
        // The table lives in device memory, so the host cannot check it: a step of unknown
        // kind, or a sum step without a positive block size, stops this sample with code 3.
        if ((st.kind != 0 && st.kind != 1 && st.kind != 2) || (st.kind == 0 && st.bs <= 0)) {
            atomicExch(err, 3);
            return;
        }
        if (st.kind == 0) {  // sum layer: each active node of the layer picks one child element
            int keep = 0;
            for (int j = 0; j < n; ++j) {
                const int id = nl[j];
                if (id < st.lo || id >= st.hi) { nl[keep++] = id; continue; }
                const int g = st.node2blk[(id - st.lo) / st.bs];
                const int i = id - st.blk_first[g];
                const int off = st.blk_off[g];
                const int cnt = st.blk_cnt[g];
                const float u = uniform(seed, (uint32_t)id, (uint32_t)s);
                float cum = 0.f;
                int pick = -1, last_nz = 0;
                for (int k = 0; k < cnt; ++k) {
                    const float w = st.params[(int64_t)st.weight_base[off + k] + i];
                    cum += w;
                    if (w > 0.f) last_nz = k;
                    if (u < cum) { pick = k; break; }
                }
                if (pick < 0) pick = last_nz;
                if (ne < cap_e) el[ne++] = st.children[off + pick];
                else atomicExch(err, 1);
            }
            n = keep;
        } else if (st.kind == 1) {  // product layer: each active element activates its children
            int keep = 0;
            for (int j = 0; j < ne; ++j) {
                const int id = el[j];
                if (id < st.lo || id >= st.hi) { el[keep++] = id; continue; }
                const int g = st.node2blk[id - st.lo];
                if (g < 0) { atomicExch(err, 2); continue; }
                const int i = id - st.blk_first[g];
                const int off = st.blk_off[g];
                const int cnt = st.blk_cnt[g];
                for (int c = 0; c < cnt; ++c) {
                    if (n < cap_n) nl[n++] = st.children[off + c] + i;
                    else atomicExch(err, 1);
                }
            }
            ne = keep;
        } else {  // kind 2, input layer: each active input node draws its category
            for (int j = 0; j < n; ++j) {
                const int id = nl[j];
                if (id < st.lo || id >= st.hi) continue;
                const int li = id - st.lo;
                const int K = st.ncats[li];
                const int64_t sp = st.s_pids[li];
                const float u = uniform(seed, (uint32_t)id, (uint32_t)s);
                float cum = 0.f;
                int pick = -1;
                for (int k = 0; k < K; ++k) {
                    cum += st.params[sp + k];
                    if (cum >= u) { pick = k; break; }
                }
                if (pick < 0) pick = 0;
                samples[(int64_t)s * sld + st.vids[li]] = pick;
            }
        }
    }
}

// Device address of g_sample_scratch, looked up once per device (the host-side name of a
// __device__ variable is only a handle; the runtime reports the address per device).
constexpr int kMaxDevices = 64;
std::atomic<int32_t*> g_scratch_addr[kMaxDevices];

}  // namespace

extern "C" int pcb_sample_circuit_noalloc(const PcbSampleStep* steps, int32_t num_steps, int32_t root_id, int32_t S,
                                          int32_t cap_n, int32_t cap_e, int64_t* samples, int64_t sld, uint64_t seed,
                                          int32_t* err, void* stream) {
    if (!steps || !samples || !err || num_steps < 0 || S < 0 || cap_n <= 0 || cap_e <= 0 || sld <= 0 || root_id < 0)
        return pcb::set_error(PCB_E_ARG, "pcb_sample_circuit_noalloc: bad arguments");
    const int64_t need = (int64_t)S * ((int64_t)cap_n + cap_e);
    if (need > kScratchInts)
        return pcb::set_error(PCB_E_ARG,
                              "pcb_sample_circuit_noalloc: %d samples x (%d + %d) list slots = %lld int32 exceed "
                              "the fixed working area of %lld int32; sample in smaller batches",
                              S, cap_n, cap_e, (long long)need, (long long)kScratchInts);
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return pcb::set_error(PCB_E_CUDA, "pcb_sample_circuit_noalloc: cudaGetDevice failed: %s",
                              cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices)
        return pcb::set_error(PCB_E_CUDA, "pcb_sample_circuit_noalloc: device %d out of range", dev);
    int32_t* scratch = g_scratch_addr[dev].load(std::memory_order_acquire);
    if (scratch == nullptr) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_sample_scratch);
        if (e != cudaSuccess || p == nullptr)
            return pcb::set_error(PCB_E_CUDA, "pcb_sample_circuit_noalloc: cudaGetSymbolAddress failed: %s",
                                  cudaGetErrorString(e));
        scratch = static_cast<int32_t*>(p);
        g_scratch_addr[dev].store(scratch, std::memory_order_release);
    }
    cudaStream_t st = pcb::as_stream(stream);
    e = cudaMemsetAsync(err, 0, sizeof(int32_t), st);
    if (e != cudaSuccess)
        return pcb::set_error(PCB_E_CUDA, "pcb_sample_circuit_noalloc: clearing *err failed: %s",
                              cudaGetErrorString(e));
    if (S == 0) return PCB_OK;
    sample_circuit_kernel<<<(unsigned)pcb::cdiv(S, 128), 128, 0, st>>>(scratch, steps, num_steps, root_id, S, cap_n,
                                                                       cap_e, samples, sld, seed, err);
    return pcb::check_launch("pcb_sample_circuit_noalloc");
}
