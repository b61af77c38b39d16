// sample.cu -- basis-state sampling from |amp|^2 (the serving path's read-out).
//
//   sampleBlockSums   sum of |a|^2 over each run of 2^12 consecutive
//                     amplitudes (one CTA per run, fixed reduction order)
//   sampleScan        inclusive prefix of those sums (one CTA, fixed order)
//   sampleFind        one warp per sample: binary search of the prefix for
//                     the run, then a lane-ordered scan inside the run
// A sample with uniform u is the smallest address whose cumulative
// probability exceeds u x total, in the buffer's address order. The lazy
// collapse of a measurement (mask, value, scale) is applied on the fly.
// dgQuEST has no sampler (its measure is unimplemented); this is the
// multi-shot counterpart of the measurement rule of QuEST_common.c:97-115.
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.h"

namespace dgq {

namespace {

constexpr int kRunBits = 12;
constexpr uint32_t kRun = 1u << kRunBits;

template <class V>
__device__ __forceinline__ double prob(const V *st, uint64_t i, const SampleArgs &a) {
    const V v = st[i];
    const double p = (double) v.x * (double) v.x + (double) v.y * (double) v.y;
    if (a.restrictMask == 0) return p;
    return ((i & a.restrictMask) == a.restrictValue) ? p * a.restrictScale2 : 0.0;
}

template <class V>
__global__ void __launch_bounds__(256) sampleBlockSums(const V *__restrict__ st, const __grid_constant__ SampleArgs a,
                                                       double *__restrict__ sums) {
    __shared__ double red[8];
    const uint64_t base = (uint64_t) blockIdx.x << kRunBits;
    const uint64_t end = a.numAmps < base + kRun ? a.numAmps : base + kRun;
    double s = 0.0;
    for (uint64_t i = base + threadIdx.x; i < end; i += 256) s += prob(st, i, a);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; w++) t += red[w];
        sums[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(1024) sampleScan(double *__restrict__ sums, uint64_t n) {
    __shared__ double part[1024];
    const uint64_t chunk = (n + 1023) / 1024;
    const uint64_t b = threadIdx.x * chunk;
    const uint64_t e = b + chunk < n ? b + chunk : n;
    double s = 0.0;
    for (uint64_t i = b; i < e; i++) s += sums[i];
    part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double acc = 0.0;
        for (int t = 0; t < 1024; t++) {
            const double v = part[t];
            part[t] = acc;
            acc += v;
        }
    }
    __syncthreads();
    double acc = part[threadIdx.x];
    for (uint64_t i = b; i < e; i++) {
        acc += sums[i];
        sums[i] = acc;
    }
}

template <class V>
__global__ void __launch_bounds__(256) sampleFind(const V *__restrict__ st, const __grid_constant__ SampleArgs a,
                                                  const double *__restrict__ prefix, uint64_t numRuns,
                                                  const double *__restrict__ uniforms, int count,
                                                  uint64_t *__restrict__ out) {
    const int k = (int) ((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (k >= count) return;
    const double total = prefix[numRuns - 1];
    const double t = uniforms[k] * total;
    // first run whose inclusive prefix exceeds t
    uint64_t lo = 0, hi = numRuns - 1;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (prefix[mid] > t)
            hi = mid;
        else
            lo = mid + 1;
    }
    const uint64_t run = lo;
    const double r = t - (run > 0 ? prefix[run - 1] : 0.0);
    const uint64_t base = run << kRunBits;
    const uint64_t len = a.numAmps - base < kRun ? a.numAmps - base : kRun;
    const uint32_t per = (uint32_t) ((len + 31) / 32);
    const uint64_t lb = base + (uint64_t) lane * per;
    const uint64_t le = lb + per < base + len ? lb + per : base + len;
    double s = 0.0;
    uint64_t lastNz = ~0ULL;
    for (uint64_t i = lb; i < le; i++) {
        const double p = prob(st, i, a);
        s += p;
        if (p > 0.0) lastNz = i;
    }
    // inclusive scan of the lane sums in lane order
    double inc = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double v = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += v;
    }
    const uint32_t hit = __ballot_sync(0xffffffffu, inc > r && s > 0.0);
    uint64_t pick = ~0ULL;
    if (hit) {
        const int L = __ffs(hit) - 1;
        if (lane == L) {
            double acc = inc - s;
            for (uint64_t i = lb; i < le; i++) {
                const double p = prob(st, i, a);
                acc += p;
                if (acc > r && p > 0.0) {
                    pick = i;
                    break;
                }
            }
            if (pick == ~0ULL) pick = lastNz;
        }
        pick = __shfl_sync(0xffffffffu, pick, L);
    } else {
        // t at or beyond the run's total by rounding: its last nonzero amplitude
        const uint32_t nz = __ballot_sync(0xffffffffu, lastNz != ~0ULL);
        if (nz) {
            const int L = 31 - __clz(nz);
            pick = __shfl_sync(0xffffffffu, lastNz, L);
        } else {
            pick = base;
        }
    }
    if (lane == 0) out[k] = pick;
}

template <class V>
cudaError_t launchSampleV(const void *st, const SampleArgs &a, double *sums, const double *uniforms, int count,
                          uint64_t *out, cudaStream_t s) {
    const V *p = reinterpret_cast<const V *>(st);
    const uint64_t runs = (a.numAmps + kRun - 1) >> kRunBits;
    sampleBlockSums<V><<<(unsigned) runs, 256, 0, s>>>(p, a, sums);
    sampleScan<<<1, 1024, 0, s>>>(sums, runs);
    if (count > 0) sampleFind<V><<<(unsigned) ((count + 7) / 8), 256, 0, s>>>(p, a, sums, runs, uniforms, count, out);
    return cudaGetLastError();
}

}  // namespace

uint64_t sampleScratchCount(uint64_t numAmps) { return (numAmps + kRun - 1) >> kRunBits; }

cudaError_t launchSample(const void *st, bool single, const SampleArgs &a, double *sums, const double *uniforms,
                         int count, uint64_t *out, cudaStream_t s) {
    return single ? launchSampleV<float2>(st, a, sums, uniforms, count, out, s)
                  : launchSampleV<double2>(st, a, sums, uniforms, count, out, s);
}

}  // namespace dgq
