// prob_static.cu -- P(bit = 0) for every address bit, without allocating.
//
// dgq_calcProbOfAllZeroNoAlloc runs the same two kernels as the register
// read-out (probKernel + probFinalize in kernels.cu), but their scratch (the
// per-CTA partial sums) lives in the file-scope device array below instead
// of a buffer from cudaMalloc. It is meant for callers that must not
// allocate GPU memory while they call us:
//   * hosts that reserve all device memory up front and hand out pieces
//     themselves (a framework's caching allocator, a serving process with a
//     fixed HBM budget), where an allocation behind their back can fail or
//     fragment their pool,
//   * latency-sensitive loops, where cudaMalloc/cudaFree would synchronise
//     the device.
// The state and the output must live on the device that is current when
// the call is made (checked with cudaPointerGetAttributes, a host query);
// the scratch is that device's copy of the array.
// The array holds kStaticProbCtas x 17 doubles (2,228,224 bytes = 2.125 MiB)
// and stays resident on every GPU that loads libdgq until the process exits.
// That bounds the state to 2^30 amplitudes (numBits <= 30). All calls share
// the array and it keeps the last call's partial sums; nothing in it needs
// to start at zero (each CTA writes every slot it owns before the finalise
// kernel reads it), but calls whose kernels overlap on the GPU (different
// streams, no ordering between them) race on it and give wrong results.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>

#include "dgq.h"
#include "kernels.h"

namespace dgq {

constexpr int kStaticProbCtas = 1 << 14;     // 2^30 amplitudes at 2^16 per CTA
constexpr int kStaticProbMaxBits = 30;

static __device__ __align__(256) double g_probScratch[kStaticProbCtas * 17];

// host-side copy of the scratch array's device address, per device
static std::mutex g_scratchMutex;
static double *g_scratchAddr[64] = {nullptr};

bool raiseExternal(int code, const char *func, const char *detail);

}  // namespace dgq

extern "C" int dgq_calcProbOfAllZeroNoAlloc(const void *deviceState, int numBits, double *deviceProbs,
                                            void *stream) {
    using namespace dgq;
    if (!deviceState || !deviceProbs) {
        raiseExternal(104, __func__, "null state or output pointer");
        return -1;
    }
    if (numBits < 1 || numBits > kStaticProbMaxBits) {
        char msg[160];
        snprintf(msg, sizeof msg, "numBits = %d is outside 1..%d, the size the static scratch (%d x 17 doubles) holds",
                 numBits, kStaticProbMaxBits, kStaticProbCtas);
        raiseExternal(104, __func__, msg);
        return -1;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64) {
        raiseExternal(103, __func__, e != cudaSuccess ? cudaGetErrorString(e) : "device ordinal >= 64");
        return -2;
    }
    // both buffers on the current device: the scratch is this device's array,
    // and a pointer into another GPU would make the kernels read peer memory
    for (const void *p : {deviceState, (const void *) deviceProbs}) {
        cudaPointerAttributes at;
        e = cudaPointerGetAttributes(&at, p);
        if (e != cudaSuccess) {
            cudaGetLastError();
            raiseExternal(104, __func__, "state or output pointer is not CUDA memory");
            return -1;
        }
        if ((at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged) ||
            (at.type == cudaMemoryTypeDevice && at.device != dev)) {
            raiseExternal(104, __func__, "state and output must be device memory of the current device");
            return -1;
        }
    }
    double *scratch = nullptr;
    {
        // set-up, once per device, with that device current: the symbol's
        // device address (the array's name is only a host-side stand-in)
        std::lock_guard<std::mutex> lk(g_scratchMutex);
        if (!g_scratchAddr[dev]) {
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_probScratch);
            if (e != cudaSuccess || !p) {
                raiseExternal(103, __func__, e != cudaSuccess ? cudaGetErrorString(e) : "null symbol address");
                return -2;
            }
            g_scratchAddr[dev] = (double *) p;
        }
        scratch = g_scratchAddr[dev];
    }
    ProbArgs a;
    a.nFree = numBits;
    a.kappa = numBits > 16 ? 4 : (numBits > 12 ? numBits - 12 : 0);
    a.rValue = 0;
    for (int i = 0; i < kMaxStateBits; i++) a.freePos[i] = (uint8_t) (i < numBits ? i : 0);
    if (probNumCtas(a) > kStaticProbCtas) {
        raiseExternal(104, __func__, "state larger than the static scratch holds");
        return -1;
    }
    e = launchProb(deviceState, false, a, scratch, deviceProbs, (cudaStream_t) stream);
    if (e != cudaSuccess) {
        raiseExternal(103, __func__, cudaGetErrorString(e));
        return -2;
    }
    return 0;
}
