// kc_measure_peaks (include/kmer_peaks.h): the roofline denominators of the
// counting path, measured on the device it runs on.
//
//   * HBM: a 16-byte-vector device copy of half the footprint into the other
//     half (bytes read + written per second);
//   * random atomics: one u32 atomic per thread iteration at an index hashed
//     from the iteration number over the whole footprint (far above L2, so
//     nearly every atomic misses L2 as the counter's filter and table atomics
//     do).  Two forms: atomicAdd with the result unused (a reduction, as the
//     count add) and atomicOr whose old value is consumed (as the filter's
//     first-occurrence test); then both again on a 32 MiB footprint that
//     stays in L2;
//   * the pinned host -> device link (cudaMemcpyAsync of one pinned buffer).
// Each figure is the best of three timed launches after one untimed one.

#include <cstdio>
#include <cstring>

#include <cuda_runtime.h>

#include "../../include/kmer_count.h"
#include "../../include/kmer_peaks.h"
#include "kc_internal.h"

namespace {

int err(int code, const char* what, cudaError_t e) {
    char buf[256];
    snprintf(buf, sizeof buf, "kc_measure_peaks: %s: %s", what, cudaGetErrorString(e));
    return kc_internal_set_error(code, buf);
}

// splitmix64's output function (Steele, Lea, Flood 2014): a bijective 64-bit
// mix, so iteration numbers map to well-spread indices.
__device__ __forceinline__ uint64_t mix64(uint64_t x) {
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

__global__ void __launch_bounds__(256) copy16(const uint4* __restrict__ src, uint4* __restrict__ dst, uint64_t n) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) dst[i] = src[i];
}

// RETURN = false: atomicAdd(+1), result unused (compiled as a reduction).
// RETURN = true: atomicOr of one bit, old value folded into `acc`, which is
// stored only if it equals a value it never takes in practice (keeps the
// returns live without adding traffic).
template <bool RETURN>
__global__ void __launch_bounds__(256) random_atomics(uint32_t* words, uint64_t mask, uint64_t ops, uint64_t seed) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint32_t acc = 0;
#pragma unroll 4
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ops; i += stride) {
        const uint64_t h = mix64(i + seed);
        uint32_t* p = words + (h & mask);
        if constexpr (RETURN) {
            acc += atomicOr(p, 1u << (h >> 59));
        } else {
            atomicAdd(p, 1u);
        }
    }
    if constexpr (RETURN) {
        if (acc == 0x9e3779b9u) words[0] = acc;
    }
}

struct Scratch {
    void* dev = nullptr;
    void* host = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    ~Scratch() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
        if (s) cudaStreamDestroy(s);
        if (dev) cudaFree(dev);
        if (host) cudaFreeHost(host);
    }
};

struct DeviceGuard {
    int prev = -1;
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

extern "C" int kc_measure_peaks(int device, uint64_t footprint_bytes, kc_peaks* out) {
    if (!out) return kc_internal_set_error(KC_ERR_INVALID, "kc_measure_peaks: out is NULL");
    if (footprint_bytes < (256ull << 20) || footprint_bytes > (32ull << 30) ||
        (footprint_bytes & (footprint_bytes - 1)))
        return kc_internal_set_error(KC_ERR_INVALID,
                                     "kc_measure_peaks: footprint must be a power of two from 256 MiB to 32 GiB");
    if (device < 0) return kc_internal_set_error(KC_ERR_INVALID, "kc_measure_peaks: negative device");
    memset(out, 0, sizeof *out);

    DeviceGuard guard;
    cudaError_t e;
    if ((e = cudaGetDevice(&guard.prev)) != cudaSuccess) return err(KC_ERR_DEVICE, "cudaGetDevice", e);
    if ((e = cudaSetDevice(device)) != cudaSuccess) return err(KC_ERR_DEVICE, "cudaSetDevice", e);
    int sms = 0, per_sm = 0;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess)
        return err(KC_ERR_DEVICE, "cudaDeviceGetAttribute", e);

    Scratch w;
    const uint64_t link_bytes = footprint_bytes < (1ull << 30) ? footprint_bytes : (1ull << 30);
    if ((e = cudaMalloc(&w.dev, footprint_bytes)) != cudaSuccess) return err(KC_ERR_NOMEM, "cudaMalloc", e);
    if ((e = cudaHostAlloc(&w.host, link_bytes, cudaHostAllocDefault)) != cudaSuccess)
        return err(KC_ERR_NOMEM, "cudaHostAlloc", e);
    memset(w.host, 0x5a, link_bytes);
    if ((e = cudaStreamCreateWithFlags(&w.s, cudaStreamNonBlocking)) != cudaSuccess)
        return err(KC_ERR_DEVICE, "cudaStreamCreate", e);
    if ((e = cudaEventCreate(&w.a)) != cudaSuccess || (e = cudaEventCreate(&w.b)) != cudaSuccess)
        return err(KC_ERR_DEVICE, "cudaEventCreate", e);
    if ((e = cudaMemsetAsync(w.dev, 0, footprint_bytes, w.s)) != cudaSuccess)
        return err(KC_ERR_DEVICE, "cudaMemsetAsync", e);

    auto best_ms = [&](auto&& launch, float* ms) -> int {
        *ms = 0.f;
        for (int rep = 0; rep < 4; ++rep) {
            cudaError_t e2;
            if ((e2 = cudaEventRecord(w.a, w.s)) != cudaSuccess) return err(KC_ERR_DEVICE, "cudaEventRecord", e2);
            if ((e2 = launch(rep)) != cudaSuccess) return err(KC_ERR_DEVICE, "launch", e2);
            if ((e2 = cudaEventRecord(w.b, w.s)) != cudaSuccess) return err(KC_ERR_DEVICE, "cudaEventRecord", e2);
            if ((e2 = cudaEventSynchronize(w.b)) != cudaSuccess) return err(KC_ERR_DEVICE, "synchronize", e2);
            float t = 0.f;
            if ((e2 = cudaEventElapsedTime(&t, w.a, w.b)) != cudaSuccess)
                return err(KC_ERR_DEVICE, "cudaEventElapsedTime", e2);
            if (rep > 0 && (*ms == 0.f || t < *ms)) *ms = t;  // rep 0 is the untimed warm-up
        }
        return KC_OK;
    };

    // HBM copy: first half -> second half.
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, copy16, 256, 0)) != cudaSuccess)
        return err(KC_ERR_DEVICE, "occupancy", e);
    const uint64_t half16 = footprint_bytes / 2 / 16;
    const uint4* src = (const uint4*)w.dev;
    uint4* dst = (uint4*)w.dev + half16;
    float ms = 0.f;
    int rc = best_ms([&](int) {
        copy16<<<sms * per_sm, 256, 0, w.s>>>(src, dst, half16);
        return cudaGetLastError();
    }, &ms);
    if (rc) return rc;
    out->hbm_copy_gbs = 2.0 * (double)(half16 * 16) / (ms * 1e-3) / 1e9;

    // Random atomics over the whole footprint, one op per word on average.
    const uint64_t nwords = footprint_bytes / 4;
    const uint64_t mask = nwords - 1;
    out->footprint_bytes = footprint_bytes;
    out->ops = nwords;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, random_atomics<false>, 256, 0)) != cudaSuccess)
        return err(KC_ERR_DEVICE, "occupancy", e);
    rc = best_ms([&](int rep) {
        random_atomics<false><<<sms * per_sm, 256, 0, w.s>>>((uint32_t*)w.dev, mask, nwords, (uint64_t)rep << 40);
        return cudaGetLastError();
    }, &ms);
    if (rc) return rc;
    out->red_add_gops = (double)nwords / (ms * 1e-3) / 1e9;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, random_atomics<true>, 256, 0)) != cudaSuccess)
        return err(KC_ERR_DEVICE, "occupancy", e);
    rc = best_ms([&](int rep) {
        random_atomics<true><<<sms * per_sm, 256, 0, w.s>>>((uint32_t*)w.dev, mask, nwords, ((uint64_t)rep << 40) | (1ull << 39));
        return cudaGetLastError();
    }, &ms);
    if (rc) return rc;
    out->or_return_gops = (double)nwords / (ms * 1e-3) / 1e9;

    // The same atomics on an L2-resident footprint (the first 32 MiB).
    const uint64_t l2_words = (32ull << 20) / 4;
    out->l2_footprint_bytes = l2_words * 4;
    rc = best_ms([&](int rep) {
        random_atomics<false><<<sms * per_sm, 256, 0, w.s>>>((uint32_t*)w.dev, l2_words - 1, nwords,
                                                             ((uint64_t)rep << 40) | (1ull << 38));
        return cudaGetLastError();
    }, &ms);
    if (rc) return rc;
    out->l2_red_add_gops = (double)nwords / (ms * 1e-3) / 1e9;
    rc = best_ms([&](int rep) {
        random_atomics<true><<<sms * per_sm, 256, 0, w.s>>>((uint32_t*)w.dev, l2_words - 1, nwords,
                                                            ((uint64_t)rep << 40) | (3ull << 38));
        return cudaGetLastError();
    }, &ms);
    if (rc) return rc;
    out->l2_or_return_gops = (double)nwords / (ms * 1e-3) / 1e9;

    // Pinned host -> device.
    rc = best_ms([&](int) { return cudaMemcpyAsync(w.dev, w.host, link_bytes, cudaMemcpyHostToDevice, w.s); }, &ms);
    if (rc) return rc;
    out->h2d_gbs = (double)link_bytes / (ms * 1e-3) / 1e9;
    return KC_OK;
}
