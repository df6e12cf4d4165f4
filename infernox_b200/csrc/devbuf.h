// Grow-only device buffers owned by a filter or model handle, reused across
// calls so that a scoring call does not pay cudaMalloc/cudaFree each time.
// Every call synchronises its stream before returning, so a buffer is idle
// whenever the next call grows (frees and reallocates) it.  A handle's
// buffers are not shared between threads: one thread per handle at a time.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

namespace cmx {

struct DevArena {
    struct Slot {
        void *p = nullptr;
        size_t cap = 0;
    };
    std::vector<Slot> slots;
    DevArena() = default;
    DevArena(const DevArena &) = delete;
    DevArena &operator=(const DevArena &) = delete;
    ~DevArena() { release(); }
    void release() {
        for (Slot &s : slots) cudaFree(s.p);
        slots.clear();
    }
    template <class T>
    cudaError_t get(int slot, T **out, size_t bytes) {
        if (slots.size() <= (size_t)slot) slots.resize(slot + 1);
        Slot &s = slots[slot];
        if (s.cap < bytes || !s.p) {
            cudaFree(s.p);
            s.p = nullptr;
            s.cap = 0;
            const size_t nb = std::max<size_t>(bytes + bytes / 4, 256);
            cudaError_t e = cudaMalloc(&s.p, nb);
            if (e != cudaSuccess) return e;
            s.cap = nb;
        }
        *out = (T *)s.p;
        return cudaSuccess;
    }
};

// Grow-only pinned host staging buffer (for large host-built tables that are
// copied to the device every call).
struct PinnedBuf {
    void *p = nullptr;
    size_t cap = 0;
    PinnedBuf() = default;
    PinnedBuf(const PinnedBuf &) = delete;
    PinnedBuf &operator=(const PinnedBuf &) = delete;
    ~PinnedBuf() { release(); }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
    }
    template <class T>
    T *get(size_t count) {
        const size_t bytes = count * sizeof(T);
        if (cap < bytes || !p) {
            release();
            const size_t nb = std::max<size_t>(bytes + bytes / 4, 4096);
            if (cudaHostAlloc(&p, nb, cudaHostAllocDefault) != cudaSuccess) {
                p = nullptr;
                return nullptr;
            }
            cap = nb;
        }
        return (T *)p;
    }
};

// true if any of the n residue codes is above 17 (branch-free, vectorisable)
inline bool any_code_above_17(const uint8_t *p, int64_t n) {
    uint8_t acc = 0;
    for (int64_t x = 0; x < n; x++) acc |= (uint8_t)(p[x] > 17);
    return acc != 0;
}

// Let `kern` take as much dynamic shared memory as the current device allows
// a block.  The attribute is process-wide per kernel, so every caller sets
// the same value: host threads launching the same kernel with different
// shared-memory sizes cannot lower the limit under one another's launch.
template <class F>
inline cudaError_t allow_max_dynamic_smem(F kern) {
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa;
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, kern);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
    return e;
}

}  // namespace cmx
