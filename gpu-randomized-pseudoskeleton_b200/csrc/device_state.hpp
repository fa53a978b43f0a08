// Per-device bookkeeping of state the library sets up once (plain C++, no CUDA types, so the
// host logic is testable without a GPU).
//
// CUDA keeps a kernel's dynamic-shared-memory limit per device: a limit raised while device 0
// was current does not apply on device 1. Every "set once" step is therefore keyed by the
// device ordinal as well as by the kernel.
#pragma once

#include <cstddef>
#include <map>
#include <mutex>
#include <utility>

namespace pskel {

constexpr int kMaxDevices = 64;

// Largest dynamic-shared-memory limit set so far for each (kernel, device).
class SmemAttrTable {
public:
    // Makes sure the limit of (func, dev) is at least `bytes`: when the recorded limit is
    // lower, calls set(bytes) (which applies the attribute and returns true on success) and
    // records the new limit. Limits only grow, so a kernel launched concurrently from another
    // host thread with a smaller need keeps a valid limit. Returns false if set() failed.
    template <typename Set>
    bool raise(const void *func, int dev, size_t bytes, Set &&set) {
        std::lock_guard<std::mutex> lk(mu_);
        size_t &have = table_[std::make_pair(func, dev)];
        if (have >= bytes) return true;
        if (!set(bytes)) return false;
        have = bytes;
        return true;
    }
    size_t recorded(const void *func, int dev) {
        std::lock_guard<std::mutex> lk(mu_);
        auto it = table_.find(std::make_pair(func, dev));
        return it == table_.end() ? 0 : it->second;
    }

private:
    std::mutex mu_;
    std::map<std::pair<const void *, int>, size_t> table_;
};

// One lazily used slot of T per device ordinal; get() returns null for an ordinal outside
// [0, kMaxDevices).
template <typename T>
class PerDevice {
public:
    T *get(int dev) { return dev >= 0 && dev < kMaxDevices ? &slots_[dev] : nullptr; }

private:
    T slots_[kMaxDevices];
};

}  // namespace pskel
