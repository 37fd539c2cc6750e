// Process-wide cache of packed translation operators (mixed form).
//
// The folded M2M / L2L / M2L operators and the E2 skeleton factors depend on
// the operator files, the kernel, the accuracy level and the (width, wedge,
// child or offset) they serve -- not on the geometry -- so every session on a
// device that uses the same files shares one packed copy of each.  Entries are
// reference counted: a session holds the entries it uses, the cache keeps
// only weak references, and the device memory (16 MiB chunks shared by many
// operators) is released with the last session that uses any operator in it.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <mutex>
#include <string>

namespace ddfmm {

// One device allocation, freed when its last holder goes away.
class DevChunk {
public:
    DevChunk(int device, size_t bytes);
    ~DevChunk();
    DevChunk(const DevChunk&) = delete;
    DevChunk& operator=(const DevChunk&) = delete;
    float* data() const { return p_; }
    size_t bytes() const { return bytes_; }
    // bytes of all chunks alive on a device (packed operators of every session)
    static size_t live_bytes(int device);

private:
    float* p_ = nullptr;
    size_t bytes_ = 0;
    int device_ = 0;
};

struct PackedOp {
    std::shared_ptr<DevChunk> chunk;  // keeps the memory alive
    const float* p;
};

class OpCache {
public:
    // the live entry under key, or null
    static std::shared_ptr<PackedOp> find(const std::string& key);
    // Publishes op under key unless a live entry exists; returns the entry
    // that is in the cache afterwards (op itself or the earlier one).
    static std::shared_ptr<PackedOp> publish(const std::string& key, const std::shared_ptr<PackedOp>& op);
    // the part of a key that identifies files, kernel, accuracy, layout and device
    static std::string context(int device, int kernel, int accu, int npq, const std::string& ld_path,
                               const std::string& hd_path);
};

}  // namespace ddfmm
