// Shared packed-operator cache (see opcache.hpp).
#include "opcache.hpp"

#include <sys/stat.h>

#include <cstdio>
#include <stdexcept>

#include "kernels.cuh"

namespace ddfmm {

namespace {
std::mutex g_mu;
std::map<int, size_t> g_live;                              // device -> live chunk bytes
std::map<std::string, std::weak_ptr<PackedOp> > g_entries;  // key -> entry
}  // namespace

DevChunk::DevChunk(int device, size_t bytes) : bytes_(bytes), device_(device) {
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    const cudaError_t e = cudaMalloc(&p_, bytes ? bytes : 16);
    cudaSetDevice(prev);
    if (e != cudaSuccess) {
        p_ = nullptr;
        throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(e) + " (packed operator chunk)");
    }
    std::lock_guard<std::mutex> lk(g_mu);
    g_live[device_] += bytes_;
}

DevChunk::~DevChunk() {
    if (!p_) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device_);
    cudaFree(p_);
    cudaSetDevice(prev);
    std::lock_guard<std::mutex> lk(g_mu);
    g_live[device_] -= bytes_;
}

size_t DevChunk::live_bytes(int device) {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_live.find(device);
    return it == g_live.end() ? 0 : it->second;
}

std::shared_ptr<PackedOp> OpCache::find(const std::string& key) {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_entries.find(key);
    if (it == g_entries.end()) return nullptr;
    std::shared_ptr<PackedOp> p = it->second.lock();
    if (!p) g_entries.erase(it);
    return p;
}

std::shared_ptr<PackedOp> OpCache::publish(const std::string& key, const std::shared_ptr<PackedOp>& op) {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_entries.find(key);
    if (it != g_entries.end()) {
        std::shared_ptr<PackedOp> p = it->second.lock();
        if (p) return p;
    }
    g_entries[key] = op;
    return op;
}

std::string OpCache::context(int device, int kernel, int accu, int npq, const std::string& ld_path,
                             const std::string& hd_path) {
    auto ident = [](const std::string& path) {
        struct stat st;
        if (stat(path.c_str(), &st) != 0) return path + ":?";
        char b[128];
        snprintf(b, sizeof b, ":%lld:%lld:%lld:%lld", (long long)st.st_dev, (long long)st.st_ino,
                 (long long)st.st_size, (long long)st.st_mtime);
        return path + b;
    };
    char head[96];
    // the packed layout depends on the K block of the tensor-core kernel
    snprintf(head, sizeof head, "dev%d|k%d|a%d|npq%d|nkb16=%d|", device, kernel, accu, npq, umma_nkb(8));
    return head + ident(ld_path) + "|" + ident(hd_path);
}

}  // namespace ddfmm
