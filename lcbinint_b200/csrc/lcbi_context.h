// Host-side state of one lcbi_gpu_context: device, stream, and growable
// device workspaces reused across calls (no allocation on the steady path).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace lcbi {

struct Buffer {
    void* ptr = nullptr;
    size_t bytes = 0;
};

struct Context {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    std::string error;
    int64_t launches = 0;

    Buffer in[8];
    Buffer out[8];
    Buffer work[8];

    std::vector<Buffer*> all_buffers()
    {
        std::vector<Buffer*> v;
        for (auto& b : in) v.push_back(&b);
        for (auto& b : out) v.push_back(&b);
        for (auto& b : work) v.push_back(&b);
        return v;
    }

    ~Context();
    bool fail(const char* what, cudaError_t e);
    bool fail(const std::string& what);
    bool check(const char* what, cudaError_t e);
    bool ensure(Buffer& b, size_t bytes);
    bool finish();

    template <typename T>
    bool stage_in(Buffer& buf, const T* src, size_t count, bool device_ptrs, const T** out);
    template <typename T>
    bool stage_out(Buffer& buf, T* dst, size_t count, bool device_ptrs, T** out);
    template <typename T>
    bool copy_back(T* dst, const T* dev, size_t count, bool device_ptrs);
};

} // namespace lcbi
