// Stand-in for the RR-CUDA helper library, whose git submodule is empty in the reference tree.
// Only the API the reference's kernel libraries call is provided (inferred from their call
// sites, e.g. solver/lib/rrgsim_common/src/co_grid_context.cu:20-42): an owning device array,
// a checked launcher, symbol/array copies and a device sync. Test infrastructure only.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace RR::CUDA {

inline void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

enum CopyKind { ToDevice, ToHost, DeviceToDevice };

template <typename T>
class CuDarray {
public:
    CuDarray() = default;
    explicit CuDarray(size_t n) { alloc(n); }
    CuDarray(const CuDarray&) = delete;
    CuDarray& operator=(const CuDarray&) = delete;
    CuDarray(CuDarray&& o) noexcept { steal(o); }
    CuDarray& operator=(CuDarray&& o) noexcept {
        if (this != &o) { release(); steal(o); }
        return *this;
    }
    CuDarray& operator=(const std::vector<T>& v) {
        alloc(v.size());
        if (!v.empty()) check(cudaMemcpy(p_, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice), "H2D");
        return *this;
    }
    ~CuDarray() { release(); }

    operator T*() const { return p_; }
    size_t size() const { return n_; }
    void set_zero() { if (p_) check(cudaMemset(p_, 0, sizeof(T) * n_), "memset"); }
    std::vector<T> to_vector() const {
        std::vector<T> v(n_);
        to_vector(v);
        return v;
    }
    void to_vector(std::vector<T>& v) const {
        v.resize(n_);
        if (n_) check(cudaMemcpy(v.data(), p_, sizeof(T) * n_, cudaMemcpyDeviceToHost), "D2H");
    }
    T to_mem() const {
        T v{};
        to_mem(v);
        return v;
    }
    void to_mem(T& v) const { check(cudaMemcpy(&v, p_, sizeof(T), cudaMemcpyDeviceToHost), "D2H"); }
    static double get_total_allocated_mb() { return total() / (1024.0 * 1024.0); }
    friend void swap(CuDarray& a, CuDarray& b) noexcept {
        std::swap(a.p_, b.p_);
        std::swap(a.n_, b.n_);
    }

private:
    static size_t& total() { static size_t t = 0; return t; }
    void alloc(size_t n) {
        release();
        if (n) {
            check(cudaMalloc(&p_, sizeof(T) * n), "cudaMalloc");
            total() += sizeof(T) * n;
        }
        n_ = n;
    }
    void release() {
        if (p_) { cudaFree(p_); total() -= sizeof(T) * n_; }
        p_ = nullptr;
        n_ = 0;
    }
    void steal(CuDarray& o) {
        p_ = o.p_; n_ = o.n_;
        o.p_ = nullptr; o.n_ = 0;
    }
    T* p_ = nullptr;
    size_t n_ = 0;
};

template <typename K>
struct Launcher {
    K kernel;
    dim3 grid, block;
    size_t smem;
    template <typename... A>
    void operator()(A&&... args) const {
        kernel<<<grid, block, smem>>>(std::forward<A>(args)...);
        check(cudaGetLastError(), "kernel launch");
    }
};

template <typename K>
Launcher<K> CuCall(K kernel, dim3 grid, dim3 block, size_t smem = 0) {
    return Launcher<K>{kernel, grid, block, smem};
}

template <typename T>
void CuCopyToSymbol(const T& value, const T& symbol, CopyKind) {
    check(cudaMemcpyToSymbol(symbol, &value, sizeof(T)), "cudaMemcpyToSymbol");
}

template <typename T>
void CuCopyFromTo(const CuDarray<T>& src, CuDarray<T>& dst, CopyKind) {
    check(cudaMemcpy(static_cast<T*>(dst), static_cast<T*>(src), sizeof(T) * src.size(),
                     cudaMemcpyDeviceToDevice), "D2D");
}

inline void CuDeviceSync() { check(cudaDeviceSynchronize(), "cudaDeviceSynchronize"); }

}  // namespace RR::CUDA
