// Host and device N-dimensional arrays with the reference's public interface
// (include/Array.h:94-634 of rte-rrtmgp-cpp, the parts callers of the radiation classes use):
// Fortran order (first index fastest), 1-based element access, dims queried with dim(i),
// raw storage with ptr().  Array_gpu owns device memory obtained with cudaMalloc when it is
// created with dimensions or from a host Array; callers own every array they pass to the
// radiation classes, as in the reference.
#ifndef RRTMGP_B200_CPP_ARRAY_H
#define RRTMGP_B200_CPP_ARRAY_H

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <numeric>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "rrtmgp_b200_cpp.h"

template <typename T, int N> class Array_gpu;

namespace rrtmgp_b200_cpp {
template <int N>
inline int product(const std::array<int, N>& d)
{
    long long p = 1;
    for (int i = 0; i < N; ++i) {
        if (d[i] < 0) throw std::runtime_error("Array: negative dimension");
        p *= d[i];
    }
    if (p > 0x7fffffffLL) throw std::runtime_error("Array: more than 2^31-1 elements");
    return int(p);
}
}  // namespace rrtmgp_b200_cpp

template <typename T, int N>
class Array
{
  public:
    Array() { dims_.fill(0); }
    explicit Array(const std::array<int, N>& dims) : dims_(dims), data_(rrtmgp_b200_cpp::product<N>(dims)) {}
    Array(std::vector<T>&& data, const std::array<int, N>& dims) : dims_(dims), data_(std::move(data))
    {
        if (int(data_.size()) != rrtmgp_b200_cpp::product<N>(dims_))
            throw std::runtime_error("Array: data size does not match the dimensions");
    }
    Array(const std::vector<T>& data, const std::array<int, N>& dims) : Array(std::vector<T>(data), dims) {}
    // Device-to-host copy (synchronous).
    explicit Array(const Array_gpu<T, N>& a);

    void set_dims(const std::array<int, N>& dims)
    {
        if (!data_.empty() && int(data_.size()) != rrtmgp_b200_cpp::product<N>(dims))
            throw std::runtime_error("Array: initialised arrays can not be resized");
        dims_ = dims;
        data_.resize(rrtmgp_b200_cpp::product<N>(dims));
    }

    T* ptr() { return data_.data(); }
    const T* ptr() const { return data_.data(); }
    std::vector<T>& v() { return data_; }
    const std::vector<T>& v() const { return data_; }
    int size() const { return int(data_.size()); }
    int dim(int i) const { return dims_.at(i - 1); }
    const std::array<int, N>& get_dims() const { return dims_; }

    // 1-based, first index fastest.
    T& operator()(const std::array<int, N>& idx) { return data_[offset(idx)]; }
    const T& operator()(const std::array<int, N>& idx) const { return data_[offset(idx)]; }

    T max() const { return *std::max_element(data_.begin(), data_.end()); }
    T min() const { return *std::min_element(data_.begin(), data_.end()); }
    void fill(const T v) { std::fill(data_.begin(), data_.end(), v); }

  private:
    int offset(const std::array<int, N>& idx) const
    {
        int o = 0, stride = 1;
        for (int i = 0; i < N; ++i) {
            o += (idx[i] - 1) * stride;
            stride *= dims_[i];
        }
        return o;
    }
    std::array<int, N> dims_;
    std::vector<T> data_;
};

template <typename T, int N>
class Array_gpu
{
  public:
    Array_gpu() { dims_.fill(0); }
    explicit Array_gpu(const std::array<int, N>& dims) : dims_(dims), n_(rrtmgp_b200_cpp::product<N>(dims)) { alloc(); }
    explicit Array_gpu(const Array<T, N>& a) : dims_(a.get_dims()), n_(a.size())
    {
        alloc();
        if (n_)
            rrtmgp_b200_cpp::check_cuda(cudaMemcpy(ptr_, a.ptr(), bytes(), cudaMemcpyHostToDevice), "Array_gpu H2D");
    }
    Array_gpu(const Array_gpu& a) : dims_(a.dims_), n_(a.n_)
    {
        alloc();
        if (n_)
            rrtmgp_b200_cpp::check_cuda(cudaMemcpy(ptr_, a.ptr_, bytes(), cudaMemcpyDeviceToDevice), "Array_gpu D2D");
    }
    Array_gpu(Array_gpu&& a) noexcept : dims_(a.dims_), n_(a.n_), ptr_(a.ptr_)
    {
        a.ptr_ = nullptr;
        a.n_ = 0;
        a.dims_.fill(0);
    }
    // Assignment copies into an array of the same size, or into an empty one.
    Array_gpu& operator=(const Array_gpu& a)
    {
        if (this == &a) return *this;
        if (!(n_ == a.n_ || (n_ == 0 && ptr_ == nullptr)))
            throw std::runtime_error("Initialised arrays can not be resized");
        dims_ = a.dims_;
        if (ptr_ == nullptr) {
            n_ = a.n_;
            alloc();
        }
        if (n_)
            rrtmgp_b200_cpp::check_cuda(cudaMemcpy(ptr_, a.ptr_, bytes(), cudaMemcpyDeviceToDevice), "Array_gpu D2D");
        return *this;
    }
    Array_gpu& operator=(Array_gpu&& a) noexcept
    {
        std::swap(dims_, a.dims_);
        std::swap(n_, a.n_);
        std::swap(ptr_, a.ptr_);
        return *this;
    }
    ~Array_gpu()
    {
        if (ptr_) cudaFree(ptr_);
    }

    void set_dims(const std::array<int, N>& dims)
    {
        const int n = rrtmgp_b200_cpp::product<N>(dims);
        if (ptr_ && n != n_) throw std::runtime_error("Initialised arrays can not be resized");
        dims_ = dims;
        if (!ptr_) {
            n_ = n;
            alloc();
        }
    }

    T* ptr() { return ptr_; }
    const T* ptr() const { return ptr_; }
    int size() const { return n_; }
    int dim(int i) const { return dims_.at(i - 1); }
    const std::array<int, N>& get_dims() const { return dims_; }

  private:
    size_t bytes() const { return size_t(n_) * sizeof(T); }
    void alloc()
    {
        if (n_ > 0) rrtmgp_b200_cpp::check_cuda(cudaMalloc(reinterpret_cast<void**>(&ptr_), bytes()), "Array_gpu cudaMalloc");
    }
    std::array<int, N> dims_;
    int n_ = 0;
    T* ptr_ = nullptr;
};

template <typename T, int N>
Array<T, N>::Array(const Array_gpu<T, N>& a) : dims_(a.get_dims()), data_(a.size())
{
    // The class API's work runs on rrtmgp_b200_cpp::stream(); finish it before reading.
    rrtmgp_b200_cpp::check_cuda(cudaStreamSynchronize(rrtmgp_b200_cpp::stream_ref()), "Array D2H sync");
    if (a.size())
        rrtmgp_b200_cpp::check_cuda(cudaMemcpy(data_.data(), a.ptr(), sizeof(T) * data_.size(), cudaMemcpyDeviceToHost),
                                    "Array D2H");
}

#endif
