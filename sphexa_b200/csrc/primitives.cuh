// Device buffers, scans and gathers used by the domain and tree code.
#pragma once

#include "common.cuh"

namespace sphb
{

//! Owning device array that only grows; contents are kept on growth when `keep` is set.
template<class T>
class DeviceBuffer
{
public:
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    ~DeviceBuffer() { release(); }

    int reserve(size_t n, bool keep = false, cudaStream_t stream = 0)
    {
        if (n <= cap_) { return kOk; }
        size_t newCap = n + n / 16 + 16;
        T* p          = nullptr;
        SPHB_CUDA_TRY(cudaMalloc(&p, newCap * sizeof(T)));
        if (keep && ptr_ && cap_)
        {
            SPHB_CUDA_TRY(cudaMemcpyAsync(p, ptr_, cap_ * sizeof(T), cudaMemcpyDeviceToDevice, stream));
            SPHB_CUDA_TRY(cudaStreamSynchronize(stream));
        }
        release();
        ptr_ = p;
        cap_ = newCap;
        return kOk;
    }
    void release()
    {
        if (ptr_) { cudaFree(ptr_); }
        ptr_ = nullptr;
        cap_ = 0;
    }
    void swap(DeviceBuffer& o)
    {
        std::swap(ptr_, o.ptr_);
        std::swap(cap_, o.cap_);
    }
    T* data() const { return ptr_; }
    size_t capacity() const { return cap_; }

private:
    T* ptr_{nullptr};
    size_t cap_{0};
};

//! exclusive prefix sum of n int32 values into out (out may alias in); out[n] receives the total.
//! Uses tmp (>= scanTempInts(n) ints).
size_t scanTempInts(size_t n);
int exclusiveScan(const int* in, int* out, size_t n, int* tmp, cudaStream_t stream);

//! dst_f[i] = src_f[order[i]] for up to 16 fields of 8-byte elements
int gather8(const uint32_t* order, size_t n, int numFields, const void* const* src, void* const* dst,
            cudaStream_t stream);

//! number of kernel launches issued by this library in this process (launch accounting)
uint64_t& launchCounter();
inline void countLaunch(uint64_t k = 1) { launchCounter() += k; }

} // namespace sphb
