// Per-particle FP64 kernels around the neighbour sums (see integrate.cu).
#pragma once

#include "common.cuh"

namespace sphb
{

template<class T>
struct IntegrateArrays
{
    double *x, *y, *z;
    double *vx, *vy, *vz;
    double *xm1, *ym1, *zm1;
    double* temp;
    double* duM1;
    const double* du;
    const T *ax, *ay, *az;
    BatchView batch; // an ensemble: per-instance dt, dtm1, cv; padding slots skipped
};

//! the fixed-point frame of the FP32 J-loops: q = (x - lo) * invUnit, x - lo = q * unit
struct FixedFrame
{
    double lo[3];
    double invUnit[3];
    double unit[3];
};

FixedFrame fixedFrameOf(const DevBox& box);

//! pos = (x, y, z, m) in FP64 and/or posq = fixed-point (x, y, z) + float m; either pointer may be null
int packPositions(const double* x, const double* y, const double* z, const double* m, size_t n, double4* pos,
                  int4* posq, const DevBox& box, cudaStream_t s);

//! packPositions and, in the same pass, the bounding boxes of computeBlockBoxes (neighbors.cuh)
int packPositionsAndBoxes(const double* x, const double* y, const double* z, const double* m, size_t n, double4* pos,
                          int4* posq, const DevBox& box, float4* boxLo, float4* boxHi, cudaStream_t s);

template<class T>
int launchPositions(size_t n, const IntegrateArrays<T>& a, const DevBox& box, double dt, double dtm1, double cv,
                    cudaStream_t s);

int launchUpdateH(size_t n, unsigned ng0, const unsigned* nc, double* h, uint64_t* keys, unsigned* flag,
                  cudaStream_t s, const uint8_t* inst = nullptr);

//! eKin (sum m v^2), eInt, linear momentum (3), angular momentum (3), sum nc -> out9 (device)
int conservedSums(size_t n, const double* x, const double* y, const double* z, const double* vx, const double* vy,
                  const double* vz, const double* m, const double* temp, const unsigned* nc, double cv,
                  double* partial, int maxBlocks, double* out9, cudaStream_t s);

//! the extrema of x, y and z into out6 as ordered bits {min x, max x, min y, max y, min z, max z}, stream-ordered
int minMax3(const double* x, const double* y, const double* z, size_t n, unsigned long long* out6, cudaStream_t s);
/*! the smoothing lengths the end-of-step update (launchUpdateH) will produce from nc and h, into out as SPHB_F32 or
 *  SPHB_F64, with none of its other effects: for copying them out before the step ends */
int predictH(size_t n, unsigned ng0, const unsigned* nc, const double* h, void* out, int outType, cudaStream_t s);

/*! dst[0] = v0 and, with count 2, dst[1] = v1, written by a kernel: unlike a copy from host memory, it never waits on
 *  the stream for a copy engine busy with another stream's transfers */
int setWords(unsigned long long* dst, int count, unsigned long long v0, unsigned long long v1, cudaStream_t s);

} // namespace sphb
