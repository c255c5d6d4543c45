// The typed boundary: particle fields in the caller's own element types, and the stages of the VE force computation
// run in place on a caller's device arrays, bound by the reference's field names
// (sph/include/sph/particles_data.hpp:262-266). This is the drop-in for the reference's per-stage GPU dispatch
// sph::gpu::computeXMass / computeVeDefGradh / computeIdealGasEOS / computeIadDivvCurlv / computeAVswitches /
// computeMomentumEnergy, computePositionsGpu and updateSmoothingLengthGpu (sph/include/sph/sph_gpu.hpp:24-87), whose
// Dataset holds float and double fields side by side (sph/types.hpp:39-46).
//
// Each stage imports the fields it reads from the bound arrays into the simulation's own buffers (converted on the
// device), repacks the neighbour-side records it gathers from them, runs the same kernel as sphb_sim's stage, and
// exports what the reference's function writes, converted to the caller's types. The neighbour lists are built by
// sphb_dataset_xmass (which, like the reference's computeXMass, also runs the search and the smoothing-length
// iteration) and are reused by the later stages of the same force computation.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <initializer_list>

#include "sim.cuh"

namespace sphb
{
namespace
{

size_t widthOf(int dtype) { return dtype == SPHB_F32 || dtype == SPHB_U32 ? 4 : 8; }

bool validDtype(int dtype) { return dtype >= SPHB_F32 && dtype <= SPHB_U64; }

//! the element type of an internal field kind (simimpl::findField: 0 double, 1 J-loop type, 2 uint32, 3 uint64)
int dtypeOfKind(const sphb_sim& s, int kind)
{
    switch (kind)
    {
    case 0: return SPHB_F64;
    case 1: return s.mixed ? SPHB_F32 : SPHB_F64;
    case 2: return SPHB_U32;
    default: return SPHB_U64;
    }
}

__device__ __forceinline__ double loadAs(const void* p, int t, size_t i)
{
    switch (t)
    {
    case SPHB_F32: return double(static_cast<const float*>(p)[i]);
    case SPHB_F64: return static_cast<const double*>(p)[i];
    case SPHB_U32: return double(static_cast<const uint32_t*>(p)[i]);
    default: return double(static_cast<const uint64_t*>(p)[i]);
    }
}

__device__ __forceinline__ void storeAs(void* p, int t, size_t i, double v)
{
    switch (t)
    {
    case SPHB_F32: static_cast<float*>(p)[i] = float(v); break;
    case SPHB_F64: static_cast<double*>(p)[i] = v; break;
    case SPHB_U32: static_cast<uint32_t*>(p)[i] = uint32_t(v); break;
    default: static_cast<uint64_t*>(p)[i] = uint64_t(v); break;
    }
}

//! dst[i] = src[i] converted between element types (64-bit integers are copied bit for bit)
__global__ void convertKernel(const void* src, int st, void* dst, int dt, size_t n)
{
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    {
        if (st == SPHB_U64 && dt == SPHB_U64) { static_cast<uint64_t*>(dst)[i] = static_cast<const uint64_t*>(src)[i]; }
        else { storeAs(dst, dt, i, loadAs(src, st, i)); }
    }
}

int convert(const void* src, int st, void* dst, int dt, size_t n, cudaStream_t stream)
{
    if (n == 0) { return kOk; }
    if (st == dt)
    {
        SPHB_CUDA_TRY(cudaMemcpyAsync(dst, src, n * widthOf(st), cudaMemcpyDeviceToDevice, stream));
        return kOk;
    }
    unsigned blocks = unsigned(std::min<size_t>(ceilDiv(n, 256), size_t(smCount()) * 8));
    convertKernel<<<blocks, 256, 0, stream>>>(src, st, dst, dt, n);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

//! a caller array (host or device) into a device array of another element type, through staging for host data
int importArray(const void* src, int st, bool onDevice, void* dst, int dt, size_t n, void* staging,
                cudaStream_t stream)
{
    if (onDevice) { return convert(src, st, dst, dt, n, stream); }
    if (st == dt)
    {
        SPHB_CUDA_TRY(cudaMemcpyAsync(dst, src, n * widthOf(st), cudaMemcpyHostToDevice, stream));
        return kOk;
    }
    SPHB_CUDA_TRY(cudaMemcpyAsync(staging, src, n * widthOf(st), cudaMemcpyHostToDevice, stream));
    return convert(staging, st, dst, dt, n, stream);
}

const sphb_field* findDesc(const sphb_field* f, int num, const char* name)
{
    for (int q = 0; q < num; ++q)
    {
        if (f[q].name && std::strcmp(f[q].name, name) == 0) { return f + q; }
    }
    return nullptr;
}

/*! a host-to-device copy as pieces of at most 4 MiB, so that small copies of the compute stream, which may share
 *  the copy engine, wait behind one piece at most */
int copyInPieces(void* dst, const void* src, size_t bytes, cudaStream_t stream)
{
    constexpr size_t kPiece = size_t(4) << 20;
    for (size_t off = 0; off < bytes; off += kPiece)
    {
        SPHB_CUDA_TRY(cudaMemcpyAsync(static_cast<char*>(dst) + off, static_cast<const char*>(src) + off,
                                      std::min(kPiece, bytes - off), cudaMemcpyHostToDevice, stream));
    }
    return kOk;
}

/*! the conserved fields and ids of a typed upload or load: into s.f[k] (FP64) and s.idAlt. With lateCopy (a load
 *  from host memory) only x, y, z and m go through the compute stream. The rest follows on the copy stream, after
 *  every earlier use of their buffers on the compute stream, in three groups; the compute stream waits for each only
 *  where the step first reads it (simimpl::waitMidFields, waitLateGroup). h and the ids overlap the sync (unless it
 *  reorders); temp, v and alpha the search and XMass; x_m1, y_m1, z_m1 and du_m1 the J-loops. */
int importConserved(sphb_sim& s, const sphb_field* f, int num, bool onDevice, bool lateCopy = false)
{
    if (!f || num <= 0) { return kErrArg; }
    for (int k = 0; k < kNumConserved; ++k)
    {
        const sphb_field* d = findDesc(f, num, kConservedNames[k]);
        if (!d || !d->data || (d->dtype != SPHB_F32 && d->dtype != SPHB_F64)) { return kErrArg; }
    }
    const sphb_field* idDesc = findDesc(f, num, "id");
    if (!idDesc || !idDesc->data || idDesc->dtype != SPHB_U64) { return kErrArg; }
    bool split = lateCopy && !onDevice && s.copyStream;
    for (int k = 0; k < kNumConserved; ++k)
    {
        // split: x, y, z and m here (the sync reads nothing else unless it reorders), the rest below
        if (split && k != fX && k != fY && k != fZ && k != fM) { continue; }
        const sphb_field* d = findDesc(f, num, kConservedNames[k]);
        SPHB_TRY(importArray(d->data, d->dtype, onDevice, s.f[k].data(), SPHB_F64, s.n, s.fAlt[k].data(), s.stream));
    }
    if (!split)
    {
        SPHB_TRY(importArray(idDesc->data, SPHB_U64, onDevice, s.idAlt.data(), SPHB_U64, s.n, nullptr, s.stream));
        return kOk;
    }
    // the other copies start after x, y, z and m (and after every earlier use of their buffers), in the order the step
    // reads them: issued at once, the copy engine would interleave them and delay what the step needs first. Within
    // each group the copies go first and the conversions of narrower fields after them, so that the copy engine does
    // not wait for a kernel between two copies (the copy stream has the highest priority, so that its conversions
    // do not wait for the blocks of the step's kernels either)
    SPHB_CUDA_TRY(cudaEventRecord(s.copyFork, s.stream));
    SPHB_CUDA_TRY(cudaStreamWaitEvent(s.copyStream, s.copyFork, 0));
    auto group = [&](int which, cudaEvent_t ready) -> int {
        // which: -1 h (with the ids), else a late group
        auto inGroup = [&](int k) { return which < 0 ? k == fH : simimpl::lateGroupOf(k) == which; };
        for (int k = fH; k < kNumConserved; ++k)
        {
            if (!inGroup(k)) { continue; }
            const sphb_field* d = findDesc(f, num, kConservedNames[k]);
            void* dst           = d->dtype == SPHB_F64 ? s.f[k].data() : s.fAlt[k].data();
            SPHB_TRY(copyInPieces(dst, d->data, s.n * widthOf(d->dtype), s.copyStream));
        }
        if (which < 0) { SPHB_TRY(copyInPieces(s.idAlt.data(), idDesc->data, s.n * sizeof(uint64_t), s.copyStream)); }
        for (int k = fH; k < kNumConserved; ++k)
        {
            const sphb_field* d = findDesc(f, num, kConservedNames[k]);
            if (inGroup(k) && d->dtype != SPHB_F64)
            {
                SPHB_TRY(convert(s.fAlt[k].data(), d->dtype, s.f[k].data(), SPHB_F64, s.n, s.copyStream));
            }
        }
        SPHB_CUDA_TRY(cudaEventRecord(ready, s.copyStream));
        return kOk;
    };
    SPHB_TRY(group(-1, s.midReady));
    s.midPending = true;
    for (int g = 0; g < sphb_sim::kLateGroups; ++g)
    {
        SPHB_TRY(group(g, s.lateReady[g]));
        s.latePending[g] = true;
    }
    return kOk;
}

//! names a binding may use: every field this library keeps, plus the EOS outputs rho and p and the energy u
bool bindableName(sphb_sim& s, const char* name, int dtype)
{
    if (std::strcmp(name, "id") == 0 || std::strcmp(name, "keys") == 0) { return dtype == SPHB_U64; }
    if (std::strcmp(name, "nc") == 0) { return dtype == SPHB_U32; }
    bool real = dtype == SPHB_F32 || dtype == SPHB_F64;
    if (std::strcmp(name, "rho") == 0 || std::strcmp(name, "p") == 0 || std::strcmp(name, "u") == 0) { return real; }
    void* ptr = nullptr;
    int kind  = 0;
    return real && simimpl::findField(s, name, &ptr, &kind);
}

const sphb_sim::Binding* boundField(const sphb_sim& s, const char* name)
{
    for (const auto& b : s.bound)
    {
        if (b.name == name) { return &b; }
    }
    return nullptr;
}

//! bound array -> the simulation's buffer of the same field
int importBound(sphb_sim& s, const char* name)
{
    const sphb_sim::Binding* b = boundField(s, name);
    if (!b)
    {
        std::fprintf(stderr, "sphb200: field \"%s\" is not bound\n", name);
        return kErrArg;
    }
    void* ptr = nullptr;
    int kind  = 0;
    if (!simimpl::findField(s, name, &ptr, &kind)) { return kErrArg; }
    return convert(b->data, b->dtype, ptr, dtypeOfKind(s, kind), s.n, s.stream);
}

int importBound(sphb_sim& s, std::initializer_list<const char*> names)
{
    for (const char* name : names)
    {
        SPHB_TRY(importBound(s, name));
    }
    return kOk;
}

//! the simulation's buffer of a field -> the bound array (which must exist unless optional)
int exportBound(sphb_sim& s, const char* name, bool optional = false)
{
    const sphb_sim::Binding* b = boundField(s, name);
    if (!b)
    {
        if (optional) { return kOk; }
        std::fprintf(stderr, "sphb200: field \"%s\" is not bound\n", name);
        return kErrArg;
    }
    void* ptr = nullptr;
    int kind  = 0;
    if (!simimpl::findField(s, name, &ptr, &kind)) { return kErrArg; }
    return convert(ptr, dtypeOfKind(s, kind), b->data, b->dtype, s.n, s.stream);
}

int exportBound(sphb_sim& s, std::initializer_list<const char*> names)
{
    for (const char* name : names)
    {
        SPHB_TRY(exportBound(s, name));
    }
    return kOk;
}

// ------------------------------------------------------------------------------------------------------------------
// neighbour-side records rebuilt from imported fields, exactly as the producing J-loops write them (hydro_ve.cu)
// ------------------------------------------------------------------------------------------------------------------

template<class T>
__global__ void packRecordsKernel(size_t n, const double* h, const double* vx, const double* vy, const double* vz,
                                  const double* alpha, const T* xm, const T* kx, const T* c, const T* prho,
                                  const T* c11, const T* c12, const T* c13, const T* c22, const T* c23, const T* c33,
                                  const T* divv, HydroRec<T>* hrec, GradRec<T>* grec, AVRec<T>* avrec)
{
    size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) { return; }
    T hi            = T(h[i]);
    HydroRec<T> hr  = {T(vx[i]), T(vy[i]), T(vz[i]), T(1) / hi, xm[i], xm[i] / kx[i], c[i], prho[i]};
    hrec[i]         = hr;
    if (grec) { grec[i] = GradRec<T>{c11[i], c12[i], c13[i], c22[i], c23[i], c33[i], divv[i], T(alpha[i])}; }
    if (avrec) { avrec[i] = AVRec<T>{hr.vx, hr.vy, hr.vz, hr.c, hr.vol, divv[i], T(0), T(0)}; }
}

template<class T>
int packRecordsT(sphb_sim& s, bool withGrad)
{
    auto* hrec  = reinterpret_cast<HydroRec<T>*>(s.hrec.data());
    auto* grec  = withGrad ? reinterpret_cast<GradRec<T>*>(s.grec.data()) : nullptr;
    auto* avrec = withGrad ? reinterpret_cast<AVRec<T>*>(s.avrec.data()) : nullptr;
    packRecordsKernel<T><<<ceilDiv(s.n, 256), 256, 0, s.stream>>>(
        s.n, s.f[fH].data(), s.f[fVx].data(), s.f[fVy].data(), s.f[fVz].data(), s.f[fAlpha].data(), s.dptr<T>(dXm),
        s.dptr<T>(dKx), s.dptr<T>(dC), s.dptr<T>(dPrho), s.dptr<T>(dC11), s.dptr<T>(dC12), s.dptr<T>(dC13),
        s.dptr<T>(dC22), s.dptr<T>(dC23), s.dptr<T>(dC33), s.dptr<T>(dDivv), hrec, grec, avrec);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

int packRecords(sphb_sim& s, bool withGrad)
{
    return s.mixed ? packRecordsT<float>(s, withGrad) : packRecordsT<double>(s, withGrad);
}

// ------------------------------------------------------------------------------------------------------------------
// the ideal-gas EOS on typed caller arrays (sph/include/sph/hydro_ve/eos_gpu.cu:44-61, sph/include/sph/eos.hpp:19-50)
// ------------------------------------------------------------------------------------------------------------------

struct EosArrays
{
    const void *temp, *u, *m, *kx, *xm, *gradh;
    void *prho, *c, *rho, *p;
    int tTemp, tU, tM, tKx, tXm, tGradh, tPrho, tC, tRho, tP;
};

__global__ void idealGasEosKernel(size_t first, size_t last, double cv, double gamma, EosArrays a)
{
    size_t i = first + blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= last) { return; }
    double kx   = loadAs(a.kx, a.tKx, i);
    double m    = loadAs(a.m, a.tM, i);
    double xm   = loadAs(a.xm, a.tXm, i);
    double rho  = kx * m / xm;
    double u    = a.u ? loadAs(a.u, a.tU, i) : cv * loadAs(a.temp, a.tTemp, i);
    double tmp  = u * (gamma - 1.0);
    double p    = rho * tmp;
    double c    = sqrt(gamma * tmp);
    double prho = p / (kx * m * m * loadAs(a.gradh, a.tGradh, i));
    storeAs(a.prho, a.tPrho, i, prho);
    storeAs(a.c, a.tC, i, c);
    if (a.rho) { storeAs(a.rho, a.tRho, i, rho); }
    if (a.p) { storeAs(a.p, a.tP, i, p); }
}

//! the particle range of a GroupView at one rank without halos: all particles
int checkRange(const sphb_sim& s, size_t first, size_t last)
{
    return first == 0 && last == s.n ? kOk : kErrArg;
}

//! the later stages of a force computation use the box of its sphb_dataset_xmass
int checkBox(const sphb_sim& s, const sphb_box* box)
{
    if (!box) { return kErrArg; }
    for (int k = 0; k < 3; ++k)
    {
        if (box->lo[k] != s.hbox.lo[k] || box->hi[k] != s.hbox.hi[k] ||
            (box->periodic[k] != 0) != (s.hbox.periodic[k] != 0))
        {
            return kErrState;
        }
    }
    return kOk;
}

int boundEntry(sphb_sim* s, size_t first, size_t last)
{
    if (!s) { return kErrArg; }
    if (s->bound.empty() || s->bdt) { return kErrState; }
    return checkRange(*s, first, last);
}

} // namespace
} // namespace sphb

using namespace sphb;

extern "C" int sphb_sim_upload_fields(sphb_sim* s, const sphb_field* fields, int num_fields, int on_device)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    if (!s) { return SPHB_ERR_ARG; }
    SPHB_TRY(importConserved(*s, fields, num_fields, on_device != 0));
    s->id.swap(s->idAlt);
    return simimpl::finishUpload(*s);
}

extern "C" int sphb_sim_load_fields(sphb_sim* s, const sphb_field* fields, int num_fields, int on_device)
{
    if (!s) { return SPHB_ERR_ARG; }
    if (!s->uploaded) { return SPHB_ERR_STATE; }
    SPHB_TRY(simimpl::waitLateFields(*s, true)); // a previous load's late fields, before this one's replace them
    SPHB_TRY(importConserved(*s, fields, num_fields, on_device != 0, true));
    return simimpl::finishLoad(*s);
}

extern "C" int sphb_sim_store_fields(sphb_sim* s, const sphb_field* fields, int num_fields, int on_device)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    if (!s || !fields || num_fields <= 0) { return SPHB_ERR_ARG; }
    for (int q = 0; q < num_fields; ++q)
    {
        const sphb_field& d = fields[q];
        void* ptr           = nullptr;
        int kind            = 0;
        if (!d.name || !d.data || !validDtype(d.dtype)) { return SPHB_ERR_ARG; }
        if (!simimpl::findField(*s, d.name, &ptr, &kind)) { return SPHB_ERR_ARG; }
        int src = dtypeOfKind(*s, kind);
        if ((src == SPHB_U64) != (d.dtype == SPHB_U64)) { return SPHB_ERR_ARG; } // ids and keys stay 64-bit
        if (on_device)
        {
            SPHB_TRY(convert(ptr, src, d.data, d.dtype, s->n, s->stream));
            continue;
        }
        const void* from = ptr;
        if (src != d.dtype)
        {
            SPHB_TRY(s->typedStage.reserve(s->n * 8));
            SPHB_TRY(convert(ptr, src, s->typedStage.data(), d.dtype, s->n, s->stream));
            from = s->typedStage.data();
        }
        SPHB_CUDA_TRY(cudaMemcpyAsync(d.data, from, s->n * widthOf(d.dtype), cudaMemcpyDeviceToHost, s->stream));
    }
    SPHB_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return SPHB_OK;
}

namespace sphb
{
namespace
{
//! an output field of sphb_sim_step_fields: the caller's descriptor and the element type of the device buffer
struct OutField
{
    const sphb_field* d;
    int src;
    bool done;
};

/*! the device buffer of an output field at the moment of its copy: a reordering sync swaps the field buffers, so the
 *  pointer is looked up after the stages that may swap them, never before the step */
void* outBuffer(sphb_sim& s, const OutField& o)
{
    void* ptr = nullptr;
    int kind  = 0;
    return simimpl::findField(s, o.d->name, &ptr, &kind) ? ptr : nullptr;
}

/*! start the device-to-host copies of the named output fields on the copy stream, after the compute stream's work
 *  so far (their values are final: the step changes them no more). Converted fields go through their own staging
 *  slot of s.earlyStage. */
int exportEarly(sphb_sim& s, std::vector<OutField>& out, std::initializer_list<const char*> names, size_t& slot)
{
    SPHB_CUDA_TRY(cudaEventRecord(s.copyFork, s.stream));
    SPHB_CUDA_TRY(cudaStreamWaitEvent(s.copyStream, s.copyFork, 0));
    for (const char* name : names)
    {
        for (auto& o : out)
        {
            if (o.done || std::strcmp(o.d->name, name) != 0) { continue; }
            const void* from = outBuffer(s, o);
            if (!from) { return kErrArg; }
            if (o.src != o.d->dtype)
            {
                char* stage = s.earlyStage.data() + slot * s.n * 8;
                ++slot;
                SPHB_TRY(convert(from, o.src, stage, o.d->dtype, s.n, s.copyStream));
                from = stage;
            }
            SPHB_CUDA_TRY(cudaMemcpyAsync(o.d->data, from, s.n * widthOf(o.d->dtype), cudaMemcpyDeviceToHost,
                                          s.copyStream));
            o.done = true;
        }
    }
    return kOk;
}
/*! h as the end-of-step update will leave it: it depends only on nc and h, both final after the neighbour search, so
 *  it is computed now into a staging slot and copied out on the copy stream while the J-loops run */
int exportH(sphb_sim& s, std::vector<OutField>& out, size_t& slot)
{
    for (auto& o : out)
    {
        if (o.done || std::strcmp(o.d->name, "h") != 0) { continue; }
        char* stage = s.earlyStage.data() + slot * s.n * 8;
        ++slot;
        SPHB_TRY(predictH(s.n, s.p.ng0, s.nc.data(), s.f[fH].data(), stage, o.d->dtype, s.stream));
        SPHB_CUDA_TRY(cudaEventRecord(s.copyFork, s.stream));
        SPHB_CUDA_TRY(cudaStreamWaitEvent(s.copyStream, s.copyFork, 0));
        SPHB_CUDA_TRY(cudaMemcpyAsync(o.d->data, stage, s.n * widthOf(o.d->dtype), cudaMemcpyDeviceToHost,
                                      s.copyStream));
        o.done = true;
    }
    return kOk;
}

/*! the outputs left after the step: the fields in their own type are copied straight from their buffers on the copy
 *  stream while the compute stream converts the others into their staging slots; the converted ones follow */
int exportFinal(sphb_sim& s, std::vector<OutField>& out, size_t& slot)
{
    SPHB_CUDA_TRY(cudaEventRecord(s.copyFork, s.stream));
    SPHB_CUDA_TRY(cudaStreamWaitEvent(s.copyStream, s.copyFork, 0));
    std::vector<std::pair<OutField*, const char*>> converted;
    for (auto& o : out)
    {
        if (o.done) { continue; }
        const void* from = outBuffer(s, o);
        if (!from) { return kErrArg; }
        if (o.src == o.d->dtype)
        {
            SPHB_CUDA_TRY(cudaMemcpyAsync(o.d->data, from, s.n * widthOf(o.d->dtype), cudaMemcpyDeviceToHost,
                                          s.copyStream));
        }
        else
        {
            char* stage = s.earlyStage.data() + slot * s.n * 8;
            ++slot;
            SPHB_TRY(convert(from, o.src, stage, o.d->dtype, s.n, s.stream));
            converted.push_back({&o, stage});
        }
        o.done = true;
    }
    if (converted.empty()) { return kOk; }
    SPHB_CUDA_TRY(cudaEventRecord(s.copyFork, s.stream));
    SPHB_CUDA_TRY(cudaStreamWaitEvent(s.copyStream, s.copyFork, 0));
    for (const auto& c : converted)
    {
        SPHB_CUDA_TRY(cudaMemcpyAsync(c.first->d->data, c.second, s.n * widthOf(c.first->d->dtype),
                                      cudaMemcpyDeviceToHost, s.copyStream));
    }
    return kOk;
}
} // namespace
} // namespace sphb

extern "C" int sphb_sim_step_fields(sphb_sim* s, const sphb_field* in, int num_in, const sphb_field* out,
                                    int num_out)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    if (!s || !in || !out || num_in <= 0 || num_out <= 0) { return SPHB_ERR_ARG; }
    if (!s->uploaded) { return SPHB_ERR_STATE; }
    if (s->bdt) { return SPHB_ERR_STATE; }
    std::vector<OutField> outs;
    for (int q = 0; q < num_out; ++q)
    {
        const sphb_field& d = out[q];
        void* ptr           = nullptr;
        int kind            = 0;
        if (!d.name || !d.data || !validDtype(d.dtype)) { return SPHB_ERR_ARG; }
        if (!simimpl::findField(*s, d.name, &ptr, &kind)) { return SPHB_ERR_ARG; }
        int src = dtypeOfKind(*s, kind);
        if ((src == SPHB_U64) != (d.dtype == SPHB_U64)) { return SPHB_ERR_ARG; }
        outs.push_back({out + q, src, false});
    }
    // one staging slot per converted output: their copies run while later conversions and kernels do
    size_t numConverted = 0;
    for (const auto& o : outs)
    {
        numConverted += o.src != o.d->dtype ? 1 : 0;
    }
    SPHB_TRY(s->earlyStage.reserve((numConverted + 1) * s->n * 8));
    SPHB_TRY(importConserved(*s, in, num_in, false, true));
    SPHB_TRY(simimpl::finishLoad(*s));
    size_t slot = 0;
    // on an error return, the copies already started still finish before the call returns
    auto fail = [&](int rc) {
        cudaStreamSynchronize(s->copyStream);
        cudaStreamSynchronize(s->stream);
        return rc;
    };
    for (int stage = sSync; stage <= sConserved; ++stage)
    {
        int rc = simimpl::runStage(*s, stage);
        // m and the ids are final once the sync has ordered them, alpha once the AV switches have updated it. m and
        // the ids are copied out from IAD on, when the loaded fields have arrived: earlier, the two directions would
        // share the link while the step waits for the loaded fields
        if (rc == kOk && stage == sNeighbors) { rc = exportH(*s, outs, slot); }
        if (rc == kOk && stage == sIad) { rc = exportEarly(*s, outs, {"m", "id"}, slot); }
        if (rc == kOk && stage == sAV) { rc = exportEarly(*s, outs, {"alpha"}, slot); }
        if (rc != kOk) { return fail(rc); }
    }
    if (int rc = sphb_sim_integrate(s); rc != SPHB_OK) { return fail(rc); }
    if (int rc = exportFinal(*s, outs, slot); rc != kOk) { return fail(rc); }
    SPHB_CUDA_TRY(cudaStreamSynchronize(s->copyStream));
    SPHB_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return SPHB_OK;
}

extern "C" int sphb_sim_bind_fields(sphb_sim* s, const sphb_field* fields, int num_fields)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    if (!s || !fields || num_fields <= 0) { return SPHB_ERR_ARG; }
    if (s->bdt || s->p.av_clean) { return SPHB_ERR_STATE; }
    std::vector<sphb_sim::Binding> b;
    for (int q = 0; q < num_fields; ++q)
    {
        const sphb_field& d = fields[q];
        if (!d.name || !d.data || !validDtype(d.dtype) || !bindableName(*s, d.name, d.dtype)) { return SPHB_ERR_ARG; }
        b.push_back({d.name, d.data, d.dtype});
    }
    s->bound = std::move(b);
    // a bound dataset starts like an upload: trees from scratch, first-call convergence, no skin rows
    return simimpl::finishUpload(*s);
}

extern "C" int sphb_dataset_xmass(sphb_sim* s, size_t first, size_t last, const sphb_box* box)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    SPHB_TRY(boundEntry(s, first, last));
    if (!box) { return SPHB_ERR_ARG; }
    for (int k = 0; k < 3; ++k)
    {
        if (!(box->hi[k] > box->lo[k]) || (box->periodic[k] != 0) != (s->hbox.periodic[k] != 0)) { return SPHB_ERR_ARG; }
    }
    s->hbox          = *box;
    s->box           = makeDevBox(*box);
    s->boxFromCaller = true;
    // ids first: if the caller's order changed since the last call, reused candidate rows are dropped
    const sphb_sim::Binding* id = boundField(*s, "id");
    if (!id) { return SPHB_ERR_ARG; }
    SPHB_TRY(convert(id->data, SPHB_U64, s->idAlt.data(), SPHB_U64, s->n, s->stream));
    SPHB_TRY(simimpl::finishLoad(*s));
    SPHB_TRY(importBound(*s, {"x", "y", "z", "h", "m"}));
    SPHB_TRY(simimpl::runStage(*s, sSync));
    if (!s->lastSyncIdentity)
    {
        std::fprintf(stderr, "sphb200: the bound particles are not in the SFC order of the given box\n");
        s->skinValid = false;
        return SPHB_ERR_STATE;
    }
    SPHB_TRY(simimpl::runStage(*s, sNeighbors));
    SPHB_TRY(simimpl::runStage(*s, sXMass));
    SPHB_TRY(exportBound(*s, {"h", "nc", "xm"}));
    SPHB_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return SPHB_OK;
}

extern "C" int sphb_dataset_ve_def_gradh(sphb_sim* s, size_t first, size_t last, const sphb_box* box)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    SPHB_TRY(boundEntry(s, first, last));
    SPHB_TRY(checkBox(*s, box));
    SPHB_TRY(importBound(*s, {"xm", "temp", "vx", "vy", "vz"}));
    SPHB_TRY(simimpl::runStage(*s, sVeDefGradh));
    SPHB_TRY(exportBound(*s, {"kx", "gradh"}));
    SPHB_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return SPHB_OK;
}

extern "C" int sphb_ideal_gas_eos(size_t first, size_t last, double mui, double gamma, const sphb_field* fields,
                                  int num_fields, void* stream)
{
    if (last < first || !(mui > 0.0) || !(gamma > 1.0) || !fields || num_fields <= 0) { return SPHB_ERR_ARG; }
    for (int q = 0; q < num_fields; ++q)
    {
        if (fields[q].data && fields[q].dtype != SPHB_F32 && fields[q].dtype != SPHB_F64) { return SPHB_ERR_ARG; }
    }
    auto get = [&](const char* name, const void** p, int* t) {
        const sphb_field* d = findDesc(fields, num_fields, name);
        *p                  = d ? d->data : nullptr;
        *t                  = d ? d->dtype : 0;
    };
    EosArrays a{};
    get("temp", &a.temp, &a.tTemp);
    get("u", &a.u, &a.tU);
    get("m", &a.m, &a.tM);
    get("kx", &a.kx, &a.tKx);
    get("xm", &a.xm, &a.tXm);
    get("gradh", &a.gradh, &a.tGradh);
    const void* out[4];
    get("prho", &out[0], &a.tPrho);
    get("c", &out[1], &a.tC);
    get("rho", &out[2], &a.tRho);
    get("p", &out[3], &a.tP);
    a.prho = const_cast<void*>(out[0]);
    a.c    = const_cast<void*>(out[1]);
    a.rho  = const_cast<void*>(out[2]);
    a.p    = const_cast<void*>(out[3]);
    if ((!a.temp && !a.u) || !a.m || !a.kx || !a.xm || !a.gradh || !a.prho || !a.c) { return SPHB_ERR_ARG; }
    if (last == first) { return SPHB_OK; }
    double cv = 8.317e7 / mui / (gamma - 1.0);
    auto st   = static_cast<cudaStream_t>(stream);
    idealGasEosKernel<<<ceilDiv(last - first, 256), 256, 0, st>>>(first, last, cv, gamma, a);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return SPHB_OK;
}

extern "C" int sphb_dataset_iad_divv_curlv(sphb_sim* s, size_t first, size_t last, const sphb_box* box)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    SPHB_TRY(boundEntry(s, first, last));
    SPHB_TRY(checkBox(*s, box));
    SPHB_TRY(importBound(*s, {"vx", "vy", "vz", "xm", "kx", "c", "prho"}));
    SPHB_TRY(packRecords(*s, false));
    SPHB_TRY(simimpl::runStage(*s, sIad));
    SPHB_TRY(exportBound(*s, {"c11", "c12", "c13", "c22", "c23", "c33", "divv", "curlv"}));
    SPHB_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return SPHB_OK;
}

extern "C" int sphb_dataset_av_switches(sphb_sim* s, size_t first, size_t last, const sphb_box* box, double min_dt)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    SPHB_TRY(boundEntry(s, first, last));
    SPHB_TRY(checkBox(*s, box));
    if (!(min_dt > 0.0)) { return SPHB_ERR_ARG; }
    SPHB_TRY(importBound(*s, {"vx", "vy", "vz", "xm", "kx", "c", "prho", "c11", "c12", "c13", "c22", "c23", "c33",
                              "divv", "alpha"}));
    SPHB_TRY(packRecords(*s, true));
    s->minDt = min_dt;
    SPHB_TRY(simimpl::runStage(*s, sAV));
    SPHB_TRY(exportBound(*s, "alpha"));
    SPHB_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return SPHB_OK;
}

extern "C" int sphb_dataset_momentum_energy(sphb_sim* s, size_t first, size_t last, const sphb_box* box,
                                            float* min_dt_courant)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    SPHB_TRY(boundEntry(s, first, last));
    SPHB_TRY(checkBox(*s, box));
    SPHB_TRY(importBound(*s, {"vx", "vy", "vz", "xm", "kx", "c", "prho", "c11", "c12", "c13", "c22", "c23", "c33",
                              "divv", "alpha"}));
    SPHB_TRY(packRecords(*s, true));
    SPHB_TRY(setWords(s->reduce.data() + 1, 1, orderedBits(INFINITY), 0, s->stream));
    SPHB_TRY(simimpl::runStage(*s, sMomentum));
    SPHB_TRY(exportBound(*s, {"ax", "ay", "az", "du"}));
    unsigned long long bits = 0;
    SPHB_CUDA_TRY(cudaMemcpyAsync(&bits, s->reduce.data() + 1, sizeof(bits), cudaMemcpyDeviceToHost, s->stream));
    SPHB_CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (min_dt_courant) { *min_dt_courant = float(fromOrderedBits(bits)); }
    return SPHB_OK;
}

extern "C" int sphb_dataset_positions(sphb_sim* s, size_t first, size_t last, double dt, double dt_m1,
                                      const sphb_box* box)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    SPHB_TRY(boundEntry(s, first, last));
    SPHB_TRY(checkBox(*s, box));
    if (!(dt > 0.0) || !(dt_m1 > 0.0)) { return SPHB_ERR_ARG; }
    SPHB_TRY(importBound(*s, {"x", "y", "z", "vx", "vy", "vz", "x_m1", "y_m1", "z_m1", "temp", "du", "du_m1", "ax",
                              "ay", "az"}));
    SPHB_TRY(simimpl::positions(*s, dt, dt_m1));
    SPHB_TRY(exportBound(*s, {"x", "y", "z", "vx", "vy", "vz", "x_m1", "y_m1", "z_m1", "temp", "du_m1"}));
    SPHB_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return SPHB_OK;
}

extern "C" int sphb_dataset_update_h(sphb_sim* s, size_t first, size_t last, unsigned ng0)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    SPHB_TRY(boundEntry(s, first, last));
    if (ng0 == 0) { return SPHB_ERR_ARG; }
    SPHB_TRY(importBound(*s, {"nc", "h"}));
    SPHB_CUDA_TRY(cudaMemsetAsync(s->status.data() + 1, 0, sizeof(unsigned), s->stream));
    SPHB_TRY(launchUpdateH(s->n, ng0, s->nc.data(), s->f[fH].data(), s->keys.data(), s->status.data() + 1,
                           s->stream));
    SPHB_TRY(exportBound(*s, "h"));
    SPHB_TRY(exportBound(*s, "keys", true));
    unsigned flag = 0;
    SPHB_CUDA_TRY(cudaMemcpyAsync(&flag, s->status.data() + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, s->stream));
    SPHB_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return flag ? SPHB_ERR_NOT_CONVERGED : SPHB_OK;
}
