// nb6_common.cuh -- shared device and host helpers of libnb6b200 (sm_100a).
//
// Device side: hi/lo float split of FP64 coordinates, double-single (two
// float) compensated sums, and the bulk-copy (TMA, non-tensor, no multicast)
// + mbarrier pipeline primitives with bounded waits.  Every wait in this
// library has an iteration limit; on expiry it records an error code in the
// device status word and the kernel returns instead of hanging.
//
// Host side: CUDA_CHECK, grow-only device / pinned buffers, the library's
// status word, and wall-clock timers for the reference-style profile lines.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <sys/time.h>

// ----------------------------------------------------------------------------
// status codes written by kernels into the device status word
// ----------------------------------------------------------------------------
enum Nb6Status : int {
    NB6_OK = 0,
    NB6_ERR_WAIT_TIMEOUT = 1,   // an mbarrier wait ran out of iterations
    NB6_ERR_BAD_ARG = 2,        // host-side argument check failed
    NB6_ERR_NAN_INPUT = 3,      // NaN found in an input array
    NB6_ERR_CUDA = 4,           // a CUDA runtime call failed
    NB6_ERR_NOT_OPEN = 5,       // call before *_open_
    NB6_ERR_TOO_LARGE = 6,      // size beyond the opened capacity
};

#define NB6_DEV __device__ __forceinline__

// ----------------------------------------------------------------------------
// numerics
// ----------------------------------------------------------------------------

// Split a double into hi = fl32(x), lo = fl32(x - hi).  For two nearby
// coordinates the hi difference is exact (Sterbenz), so
// (xjH - xiH) + (xjL - xiL) is the FP64 difference rounded to FP32 within
// one ulp.
NB6_DEV void split_hl(double x, float &hi, float &lo) {
    hi = __double2float_rn(x);
    lo = __double2float_rn(x - (double)hi);
}

// Regular-force j set in HBM, written by the send/predict pack kernels.
// Two layouts of the same data:
//   posH/posL/vel  float4 per j: (xH,yH,zH,m), (xL,yL,zL,0), (vx,vy,vz,0) --
//                  read per j by the j-parallel kernel;
//   comp           10 float arrays of npad entries, component-major
//                  (xH,yH,zH,m,xL,yL,zL,vx,vy,vz) -- tiles of it are bulk-copied
//                  to shared memory so that one LDS.128 yields 4 consecutive j
//                  of one component, the operand shape of packed f32x2 math.
// Padding slots (j >= n) are massless and far away: never neighbours.
constexpr int NB6_NCOMP = 10;

struct JSetOut {
    float4 *posH, *posL, *vel;
    float *comp;
    double *compd;  // FP64 positions, component-major (x, y, z) x npad
    size_t npad;
};

NB6_DEV void write_j(const JSetOut &o, size_t j, bool real, double x0, double x1, double x2,
                     double m, double v0, double v1, double v2) {
    float4 h, l, v;
    if (real) {
        split_hl(x0, h.x, l.x);
        split_hl(x1, h.y, l.y);
        split_hl(x2, h.z, l.z);
        h.w = (float)m;
        l.w = 0.f;
        v = make_float4((float)v0, (float)v1, (float)v2, 0.f);
    } else {
        h = make_float4(1.0e15f, 1.0e15f, 1.0e15f, 0.f);
        l = make_float4(0.f, 0.f, 0.f, 0.f);
        v = l;
    }
    o.posH[j] = h;
    o.posL[j] = l;
    o.vel[j] = v;
    float *c = o.comp + j;
    const size_t s = o.npad;
    c[0] = h.x;
    c[s] = h.y;
    c[2 * s] = h.z;
    c[3 * s] = h.w;
    c[4 * s] = l.x;
    c[5 * s] = l.y;
    c[6 * s] = l.z;
    c[7 * s] = v.x;
    c[8 * s] = v.y;
    c[9 * s] = v.z;
    double *d = o.compd + j;
    d[0] = real ? x0 : 1.0e15;
    d[s] = real ? x1 : 1.0e15;
    d[2 * s] = real ? x2 : 1.0e15;
}

// Error-free sum (Knuth TwoSum): s + e == a + b exactly.
NB6_DEV void two_sum(float a, float b, float &s, float &e) {
    s = __fadd_rn(a, b);
    float bb = __fsub_rn(s, a);
    e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}

// Fold an FP32 partial p into the double-single accumulator (hi, lo).
NB6_DEV void ds_fold(float &hi, float &lo, float p) {
    float s, e;
    two_sum(hi, p, s, e);
    hi = s;
    lo = __fadd_rn(lo, e);
}

// rsqrt.approx (MUFU) followed by the scaled Newton step
// y1 = y0 * (3 - r2*y0*y0); the result is 2/sqrt(r2) (the factor 2 is folded
// into the end-of-sum scalings, which are exact powers of two).
NB6_DEV float rsqrt2_nr(float r2) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(r2));
    float a = r2 * y;
    float b = __fmaf_rn(-a, y, 3.0f);
    return y * b;
}

// ----------------------------------------------------------------------------
// bulk copy + mbarrier (PTX ISA 8.x: cp.async.bulk.shared::cluster.global,
// mbarrier.try_wait.parity).  Single-CTA use only; no multicast anywhere.
// ----------------------------------------------------------------------------
NB6_DEV uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

NB6_DEV void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(count)
                 : "memory");
}

NB6_DEV void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

NB6_DEV void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile(
        "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
        "r"(bytes)
        : "memory");
}

// Plain arrival (count 1) on an mbarrier.
NB6_DEV void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// 1-D bulk copy global -> shared, completion counted on `bar` (bytes must be a
// multiple of 16, both addresses 16-byte aligned).
NB6_DEV void bulk_g2s(void *sdst, const void *gsrc, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
        "[%0], [%1], %2, [%3];" ::"r"(smem_u32(sdst)),
        "l"(gsrc), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

NB6_DEV uint64_t globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

NB6_DEV bool mbar_try(uint64_t *bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// Wait for `parity` with a wall-clock budget; false on expiry.
NB6_DEV bool mbar_wait_timed(uint64_t *bar, uint32_t parity, uint64_t budget_ns) {
    uint64_t t0 = 0;
    for (uint32_t it = 0;; ++it) {
        if (mbar_try(bar, parity)) return true;
        if ((it & 63u) == 63u) {
            const uint64_t now = globaltimer();
            if (t0 == 0) t0 = now;
            else if (now - t0 > budget_ns) return false;
        }
    }
}

// Order-preserving map of a float to an unsigned (for atomicMin/Max of
// positions) and back.
NB6_DEV unsigned f2ord(float f) {
    const unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
NB6_DEV float ord2f(unsigned u) { return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u); }

// The 10 low bits of v spread to every third bit (one axis of a 30-bit
// Morton key).
NB6_DEV unsigned spread10(unsigned v) {
    v &= 1023u;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

// Warp-level inclusive max/sum helpers used by the finalize kernels.
NB6_DEV double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Record the first error code (keeps the earliest failure).
NB6_DEV void set_status(int *status, int code) { atomicCAS(status, 0, code); }

// ----------------------------------------------------------------------------
// host helpers
// ----------------------------------------------------------------------------
#define NB6_CUDA_CHECK(call)                                                       \
    do {                                                                           \
        cudaError_t err__ = (call);                                                \
        if (err__ != cudaSuccess) {                                                \
            fprintf(stderr, "libnb6b200: CUDA error %s at %s:%d: %s\n",            \
                    cudaGetErrorName(err__), __FILE__, __LINE__,                   \
                    cudaGetErrorString(err__));                                    \
            nb6_fatal(NB6_ERR_CUDA);                                               \
        }                                                                          \
    } while (0)

// Results of a segmented regular-force call left on the device for a
// following kernel (see regular_seg_on_device): outf [ni][8] = (acc, jrk,
// pot, proposal), outl [ni][W] = [nnb, ids relative to the segment], and the
// predicted FP64 j set (m, x, v) the call used.
struct RegDeviceOut {
    const double *outf;
    const int *outl;
    int W;
    const double *jm, *jx, *jv;
};
bool regular_seg_on_device(int ni, int *iseg, double *h2, double *dtr, double (*xi)[3], double (*vi)[3], int lmax,
                           int nnbmax, int mflag, int nseg, int *seg_j0, RegDeviceOut *out);

extern "C" int nb6_last_status_();
void nb6_fatal(int code);          // records status and aborts unless disabled
void nb6_set_host_status(int code); // records status without aborting
int nb6_device_id();               // device picked at devinit (GPU_LIST / NB_GPU_DEVICE)
void nb6_devinit_once(int irank);
cudaStream_t nb6_stream();         // the library's stream (non-blocking)
int *nb6_dev_status();             // device status word (zeroed at init)
class CopyPool;
CopyPool &nb6_copy_pool();         // host copy threads, started on first use (copy_pool.h)
void nb6_lib_opened();             // gpunb_open_ / irr_simd_open_
void nb6_lib_closed();             // their closes: the pool stops with the last
int nb6_check_dev_status();        // read (and clear) after a stream sync
void nb6_status_fetch(cudaStream_t st);  // enqueue the status copy before that sync
bool nb6_uva();                    // device reads/writes pinned host memory in place
int nb6_num_sms();

static inline double nb6_wtime() {
    struct timeval tv;
    gettimeofday(&tv, nullptr);
    return tv.tv_sec + 1.e-6 * tv.tv_usec;
}

// Grow-only device buffer.
template <class T> struct DevBuf {
    T *ptr = nullptr;
    size_t cap = 0;
    void reserve(size_t n);
    void release();
};

// Grow-only pinned host buffer.
template <class T> struct HostBuf {
    T *ptr = nullptr;
    size_t cap = 0;
    void reserve(size_t n);
    void release();
};

template <class T> void DevBuf<T>::reserve(size_t n) {
    if (n <= cap) return;
    if (ptr) NB6_CUDA_CHECK(cudaFree(ptr));
    size_t want = n + n / 4 + 64;
    NB6_CUDA_CHECK(cudaMalloc((void **)&ptr, want * sizeof(T)));
    cap = want;
}
template <class T> void DevBuf<T>::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
}
template <class T> void HostBuf<T>::reserve(size_t n) {
    if (n <= cap) return;
    if (ptr) NB6_CUDA_CHECK(cudaFreeHost(ptr));
    size_t want = n + n / 4 + 64;
    NB6_CUDA_CHECK(cudaMallocHost((void **)&ptr, want * sizeof(T)));
    cap = want;
}
template <class T> void HostBuf<T>::release() {
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    cap = 0;
}
